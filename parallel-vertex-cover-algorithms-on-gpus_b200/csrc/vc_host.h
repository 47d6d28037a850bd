// vc_host.h -- host-side types shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <mutex>
#include <vector>

#include "vcgpu.h"
#include "vc_types.h"

namespace vch {

// Search units are warps up to this vertex capacity, CTAs above it.
#ifndef VC_WARP_MAX_NP
#define VC_WARP_MAX_NP 1024
#endif
constexpr uint32_t kWarpMaxNP = VC_WARP_MAX_NP;
constexpr uint32_t kMaxVertices = 1u << 26;

// Puts the calling thread's current device back when an entry point returns:
// the library switches devices for its own work, never for its caller.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard()
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;
};

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

struct PinBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
};

// A launch-shape choice for one size class of graphs, set by vc_autotune (or
// vc_set_tuning); `set` = 0 keeps the built-in rules.
struct Tune {
    uint32_t set = 0;
    uint32_t cta_units = 0;   // CSR classes: 1 = one 512-thread CTA per search unit, 0 = warp units
    uint32_t warps = 8;       // warps (search units) per CTA: 2, 4 or 8
    uint32_t pool = 2;        // CTA pool slots (donated subtrees) per warp: 1, 2 or 4
    int32_t ring_bias = 0;    // global-ring donations while idle CTAs minus queued records exceed this
    uint32_t ring_first = 0;  // 1: when a sibling warp and another CTA both wait, the ring gets the subtree
    float nodes_per_s = 0;    // what the calibration measured with this choice
};

// Size classes of the tuner: dense bitsets of 2, 4 and 8 words (n <= 64, 128,
// 255), the wide dense kernel (n <= 640, degrees <= 254), CSR up to 1024
// vertices, CSR above.
constexpr int kTuneClasses = 6;
inline int tune_class(uint32_t nmax, bool wide)
{
    if (nmax <= 64) return 0;
    if (nmax <= 128) return 1;
    if (nmax <= 255) return 2;
    if (wide && nmax <= 640) return 3;
    return nmax <= 1024 ? 4 : 5;
}

struct Plan {
    const void *fn = nullptr;
    uint32_t block = 0, grid = 0, smem = 0;
    uint32_t np = 0, su_bytes = 0, num_su = 0, stride = 0, cta_slots = 0;
    bool global_ws = false;
    bool dense = false;
    bool lanes = false;  // one thread per search unit (vc_lanes.cuh)
};

// Per-device state: one stream, grow-only device and pinned buffers, a lock
// that serialises solves on the device.
struct Ctx {
    int dev = -1;
    int sms = 0;
    int smem_optin = 0;
    int coop = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf rp, col, inst, st, covers, ctl, seq, data, gws, launches;
    PinBuf h_st, h_desc, h_covers;
    unsigned long long h_ctl[vcg::kCtlWords] = {};
    bool stats_on = false;
    bool force_sparse = false;
    Tune tune[kTuneClasses];
    int lanes_mode = 0;  // graphs <= 255 vertices: 0 warp search units (default), 1 lane search units
    DevBuf stats;
    std::vector<unsigned long long> last_stats;
    uint32_t last_num_su = 0;
    Plan last_plan;
    std::mutex mu;
};

struct Job {
    const uint32_t *d_rp = nullptr;
    const uint32_t *d_col = nullptr;
    std::vector<vcg::InstDesc> desc;
    double time_limit_s = 0;
    // results
    std::vector<vcg::InstState> st;
    std::vector<uint32_t> covers;
    float kernel_ms = 0;
    unsigned long long t0 = 0;
    bool aborted = false;
    bool wide = false;  // every graph may take the 20-word dense kernel
    bool half = false;  // every graph may take the 16/32-word dense kernels (16-bit degrees)
    bool dev_input = false;  // the graphs came from the caller's device memory: checked by k_check_csr
    const Tune *tune = nullptr;  // a shape to try instead of the context's table (the tuner's candidates)
    Plan plan;
};

// The largest graph of the wide dense kernel; it also needs every degree <= 254.
constexpr uint32_t kWideMaxN = 640;

// The largest graph of the dense kernels with 16-bit degrees (any degree).
constexpr uint32_t kHalfMaxN = 1024;

// True if a graph of n vertices takes a dense kernel with 16-bit degrees (when
// the byte kernels cannot take it).
inline bool half_ok(uint32_t n) { return n > 255 && n <= kHalfMaxN; }

// True if a graph of n vertices (host row offsets) fits the wide dense kernel.
inline bool wide_ok(uint32_t n, const uint32_t *row_ptr)
{
    if (n > kWideMaxN || !row_ptr) return false;
    for (uint32_t v = 0; v < n; ++v)
        if (row_ptr[v + 1] - row_ptr[v] > 254u) return false;
    return true;
}

struct PlanOpts {
    uint32_t smem_budget = 0;  // bytes per CTA for CSR workspaces, 0 = the device limit
    uint32_t warp_max_np = 0;  // largest capacity given warp units, 0 = kWarpMaxNP
    uint32_t warps = 0;        // warps per CTA with warp_gws, 0 = 8
    bool wide = false;         // graphs of 256..640 vertices may take the wide dense kernel
    bool warp_gws = false;     // warp units with global-memory workspaces
    bool lanes = false;        // graphs <= 255 vertices take the lane kernel
    bool half = false;         // graphs of 256..1024 vertices take the 16-bit-degree dense kernels
    bool team = false;         // CSR kernels walk rows with teams of lanes (average degree >= 4)
    const Tune *tune = nullptr; // the size class's tuned shape, if any
};

Ctx *get_ctx(int dev, vc_status *err);
cudaError_t make_plan(Ctx &c, uint32_t np, uint32_t nmax, Plan &pl, const PlanOpts &o = PlanOpts());
void cap_plan(const Ctx &c, Plan &pl, uint32_t per_sm);
vc_status run_job(Ctx &c, Job &job, cudaStream_t stream);
vc_status fill_result(const Job &job, uint32_t i, uint32_t ub, vc_result *out);
vc_status validate_csr(const vc_csr *g);
vc_status vc_solve_batch_impl(const vc_csr_arena *a, const vc_request *reqs, vc_result *out, const uint32_t *d_rp,
                              const uint32_t *d_col, std::chrono::steady_clock::time_point t0);

}  // namespace vch
