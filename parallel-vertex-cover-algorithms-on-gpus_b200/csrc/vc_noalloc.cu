// vc_noalloc.cu -- exact MVC / PVC of one small graph without allocating memory.
//
// Who needs this: callers that may not call cudaMalloc -- code running under a
// framework that owns all device memory through its own pool, real-time or
// embedded hosts that forbid allocation after start-up, and library callers
// that must not trigger an allocation's implicit device synchronisation.  They
// pass their own device buffers for the graph and the result; every piece of
// scratch memory the search needs (control words, the graph's state, the cover
// bitmap and the work-sharing ring) lives in one file-scope __device__ array of
// fixed size, which every GPU that loads this library holds until the process
// exits.
//
// Limits: graphs of at most kNoAllocMaxVertices (255) vertices, one graph per
// call, a ring of kRingSlots donated subtrees; kScratchBytes (256 KiB) of device
// memory per GPU.  Larger graphs are rejected with VC_ERR_TOO_LARGE.
//
// The array is shared by every call on a device and keeps the previous call's
// contents: each call first clears what must start at zero (control words,
// state, cover, ring sequence numbers).  Calls whose work overlaps on the GPU
// (different streams, or another host thread) race on the array and must be
// serialised by the caller.  The first call on a device performs the one-time
// set-up for that device (cudaGetSymbolAddress of the array with that device
// current, kernel attributes, occupancy); make that first call before any
// stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "vc_dense.cuh"
#include "vc_host.h"
#include "vcgpu.h"

using namespace vcg;

namespace vcn {

constexpr uint32_t kNoAllocMaxVertices = 255;
// A search unit gives a record to the ring only while more CTAs are idle than
// records are queued, so at most one record per CTA is ever pending: the grid
// is at most 4 CTAs per SM (1024 threads), 592 on a B200, well inside the ring.
constexpr uint32_t kRingSlots = 4096;
constexpr uint32_t kMaxStride = 12;  // 4 header words + 8 bitmap words
constexpr size_t kScratchBytes = 256 * 1024;

struct Scratch {
    unsigned long long ctl[kCtlWords];
    InstDesc desc;
    InstState st;
    uint32_t cover[8];
    unsigned long long seq[kRingSlots];
    uint32_t data[kRingSlots * kMaxStride];
};
static_assert(sizeof(Scratch) <= kScratchBytes, "scratch layout exceeds the static array");

// The only device memory this entry point uses besides the caller's buffers.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

template <int NW, unsigned NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_dense_noalloc(Params P)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t cp_hdr[kCpHdrWords];
    const uint32_t su_per_cta = NT / 32;
    uint32_t *adj = reinterpret_cast<uint32_t *>(smem);
    uint8_t *ws0 = smem + dense_adj_bytes(NW);
    CtaPool cp;
    cp.su = su_per_cta;
    cp.lp = P.cta_slots;
    cp.hdr = cp_hdr;
    cp.state = reinterpret_cast<uint32_t *>(ws0 + (size_t)su_per_cta * P.su_bytes);
    cp.data = cp.state + ((P.cta_slots + 3) / 4 * 4);
    for (uint32_t i = threadIdx.x; i < kCpHdrWords; i += blockDim.x) cp_hdr[i] = (i == kCpStaged) ? kNone : 0u;
    for (uint32_t i = threadIdx.x; i < P.cta_slots; i += blockDim.x) cp.state[i] = 0;
    __syncthreads();
    su_main_dense<NW>(P, ws0 + (size_t)WarpG::su_local() * P.su_bytes, adj, cp);
}

// Clears the shared array for a new call and writes the graph's descriptor.
__global__ void k_noalloc_reset(Scratch *s, InstDesc d)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kRingSlots) s->seq[i] = i;
    if (i < kCtlWords) s->ctl[i] = 0;
    if (i < 8) s->cover[i] = 0;
    if (i == 0) {
        s->desc = d;
        InstState st;
        st.best = d.init_best;
        st.act = 1;
        st.flags = 0;
        st.lock = 0;
        st.cover_size = kNone;
        st.pad = 0;
        st.nodes = 0;
        st.t_done = 0;
        s->st = st;
    }
}

// result words: status, size, decision, has_cover, nodes (lo, hi), 0, 0
__global__ void k_noalloc_finish(const Scratch *s, uint32_t ub, uint32_t *result, uint32_t *cover)
{
    const uint32_t i = threadIdx.x;
    const InstState &st = s->st;
    const InstDesc &d = s->desc;
    const bool has_cover = st.cover_size != kNone;
    if (cover && i < d.nw) cover[i] = has_cover ? s->cover[i] : 0u;
    if (i != 0) return;
    uint32_t status;
    if (st.flags & kBadGraph) status = VC_ERR_INVALID;
    else if (st.flags & kError) status = VC_ERR_INTERNAL;
    else if (st.flags & kBudget) status = VC_BUDGET;
    else if ((st.flags & kCut) || !(st.flags & kDone)) status = s->ctl[kAbort] ? VC_TIMEOUT : VC_ERR_INTERNAL;
    else status = VC_OK;
    uint32_t size, decision;
    if (d.mode == kModeMVC) {
        decision = 1;
        size = st.best < d.init_best ? st.best : (ub ? ub : d.n);
    } else {
        decision = (st.flags & kFound) ? 1u : 0u;
        size = decision ? st.cover_size : 0u;
    }
    result[0] = status;
    result[1] = size;
    result[2] = decision;
    result[3] = has_cover ? 1u : 0u;
    result[4] = (uint32_t)(st.nodes & 0xffffffffull);
    result[5] = (uint32_t)(st.nodes >> 32);
    result[6] = 0;
    result[7] = 0;
}

struct Setup {
    bool ready = false;
    Scratch *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
    uint32_t grid[3] = {0, 0, 0}, smem[3] = {0, 0, 0}, su_bytes[3] = {0, 0, 0}, stride[3] = {0, 0, 0};
};
static std::mutex g_setup_mu;
static Setup g_setup[64];

static uint32_t pool_bytes(uint32_t slots, uint32_t stride)
{
    return 4u * ((slots + 3) / 4 * 4) + 4u * slots * stride;
}

template <int NW>
static cudaError_t setup_variant(Setup &su, int idx, int smem_optin)
{
    const uint32_t su_bytes = dense_workspace_bytes(NW);
    const uint32_t stride = (4 + NW + 3) / 4 * 4;
    const uint32_t smem = dense_adj_bytes(NW) + 8 * su_bytes + pool_bytes(16, stride);
    if ((int)smem + 1024 > smem_optin) return cudaErrorInvalidConfiguration;
    auto fn = k_dense_noalloc<NW, 256>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    su.grid[idx] = (uint32_t)per_sm * (uint32_t)su.sms;
    su.smem[idx] = smem;
    su.su_bytes[idx] = su_bytes;
    su.stride[idx] = stride;
    return cudaSuccess;
}

// One-time set-up for the current device (called with that device current).
static vc_status setup_device(int dev, Setup **out)
{
    std::lock_guard<std::mutex> lk(g_setup_mu);
    Setup &su = g_setup[dev];
    if (!su.ready) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return VC_ERR_CUDA;
        su.scratch = reinterpret_cast<Scratch *>(p);
        int smem_optin = 0, coop = 0;
        if (cudaDeviceGetAttribute(&su.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
            return VC_ERR_CUDA;
        if (setup_variant<2>(su, 0, smem_optin) != cudaSuccess || setup_variant<4>(su, 1, smem_optin) != cudaSuccess ||
            setup_variant<8>(su, 2, smem_optin) != cudaSuccess)
            return VC_ERR_CUDA;
        su.ready = true;
    }
    *out = &su;
    return VC_OK;
}

}  // namespace vcn

using namespace vcn;

// Solves one graph of at most 255 vertices with no device or host allocation.
// g->row_ptr / g->col must be device pointers and req->flags must include
// VC_FLAG_DEVICE_INPUT.  Runs asynchronously on req->stream (NULL = the legacy
// default stream) and writes 8 words to the caller's device buffer d_result
// (status, size, decision, has_cover, tree nodes low, high, 0, 0) and, when
// d_cover is not NULL, the cover as ceil(n/32) bitmap words (bit v of word v/32
// set = v in the cover).  Values have the meaning of vc_result's fields.
extern "C" vc_status vc_solve_noalloc(const vc_csr *g, const vc_request *req, uint32_t *d_result, uint32_t *d_cover)
{
    vch::DeviceGuard dg;
    if (!g || !req || !d_result) return VC_ERR_INVALID;
    if (!(req->flags & VC_FLAG_DEVICE_INPUT)) return VC_ERR_INVALID;
    if (req->instance != VC_MVC && req->instance != VC_PVC) return VC_ERR_INVALID;
    if (g->n == 0 || !g->row_ptr || (g->m && !g->col)) return VC_ERR_INVALID;
    if (g->n > kNoAllocMaxVertices) return VC_ERR_TOO_LARGE;
    int dev = req->device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return VC_ERR_CUDA;
    if (dev >= 64) return VC_ERR_INVALID;
    if (cudaSetDevice(dev) != cudaSuccess) return VC_ERR_NO_DEVICE;
    Setup *su = nullptr;
    vc_status st = setup_device(dev, &su);
    if (st != VC_OK) return st;
    cudaStream_t stream = (cudaStream_t)req->stream;

    const uint32_t n = g->n;
    const int idx = n <= 64 ? 0 : (n <= 128 ? 1 : 2);
    const uint32_t nw_kernel = idx == 0 ? 2 : (idx == 1 ? 4 : 8);
    InstDesc d;
    d.n = n;
    d.nw = (n + 31) / 32;
    d.row_off = 0;
    d.col_off = 0;
    d.mode = req->instance == VC_PVC ? kModePVC : kModeMVC;
    d.k = req->k < n ? req->k : n;
    const uint32_t ub = req->instance == VC_MVC ? req->ub : 0;
    d.init_best = (d.mode == kModePVC) ? n + 1 : ((ub && ub < n) ? ub : n) + 1;
    d.cover_off = 0;
    d.node_limit = req->node_limit;
    d.key = 0;
    d.m2 = 2ull * g->m < (uint64_t)kNone ? (uint32_t)(2ull * g->m) : kNone;

    // Launches are checked through their own return codes, so an error the
    // caller's earlier work left pending is neither reported nor cleared here.
    Scratch *s = su->scratch;
    {
        void *a[] = {&s, &d};
        if (cudaLaunchKernel((const void *)k_noalloc_reset, dim3((kRingSlots + 255) / 256), dim3(256), a, 0, stream) !=
            cudaSuccess)
            return VC_ERR_CUDA;
    }
    {
        // the caller's CSR is device memory: check its layout before the search
        // reads it (a graph that fails is reported VC_ERR_INVALID)
        const uint32_t *rp = g->row_ptr, *cl = g->col;
        const InstDesc *di = &s->desc;
        InstState *sti = &s->st;
        uint32_t one = 1;
        void *a[] = {&rp, &cl, &di, &sti, &one};
        if (cudaLaunchKernel((const void *)k_check_csr<0>, dim3(1), dim3(256), a, 0, stream) != cudaSuccess)
            return VC_ERR_CUDA;
    }

    Params P;
    memset(&P, 0, sizeof(P));
    P.row_ptr = g->row_ptr;
    P.col = g->col;
    P.inst = &s->desc;
    P.st = &s->st;
    P.covers = s->cover;
    P.count = 1;
    P.num_su = su->grid[idx] * 8;
    P.ctl = s->ctl;
    P.pool_seq = s->seq;
    P.pool_data = s->data;
    P.q_mask = kRingSlots - 1;
    P.stride = su->stride[idx];
    P.np = 32 * nw_kernel;
    P.su_bytes = su->su_bytes[idx];
    P.cta_slots = 16;
    P.gws = nullptr;
    P.stats = nullptr;
    const double tl = req->time_limit_s > 0 ? req->time_limit_s : 300.0;
    P.time_limit_ns = (unsigned long long)(tl * 1e9);
    void *args[] = {&P};
    const void *fn = idx == 0 ? (const void *)k_dense_noalloc<2, 256>
                              : (idx == 1 ? (const void *)k_dense_noalloc<4, 256> : (const void *)k_dense_noalloc<8, 256>);
    if (cudaLaunchCooperativeKernel(fn, dim3(su->grid[idx]), dim3(256), args, su->smem[idx], stream) != cudaSuccess)
        return VC_ERR_CUDA;
    {
        const Scratch *cs = s;
        uint32_t ubv = ub;
        void *a[] = {&cs, &ubv, &d_result, &d_cover};
        if (cudaLaunchKernel((const void *)k_noalloc_finish, dim3(1), dim3(32), a, 0, stream) != cudaSuccess)
            return VC_ERR_CUDA;
    }
    return VC_OK;
}
