// vc_solver.cu -- host side of libvcgpu.so: the C ABI (include/vcgpu.h), per-device
// contexts with grow-only device buffers, graph validation, launch sizing and
// result collection.  The search itself is vc_search.cuh.
//
// Replaces the host path of the reference's src/main.cu:101-359: device query
// (:101-121), sizing (:122, auxFunctions.cpp:469-578), allocations (:219-269),
// the kernel launch (:300-344) and the read-back (:348-359).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "vc_search.cuh"
#include "vc_dense.cuh"
#include "vc_lanes.cuh"
#include "vc_host.h"
#include "vcgpu.h"

using namespace vcg;

namespace vch {

std::atomic<uint64_t> g_launches{0};

// Resident threads per SM the search kernels are register-limited for
// (1024 -> at most 64 registers per thread, 32 warps per SM).
// Team-walk kernels also come with 768 (80 registers), taken where the extra
// registers cost no resident CTAs (see plan_variant).
#ifndef VC_MIN_THREADS_PER_SM
#define VC_MIN_THREADS_PER_SM 1024
#endif
constexpr unsigned kRoomyThreadsPerSM = 768;

// ---------------------------------------------------------------- kernels
template <class G, unsigned NT, unsigned MinThreads = VC_MIN_THREADS_PER_SM>
__global__ void __launch_bounds__(NT, MinThreads / NT) k_search(Params P)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t cp_hdr[kCpHdrWords];
    if (P.server && threadIdx.x == 0) atomicAdd(&P.ctl[kStarted], 1ull);  // residency check of server lanes
    const uint32_t su_per_cta = NT / G::kSize;
    CtaPool cp;
    cp.su = su_per_cta;
    cp.lp = P.cta_slots;
    cp.hdr = cp_hdr;
    cp.state = reinterpret_cast<uint32_t *>(smem + (P.gws ? 0 : (size_t)su_per_cta * P.su_bytes));
    cp.data = cp.state + ((P.cta_slots + 3) / 4 * 4);
    for (uint32_t i = threadIdx.x; i < kCpHdrWords; i += blockDim.x) cp_hdr[i] = 0;
    for (uint32_t i = threadIdx.x; i < P.cta_slots; i += blockDim.x) cp.state[i] = 0;
    __syncthreads();
    uint8_t *ws = P.gws ? P.gws + (size_t)G::su_global() * P.su_bytes : smem + (size_t)G::su_local() * P.su_bytes;
    su_main<G>(P, ws, cp);
}

// Register budget of the dense search units (resident threads per SM): for
// 8-word graphs 1280 (48 registers, five 256-thread CTAs) beat 1024 (64
// registers) by 8% on the batched workload despite more spill traffic -- the
// search is latency bound and more resident warps hide it; for 2/4-word graphs
// 1536 (40 registers) measured best.
#ifndef VC_DENSE8_THREADS
#define VC_DENSE8_THREADS 1280
#endif
#ifndef VC_DENSE_WARPS
#define VC_DENSE_WARPS 8
#endif
#ifndef VC_DENSE4_THREADS
#define VC_DENSE4_THREADS 1536
#endif
template <int NW>
struct DenseOcc {
    // 20-word graphs: three 256-thread CTAs' worth of registers (80 per thread),
    // so that a server lane of them fits beside three 8-word CTAs per SM;
    // 16- and 32-word graphs (16-bit degrees, rows and L in registers): two and
    // one CTA per SM, as many as their staged adjacency leaves room for
    static constexpr unsigned kThreads =
        NW == 32 ? 256u : (NW == 16 ? 512u : (NW >= 16 ? 768u : (NW >= 8 ? VC_DENSE8_THREADS : VC_DENSE4_THREADS)));
    template <unsigned NT>
    static constexpr unsigned min_ctas() { return kThreads / NT < 32 ? kThreads / NT : 32; }  // 32 CTAs/SM at most
};

template <int NW, unsigned NT>
__global__ void __launch_bounds__(NT, DenseOcc<NW>::template min_ctas<NT>()) k_dense(Params P)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t cp_hdr[kCpHdrWords];
    if (P.server && threadIdx.x == 0) atomicAdd(&P.ctl[kStarted], 1ull);  // residency check of server lanes
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

// One thread per search unit (vc_lanes.cuh); NT lanes per CTA.
#ifndef VC_LANE_THREADS
#define VC_LANE_THREADS 128
#endif
template <int NW, unsigned NT>
__global__ void __launch_bounds__(NT, 1) k_lanes(Params P)
{
    extern __shared__ __align__(16) uint32_t lsm[];
    __shared__ uint32_t hdr[kLhWords];
    const LaneLayout lo(P.np / 32u, NW, NT, P.cta_slots);
    if (threadIdx.x < kLhWords) {
        const uint32_t i = threadIdx.x;
        hdr[i] = i == kLhIdle ? NT : ((i == kLhGraph || i == kLhKey) ? kNone : 0u);
    }
    for (uint32_t i = threadIdx.x; i < P.cta_slots; i += NT) lsm[lo.sstate + i] = 0;
    __syncthreads();
    lanes_main<NW, NT>(P, lsm, hdr);
}

__global__ void k_init_ring(unsigned long long *seq, uint32_t q)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < q) seq[i] = i;
}

__global__ void k_init_state(InstState *st, const InstDesc *d, uint32_t count)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        InstState s;
        s.best = d[i].init_best;
        s.act = 1;
        s.flags = 0;
        s.lock = 0;
        s.cover_size = kNone;
        s.pad = 0;
        s.nodes = 0;
        s.t_done = 0;
        st[i] = s;
    }
}

// ---------------------------------------------------------------- buffers
cudaError_t DevBuf::ensure(size_t bytes)
{
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    want = want + want / 4;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) { p = nullptr; return e; }
    cap = want;
    return cudaSuccess;
}

void DevBuf::release()
{
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

cudaError_t PinBuf::ensure(size_t bytes)
{
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 4096);
    want = want + want / 4;
    cudaError_t e = cudaMallocHost(&p, want);
    if (e != cudaSuccess) { p = nullptr; return e; }
    cap = want;
    return cudaSuccess;
}

static std::mutex g_ctx_mu;
static Ctx *g_ctx[64];

Ctx *get_ctx(int dev, vc_status *err)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) { *err = VC_ERR_NO_DEVICE; return nullptr; }
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) { *err = VC_ERR_CUDA; return nullptr; }
    }
    if (dev >= ndev || dev >= 64) { *err = VC_ERR_INVALID; return nullptr; }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (!g_ctx[dev]) {
        Ctx *c = new Ctx();
        c->dev = dev;
        if (cudaSetDevice(dev) != cudaSuccess) { delete c; *err = VC_ERR_CUDA; return nullptr; }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) { delete c; *err = VC_ERR_CUDA; return nullptr; }
        c->sms = prop.multiProcessorCount;
        c->smem_optin = (int)prop.sharedMemPerBlockOptin;
        c->coop = prop.cooperativeLaunch;
        // VC_LANES=1 selects lane search units for graphs of at most 255 vertices
        if (const char *e = getenv("VC_LANES")) c->lanes_mode = atoi(e) ? 1 : 0;
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
            delete c;
            *err = VC_ERR_CUDA;
            return nullptr;
        }
        g_ctx[dev] = c;
    }
    if (cudaSetDevice(dev) != cudaSuccess) { *err = VC_ERR_CUDA; return nullptr; }
    *err = VC_OK;
    return g_ctx[dev];
}

// ---------------------------------------------------------------- sizing
// Resident CTAs per SM of `fn` with `smem` bytes of dynamic shared memory (0 on error).
template <unsigned NT, class F>
static int ctas_per_sm(F fn, uint32_t smem)
{
    int per_sm = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)NT, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

template <unsigned NT, class F>
static cudaError_t plan_variant_fn(Ctx &c, Plan &pl, uint32_t smem_per_block, F fn)
{
    const int per_sm = ctas_per_sm<NT>(fn, smem_per_block);
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    pl.fn = (const void *)fn;
    pl.block = NT;
    pl.grid = (uint32_t)per_sm * (uint32_t)c.sms;
    pl.smem = smem_per_block;
    return cudaSuccess;
}

// The CSR kernel for group G: team-walk kernels take the 80-register build
// when shared memory already holds the SM to as few CTAs (their row walks
// keep more values live than the lane walks).
template <class G, unsigned NT>
static cudaError_t plan_variant(Ctx &c, Plan &pl, uint32_t smem_per_block)
{
    if constexpr (G::kTeam) {
        auto roomy = k_search<G, NT, kRoomyThreadsPerSM>;
        const int r = ctas_per_sm<NT>(roomy, smem_per_block);
        if (r > 0 && r >= ctas_per_sm<NT>(k_search<G, NT>, smem_per_block))
            return plan_variant_fn<NT>(c, pl, smem_per_block, roomy);
    }
    return plan_variant_fn<NT>(c, pl, smem_per_block, k_search<G, NT>);
}

static uint32_t cta_pool_bytes(uint32_t slots, uint32_t stride)
{
    return slots ? 4u * ((slots + 3) / 4 * 4) + 4u * slots * stride : 0u;
}

// Chooses the search-unit shape for a vertex capacity np: one warp per SU with
// its workspace in shared memory for np <= kWarpMaxNP (up to 8 warps per CTA,
// sharing a CTA pool of 2 slots per warp), else one 512-thread CTA per SU, in
// shared memory while it fits, else in a global workspace.

template <int NW>
static cudaError_t plan_dense(Ctx &c, Plan &pl, const Tune *t)
{
    pl.np = 32 * NW;
    pl.su_bytes = dense_workspace_bytes(NW);
    pl.stride = (4 + NW + 3) / 4 * 4;
    const uint32_t budget = (uint32_t)c.smem_optin - 1024;
    uint32_t warps = (t && t->set) ? t->warps : VC_DENSE_WARPS;  // search units sharing one staged graph
    const uint32_t per_warp = (t && t->set) ? t->pool : 2;
    // 32-word graphs (a 147 KB adjacency) step 8 -> 6 -> 4 warps, the others halve
    while (warps > 1 && dense_adj_bytes(NW) + warps * pl.su_bytes + cta_pool_bytes(per_warp * warps, pl.stride) > budget)
        warps = (NW == 32 && warps == 8) ? 6 : (warps == 6 ? 4 : warps >> 1);
    pl.cta_slots = warps > 1 ? per_warp * warps : 0;
    uint32_t smem = dense_adj_bytes(NW) + warps * pl.su_bytes + cta_pool_bytes(pl.cta_slots, pl.stride);
    cudaError_t e;
    switch (warps) {
    case 8: e = plan_variant_fn<256>(c, pl, smem, k_dense<NW, 256>); break;
    case 6:
        if constexpr (NW == 32) e = plan_variant_fn<192>(c, pl, smem, k_dense<NW, 192>);
        else e = cudaErrorInvalidConfiguration;
        break;
    case 4: e = plan_variant_fn<128>(c, pl, smem, k_dense<NW, 128>); break;
    case 2: e = plan_variant_fn<64>(c, pl, smem, k_dense<NW, 64>); break;
    default: e = plan_variant_fn<32>(c, pl, smem, k_dense<NW, 32>); break;
    }
    if (e != cudaSuccess) return e;
    pl.num_su = pl.grid * (pl.block / 32);
    pl.global_ws = false;
    pl.dense = true;
    return cudaSuccess;
}

template <int NW>
static cudaError_t plan_lanes(Ctx &c, Plan &pl, uint32_t nmax)
{
    constexpr unsigned NT = VC_LANE_THREADS;
    const uint32_t nwc = std::max<uint32_t>(1, (nmax + 31) / 32);
    pl.np = 32 * nwc;
    pl.stride = (4 + NW + 3) / 4 * 4;
    pl.cta_slots = kLanePoolSlots;
    const LaneLayout lo(nwc, NW, NT, pl.cta_slots);
    pl.su_bytes = 4u * (17u * nwc);  // degree bytes, trail bytes, flag words per lane
    cudaError_t e = plan_variant_fn<NT>(c, pl, 4u * lo.words, k_lanes<NW, NT>);
    if (e != cudaSuccess) return e;
    pl.num_su = pl.grid * NT;
    pl.global_ws = false;
    pl.dense = true;
    pl.lanes = true;
    return cudaSuccess;
}

// Warp units, `warps` to a CTA.
template <class G>
static cudaError_t plan_warps(Ctx &c, Plan &pl, uint32_t warps, uint32_t smem)
{
    switch (warps) {
    case 8: return plan_variant<G, 256>(c, pl, smem);
    case 4: return plan_variant<G, 128>(c, pl, smem);
    case 2: return plan_variant<G, 64>(c, pl, smem);
    default: return plan_variant<G, 32>(c, pl, smem);
    }
}

cudaError_t make_plan(Ctx &c, uint32_t np, uint32_t nmax, Plan &pl, const PlanOpts &o)
{
    pl.dense = false;
    pl.lanes = false;
    if (o.lanes && !c.force_sparse && nmax <= 255) {
        if (nmax <= 64) return plan_lanes<2>(c, pl, nmax);
        if (nmax <= 128) return plan_lanes<4>(c, pl, nmax);
        return plan_lanes<8>(c, pl, nmax);
    }
    const uint32_t smem_budget = o.smem_budget, warp_max_np = o.warp_max_np;
    // dense bitsets up to 255 vertices, and up to 640 when every degree fits a
    // byte (degrees are bytes; 0 = removed or isolated)
    if (nmax <= 64 && !c.force_sparse) return plan_dense<2>(c, pl, o.tune);
    if (nmax <= 128 && !c.force_sparse) return plan_dense<4>(c, pl, o.tune);
    if (nmax <= 255 && !c.force_sparse) return plan_dense<8>(c, pl, o.tune);
    if (nmax <= kWideMaxN && o.wide && !c.force_sparse) return plan_dense<20>(c, pl, o.tune);
    if (nmax <= kHalfMaxN && o.half && !c.force_sparse)
        return nmax <= 512 ? plan_dense<16>(c, pl, o.tune) : plan_dense<32>(c, pl, o.tune);
    const Tune *t = (o.tune && o.tune->set && !c.force_sparse) ? o.tune : nullptr;
    pl.np = np;
    pl.su_bytes = su_workspace_bytes(np);
    pl.stride = (4 + np / 32 + 3) / 4 * 4;
    const uint32_t static_smem = 1024;  // reductions / broadcasts / CTA pool header
    uint32_t budget = (uint32_t)c.smem_optin - static_smem;
    if (smem_budget) budget = std::min(budget, smem_budget > static_smem ? smem_budget - static_smem : 0u);
    // a tuned choice: warp units (in shared memory where their workspaces fit,
    // else in global memory) or CTA units
    const bool tuned_warps = t && !t->cta_units;
    const bool tuned_cta = t && t->cta_units;
    const uint32_t per_warp = t ? t->pool : 2;
    const bool warp_gws = o.warp_gws || (tuned_warps && np > kWarpMaxNP);
    if (!tuned_cta && np <= (warp_max_np ? warp_max_np : (tuned_warps ? (1u << 16) : kWarpMaxNP)) && warp_gws) {
        // warp units with their workspaces in global memory: the CTA holds
        // only its pool
        uint32_t warps = t ? t->warps : (o.warps ? o.warps : 8);
        pl.cta_slots = warps > 1 ? per_warp * warps : 0;
        const uint32_t smem = cta_pool_bytes(pl.cta_slots, pl.stride);
        cudaError_t e = o.team ? plan_warps<TeamG<WarpG>>(c, pl, warps, smem) : plan_warps<WarpG>(c, pl, warps, smem);
        if (e != cudaSuccess) return e;
        pl.num_su = pl.grid * (pl.block / 32);
        pl.global_ws = true;
        return cudaSuccess;
    }
    if (!tuned_cta && np <= (warp_max_np ? warp_max_np : kWarpMaxNP)) {
        uint32_t warps = t ? t->warps : 8;
        while (warps > 1 && warps * pl.su_bytes + cta_pool_bytes(per_warp * warps, pl.stride) > budget) warps >>= 1;
        if (warps * pl.su_bytes + cta_pool_bytes(warps > 1 ? per_warp * warps : 0, pl.stride) <= budget) {
            pl.cta_slots = warps > 1 ? per_warp * warps : 0;
            uint32_t smem = warps * pl.su_bytes + cta_pool_bytes(pl.cta_slots, pl.stride);
            cudaError_t e = o.team ? plan_warps<TeamG<WarpG>>(c, pl, warps, smem) : plan_warps<WarpG>(c, pl, warps, smem);
            if (e != cudaSuccess) return e;
            pl.num_su = pl.grid * (pl.block / 32);
            pl.global_ws = false;
            return cudaSuccess;
        }
    }
    pl.cta_slots = 0;
    {
        const uint32_t smem = pl.su_bytes <= budget ? pl.su_bytes : 0u;
        cudaError_t e = o.team ? plan_variant<TeamG<BlockG<512>>, 512>(c, pl, smem)
                               : plan_variant<BlockG<512>, 512>(c, pl, smem);
        if (e != cudaSuccess) return e;
        pl.global_ws = smem == 0;
    }
    pl.num_su = pl.grid;
    return cudaSuccess;
}

// Caps a plan's persistent grid at `per_sm` CTAs per SM (a server lane that
// shares the device with another lane's kernel).
void cap_plan(const Ctx &c, Plan &pl, uint32_t per_sm)
{
    const uint32_t su_per_cta = pl.grid ? pl.num_su / pl.grid : 1;
    pl.grid = std::min(pl.grid, per_sm * (uint32_t)c.sms);
    pl.num_su = pl.grid * su_per_cta;
}

// ---------------------------------------------------------------- one launch
// Runs every graph of `job` (arena already on the device) to completion and
// copies back the per-graph state and cover bitmaps.
vc_status run_job(Ctx &c, Job &job, cudaStream_t stream)
{
    const uint32_t count = (uint32_t)job.desc.size();
    if (count == 0) return VC_OK;
    uint32_t nmax = 0, cover_words = 0;
    uint64_t sum_n = 0, sum_m2 = 0;
    for (auto &d : job.desc) {
        nmax = std::max(nmax, d.n);
        d.cover_off = cover_words;
        cover_words += d.nw;
        if (d.m2 != kNone) { sum_n += d.n; sum_m2 += d.m2; }
    }
    uint32_t np = std::max<uint32_t>(32, (nmax + 31) / 32 * 32);
    Plan pl;
    PlanOpts po;
    po.wide = job.wide;
    po.half = job.half;
    po.team = sum_m2 >= 4 * sum_n && sum_n > 0;  // average degree 4 or more: rows walked by teams
    // Lane units (one thread per search unit, vc_lanes.cuh) are opt-in: they
    // execute half the instructions per tree node of warp units but, at 12
    // resident warps per SM, issue on a fifth of the cycles (ncu, batched
    // workload) and reach a quarter of the warp units' node rate.
    po.lanes = c.lanes_mode == 1;
    const Tune *tn = job.tune ? job.tune : &c.tune[tune_class(nmax, job.wide)];
    po.tune = tn->set ? tn : nullptr;
    if (make_plan(c, np, nmax, pl, po) != cudaSuccess) return VC_ERR_CUDA;
    const uint32_t stride = pl.stride;
    uint32_t q = 1024;
    const uint32_t ring_units = pl.lanes ? pl.grid : pl.num_su;  // lane CTAs poll the ring as a whole
    while (q < 2 * ring_units) q <<= 1;
    const size_t ring_cap_bytes = (size_t)512 << 20;
    while (q > 64 && (size_t)q * stride * 4 > ring_cap_bytes) q >>= 1;

    size_t gws_bytes = pl.global_ws ? (size_t)pl.num_su * pl.su_bytes : 0;
    if (c.inst.ensure(sizeof(InstDesc) * count) || c.st.ensure(sizeof(InstState) * count) ||
        c.covers.ensure(sizeof(uint32_t) * std::max<uint32_t>(cover_words, 1)) ||
        c.ctl.ensure(sizeof(unsigned long long) * kCtlWords) || c.seq.ensure(sizeof(unsigned long long) * q) ||
        c.data.ensure((size_t)q * stride * 4) || c.launches.ensure(sizeof(unsigned long long)) ||
        (gws_bytes && c.gws.ensure(gws_bytes)))
        return VC_ERR_NOMEM;
    if (c.h_st.ensure(sizeof(InstState) * count) || c.h_desc.ensure(sizeof(InstDesc) * count) ||
        c.h_covers.ensure(sizeof(uint32_t) * std::max<uint32_t>(cover_words, 1)))
        return VC_ERR_NOMEM;

    memcpy(c.h_desc.p, job.desc.data(), sizeof(InstDesc) * count);
    cudaMemcpyAsync(c.inst.p, c.h_desc.p, sizeof(InstDesc) * count, cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(c.covers.p, 0, sizeof(uint32_t) * std::max<uint32_t>(cover_words, 1), stream);
    cudaMemsetAsync(c.ctl.p, 0, sizeof(unsigned long long) * kCtlWords, stream);
    k_init_ring<<<(q + 255) / 256, 256, 0, stream>>>((unsigned long long *)c.seq.p, q);
    k_init_state<<<(count + 255) / 256, 256, 0, stream>>>((InstState *)c.st.p, (const InstDesc *)c.inst.p, count);
    g_launches += 2;
    if (job.dev_input) {
        k_check_csr<0><<<std::min<uint32_t>(count, 4096), 256, 0, stream>>>(job.d_rp, job.d_col, (const InstDesc *)c.inst.p,
                                                                        (InstState *)c.st.p, count);
        g_launches += 1;
    }

    Params P;
    memset(&P, 0, sizeof(P));
    P.row_ptr = job.d_rp;
    P.col = job.d_col;
    P.inst = (const InstDesc *)c.inst.p;
    P.st = (InstState *)c.st.p;
    P.covers = (uint32_t *)c.covers.p;
    P.count = count;
    P.num_su = pl.num_su;
    P.ctl = (unsigned long long *)c.ctl.p;
    P.pool_seq = (unsigned long long *)c.seq.p;
    P.pool_data = (uint32_t *)c.data.p;
    P.q_mask = q - 1;
    P.stride = stride;
    P.np = np;
    P.su_bytes = pl.su_bytes;
    P.cta_slots = pl.cta_slots;
    P.gws = pl.global_ws ? (uint8_t *)c.gws.p : nullptr;
    P.stats = nullptr;
    if (c.stats_on) {
        if (c.stats.ensure(sizeof(unsigned long long) * kStatWords * pl.num_su)) return VC_ERR_NOMEM;
        cudaMemsetAsync(c.stats.p, 0, sizeof(unsigned long long) * kStatWords * pl.num_su, stream);
        P.stats = (unsigned long long *)c.stats.p;
    }
    double tl = job.time_limit_s > 0 ? job.time_limit_s : 300.0;
    P.time_limit_ns = (unsigned long long)(tl * 1e9);
    P.ring_bias = po.tune ? po.tune->ring_bias : 0;
    P.ring_first = po.tune ? po.tune->ring_first : 0u;

    void *args[] = {&P};
    cudaEventRecord(c.ev0, stream);
    cudaError_t e = c.coop ? cudaLaunchCooperativeKernel(pl.fn, dim3(pl.grid), dim3(pl.block), args, pl.smem, stream)
                           : cudaErrorNotSupported;
    if (e != cudaSuccess) return VC_ERR_CUDA;
    g_launches += 1;
    cudaEventRecord(c.ev1, stream);
    cudaMemcpyAsync(c.h_st.p, c.st.p, sizeof(InstState) * count, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(c.h_covers.p, c.covers.p, sizeof(uint32_t) * std::max<uint32_t>(cover_words, 1),
                    cudaMemcpyDeviceToHost, stream);
    unsigned long long abort_flag = 0;
    cudaMemcpyAsync(c.h_ctl, c.ctl.p, sizeof(unsigned long long) * kCtlWords, cudaMemcpyDeviceToHost, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return VC_ERR_CUDA;
    abort_flag = c.h_ctl[kAbort];
    job.t0 = c.h_ctl[kT0];
    cudaEventElapsedTime(&job.kernel_ms, c.ev0, c.ev1);
    job.aborted = abort_flag != 0;
    job.st.assign((InstState *)c.h_st.p, (InstState *)c.h_st.p + count);
    job.covers.assign((uint32_t *)c.h_covers.p, (uint32_t *)c.h_covers.p + std::max<uint32_t>(cover_words, 1));
    job.plan = pl;
    if (c.stats_on) {
        c.last_stats.resize((size_t)kStatWords * pl.num_su);
        cudaMemcpy(c.last_stats.data(), c.stats.p, sizeof(unsigned long long) * kStatWords * pl.num_su,
                   cudaMemcpyDeviceToHost);
        c.last_num_su = pl.num_su;
    }
    c.last_plan = pl;
    return VC_OK;
}

// Fills one vc_result from the collected state of graph i.
vc_status fill_result(const Job &job, uint32_t i, uint32_t ub, vc_result *out)
{
    const InstDesc &d = job.desc[i];
    const InstState &s = job.st[i];
    vc_status st;
    if (s.flags & kBadGraph) st = VC_ERR_INVALID;
    else if (s.flags & kError) st = VC_ERR_INTERNAL;
    else if (s.flags & kBudget) st = VC_BUDGET;
    else if ((s.flags & kCut) || !(s.flags & kDone)) st = job.aborted ? VC_TIMEOUT : VC_ERR_INTERNAL;
    else st = VC_OK;
    out->status = st;
    out->tree_nodes = s.nodes;
    out->kernel_ms = job.kernel_ms;
    out->done_ms = (s.t_done && job.t0 && s.t_done >= job.t0) ? (float)((s.t_done - job.t0) * 1e-6) : 0.0f;
    bool have_cover = s.cover_size != kNone;
    if (d.mode == kModeMVC) {
        out->decision = 1;
        if (s.best < d.init_best) out->size = s.best;
        else out->size = ub ? ub : d.n;  // no cover below the bound: min(ub, OPT) = ub
    } else {
        out->decision = (s.flags & kFound) ? 1u : 0u;
        out->size = out->decision ? s.cover_size : 0u;
    }
    out->has_cover = have_cover ? 1u : 0u;
    if (out->cover_mask) {
        if (have_cover) {
            const uint32_t *w = job.covers.data() + d.cover_off;
            for (uint32_t v = 0; v < d.n; ++v) out->cover_mask[v] = (uint8_t)((w[v >> 5] >> (v & 31u)) & 1u);
        } else {
            memset(out->cover_mask, 0, d.n);
        }
    }
    return st;
}

}  // namespace vch

// ---------------------------------------------------------------- C ABI
using namespace vch;

extern "C" const char *vc_status_string(vc_status s)
{
    switch (s) {
    case VC_OK: return "ok";
    case VC_ERR_INVALID: return "invalid argument";
    case VC_ERR_CUDA: return "CUDA error";
    case VC_ERR_NOMEM: return "out of device memory";
    case VC_ERR_TOO_LARGE: return "graph too large";
    case VC_TIMEOUT: return "time limit reached";
    case VC_BUDGET: return "node limit reached";
    case VC_ERR_INTERNAL: return "internal error";
    case VC_ERR_NO_DEVICE: return "no CUDA device";
    case VC_PENDING: return "pending";
    }
    return "unknown";
}

extern "C" uint64_t vc_kernel_launches(void) { return g_launches.load(); }

// Diagnostics (not part of the reference surface): enable (bit 0)
// per-search-unit counters on a device, force the CSR kernel (bit 1) or lane
// search units (bit 2) for graphs of at most 255 vertices, and read the last launch's counters as rows of
// kStatWords u64 (nodes, passes, donations, failed donations, receives, roots,
// busy cycles, idle cycles, polls, restored vertices, SM id).  Returns the
// number of search units; copies at most max_rows rows.
extern "C" uint32_t vc_debug_stats(int32_t device, int32_t enable, uint64_t *rows, uint32_t max_rows,
                                   uint32_t *launch_shape)
{
    vch::DeviceGuard dg;
    vc_status err;
    Ctx *c = get_ctx(device, &err);
    if (!c) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
    if (enable >= 0) c->stats_on = (enable & 1) != 0;
    if (enable >= 0) c->force_sparse = (enable & 2) != 0;
    if (enable >= 0) c->lanes_mode = (enable & 4) ? 1 : 0;
    uint32_t nsu = c->last_num_su;
    if (rows) {
        // rows exist only for a launch that ran with the counters on
        uint32_t k = std::min(nsu, max_rows);
        k = std::min<uint32_t>(k, (uint32_t)(c->last_stats.size() / kStatWords));
        memcpy(rows, c->last_stats.data(), sizeof(uint64_t) * kStatWords * k);
    }
    if (launch_shape) {
        launch_shape[0] = c->last_plan.grid;
        launch_shape[1] = c->last_plan.block;
        launch_shape[2] = c->last_plan.smem;
        launch_shape[3] = c->last_plan.num_su;
        launch_shape[4] = c->last_plan.np | (c->last_plan.dense ? 0x80000000u : 0u);
    }
    return nsu;
}

static uint32_t init_best_for(const vc_request *r, uint32_t n)
{
    if (r->instance == VC_PVC) return n + 1;
    uint32_t ub = r->ub ? std::min<uint32_t>(r->ub, n) : n;
    return ub + 1;
}

extern "C" vc_status vc_solve(const vc_csr *g, const vc_request *req, vc_result *out)
{
    vch::DeviceGuard dg;
    auto t0 = std::chrono::steady_clock::now();
    if (!g || !req || !out) return VC_ERR_INVALID;
    if (req->instance != VC_MVC && req->instance != VC_PVC) return VC_ERR_INVALID;
    const bool dev_in = (req->flags & VC_FLAG_DEVICE_INPUT) != 0;
    if (!dev_in && !(req->flags & VC_FLAG_NO_VALIDATE)) {
        vc_status v = validate_csr(g);
        if (v != VC_OK) return v;
    } else if (!g->row_ptr || (g->m && !g->col)) {
        return VC_ERR_INVALID;
    }
    out->size = 0;
    out->decision = 0;
    out->has_cover = 0;
    out->tree_nodes = 0;
    out->kernel_ms = 0;
    if (g->n == 0) {
        out->status = VC_OK;
        out->decision = 1;
        out->has_cover = 1;
        out->total_ms = 0;
        return VC_OK;
    }
    if (g->n > kMaxVertices) return VC_ERR_TOO_LARGE;
    vc_status err;
    Ctx *c = get_ctx(req->device, &err);
    if (!c) return err;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t stream = req->stream ? (cudaStream_t)req->stream : c->stream;

    Job job;
    if (dev_in) {
        job.d_rp = g->row_ptr;
        job.d_col = g->col;
    } else {
        size_t rp_b = sizeof(uint32_t) * ((size_t)g->n + 1), col_b = sizeof(uint32_t) * std::max<size_t>(2 * (size_t)g->m, 1);
        if (c->rp.ensure(rp_b) || c->col.ensure(col_b)) return VC_ERR_NOMEM;
        cudaMemcpyAsync(c->rp.p, g->row_ptr, rp_b, cudaMemcpyHostToDevice, stream);
        if (g->m) cudaMemcpyAsync(c->col.p, g->col, sizeof(uint32_t) * 2 * (size_t)g->m, cudaMemcpyHostToDevice, stream);
        job.d_rp = (const uint32_t *)c->rp.p;
        job.d_col = (const uint32_t *)c->col.p;
    }
    InstDesc d;
    d.n = g->n;
    d.nw = (g->n + 31) / 32;
    d.row_off = 0;
    d.col_off = 0;
    d.mode = req->instance == VC_PVC ? kModePVC : kModeMVC;
    d.k = std::min<uint32_t>(req->k, g->n);
    d.init_best = init_best_for(req, g->n);
    d.cover_off = 0;
    d.node_limit = req->node_limit;
    d.key = 0;
    d.m2 = 2ull * g->m < (uint64_t)kNone ? (uint32_t)(2ull * g->m) : kNone;
    job.desc.push_back(d);
    job.time_limit_s = req->time_limit_s;
    job.wide = !dev_in && wide_ok(g->n, g->row_ptr);
    job.half = !job.wide && half_ok(g->n);
    job.dev_input = dev_in;
    vc_status s = run_job(*c, job, stream);
    if (s != VC_OK) { out->status = s; return s; }
    s = fill_result(job, 0, req->instance == VC_MVC ? req->ub : 0, out);
    out->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

extern "C" vc_status vc_solve_batch(const vc_csr_arena *a, const vc_request *reqs, vc_result *out)
{
    vch::DeviceGuard dg;
    auto t0 = std::chrono::steady_clock::now();
    if (!a || !reqs || !out) return VC_ERR_INVALID;
    if (a->count == 0) return VC_OK;
    if (!a->n || !a->row_off || !a->col_off || !a->row_ptr) return VC_ERR_INVALID;
    const bool dev_in = (reqs[0].flags & VC_FLAG_DEVICE_INPUT) != 0;
    for (uint32_t i = 1; i < a->count; ++i)
        if (((reqs[i].flags & VC_FLAG_DEVICE_INPUT) != 0) != dev_in) return VC_ERR_INVALID;
    if (dev_in) return VC_ERR_INVALID;  // per-graph sizes are read on the host: use vc_solve_batch_device
    return vc_solve_batch_impl(a, reqs, out, nullptr, nullptr, t0);
}

namespace vch {
vc_status vc_solve_batch_impl(const vc_csr_arena *a, const vc_request *reqs, vc_result *out, const uint32_t *d_rp,
                              const uint32_t *d_col, std::chrono::steady_clock::time_point t0)
{
    const uint32_t count = a->count;
    // every early failure is reported in each graph's result too
    auto fail = [&](vc_status st) {
        for (uint32_t i = 0; i < count; ++i) {
            out[i].status = st;
            out[i].size = 0;
            out[i].decision = 0;
            out[i].has_cover = 0;
            out[i].tree_nodes = 0;
        }
        return st;
    };
    uint64_t rows = 0, cols = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (reqs[i].instance != VC_MVC && reqs[i].instance != VC_PVC) return fail(VC_ERR_INVALID);
        if (a->n[i] > kMaxVertices) return fail(VC_ERR_TOO_LARGE);
        rows = std::max<uint64_t>(rows, a->row_off[i] + a->n[i] + 1);
    }
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t *rp = a->row_ptr + a->row_off[i];
        cols = std::max<uint64_t>(cols, a->col_off[i] + rp[a->n[i]]);
    }
    if (!d_rp && !(reqs[0].flags & VC_FLAG_NO_VALIDATE)) {
        for (uint32_t i = 0; i < count; ++i) {
            vc_csr g;
            g.n = a->n[i];
            const uint32_t *rp = a->row_ptr + a->row_off[i];
            g.m = rp[g.n] / 2;
            g.row_ptr = rp;
            g.col = a->col + a->col_off[i];
            g.degree = nullptr;
            vc_status v = validate_csr(&g);
            if (v != VC_OK) return fail(v);
        }
    }
    vc_status err;
    Ctx *c = get_ctx(reqs[0].device, &err);
    if (!c) return fail(err);
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t stream = reqs[0].stream ? (cudaStream_t)reqs[0].stream : c->stream;
    Job job;
    if (d_rp) {
        job.d_rp = d_rp;
        job.d_col = d_col;
    } else {
        if (c->rp.ensure(sizeof(uint32_t) * rows) || c->col.ensure(sizeof(uint32_t) * std::max<uint64_t>(cols, 1)))
            return fail(VC_ERR_NOMEM);
        cudaMemcpyAsync(c->rp.p, a->row_ptr, sizeof(uint32_t) * rows, cudaMemcpyHostToDevice, stream);
        if (cols) cudaMemcpyAsync(c->col.p, a->col, sizeof(uint32_t) * cols, cudaMemcpyHostToDevice, stream);
        job.d_rp = (const uint32_t *)c->rp.p;
        job.d_col = (const uint32_t *)c->col.p;
    }
    // One launch per kernel shape: dense bitsets (n <= 255), wide dense bitsets
    // (n <= 640, every degree <= 254), dense bitsets with 16-bit degrees (n <=
    // 1024), warp search units (n <= kWarpMaxNP), CTA search units (larger); the
    // shape is sized by the largest graph of its class, so small graphs never
    // run in a large graph's workspace.  The row offsets are host arrays on both
    // entry points.
    auto klass = [&](uint32_t i) {
        const uint32_t n = a->n[i];
        if (n <= 255) return 0;
        if (wide_ok(n, a->row_ptr + a->row_off[i])) return 1;
        if (half_ok(n)) return 2;
        return n <= kWarpMaxNP ? 3 : 4;
    };
    vc_status first = VC_OK;
    float total_kernel = 0;
    std::vector<uint32_t> members;
    for (int cl = 0; cl < 5; ++cl) {
        members.clear();
        for (uint32_t i = 0; i < count; ++i)
            if (a->n[i] > 0 && klass(i) == cl) members.push_back(i);
        if (members.empty()) continue;
        Job cj;
        cj.d_rp = job.d_rp;
        cj.d_col = job.d_col;
        cj.wide = cl == 1;
        cj.half = cl == 2;
        cj.dev_input = d_rp != nullptr;
        cj.desc.resize(members.size());
        double tl = 0;
        for (size_t j = 0; j < members.size(); ++j) {
            const uint32_t i = members[j];
            InstDesc &d = cj.desc[j];
            d.n = a->n[i];
            d.nw = (d.n + 31) / 32;
            d.row_off = a->row_off[i];
            d.col_off = a->col_off[i];
            d.mode = reqs[i].instance == VC_PVC ? kModePVC : kModeMVC;
            d.k = std::min<uint32_t>(reqs[i].k, d.n);
            d.init_best = init_best_for(&reqs[i], d.n);
            d.node_limit = reqs[i].node_limit;
            d.key = (uint32_t)j;
            d.m2 = a->row_ptr[a->row_off[i] + d.n];
            tl = std::max(tl, reqs[i].time_limit_s);
        }
        cj.time_limit_s = tl;
        vc_status s = run_job(*c, cj, stream);
        if (s != VC_OK) {
            for (uint32_t i = 0; i < count; ++i) out[i].status = s;
            return s;
        }
        total_kernel += cj.kernel_ms;
        for (size_t j = 0; j < members.size(); ++j) {
            const uint32_t i = members[j];
            vc_status si = fill_result(cj, (uint32_t)j, reqs[i].instance == VC_MVC ? reqs[i].ub : 0, &out[i]);
            if (si != VC_OK && first == VC_OK) first = si;
        }
    }
    float total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (uint32_t i = 0; i < count; ++i) {
        out[i].total_ms = total;
        out[i].kernel_ms = total_kernel;
        if (a->n[i] == 0) {
            out[i].status = VC_OK;
            out[i].size = 0;
            out[i].decision = 1;
            out[i].has_cover = 1;
            out[i].tree_nodes = 0;
            out[i].done_ms = 0;
        }
    }
    return first;
}
}  // namespace vch

// Batched solve over an arena already resident on the device: the per-graph
// sizes and offsets stay on the host (`a` holds host arrays for n, row_off,
// col_off and the row_ptr values), d_rp / d_col are the device copies.
extern "C" vc_status vc_solve_batch_device(const vc_csr_arena *a, const uint32_t *d_rp, const uint32_t *d_col,
                                           const vc_request *reqs, vc_result *out)
{
    vch::DeviceGuard dg;
    auto t0 = std::chrono::steady_clock::now();
    if (!a || !reqs || !out || !d_rp) return VC_ERR_INVALID;
    if (a->count == 0) return VC_OK;
    return vc_solve_batch_impl(a, reqs, out, d_rp, d_col, t0);
}
