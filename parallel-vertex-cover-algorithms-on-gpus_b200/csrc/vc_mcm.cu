// vc_mcm.cu -- the MCM mode: the search of the reference's default build
// (`#define VC 0`, src/main.cu:9-36), GlobalWorkList_MCM.cuh:13-190 with the
// helpers it calls (findNextEdgeByWarp helperFunctions.cuh:105-147, skipEdge
// :188-195, deleteNextEdge :218-225, getMatchedVertices :532-553).
//
// What the reference computes: an edge-branching search in CSR entry order.  A
// node is (vertex state, entry cursor); a vertex is available while it is
// unmatched and has a neighbour (degree > 0).  At a node it counts the
// unavailable vertices (matched and isolated ones: degree <= 0), finds the
// first entry at or after the cursor whose row vertex and column vertex are
// both available, and is a leaf when every vertex is unavailable, when the
// launch's maximum already equals n, or when no such entry is left; a leaf
// raises the launch's maximum to its count.  Otherwise the right child skips
// the entry (same state, cursor past it) and the left child matches it (both
// endpoints unavailable).  The finished tree's maximum is 2 * (maximum
// matching) + (isolated vertices); the reference's row records it and its CLI
// prints half of it as "Size of maximum matching".
//
// Here: one warp per search unit; the available set is a bitmap held one word
// per lane (graphs of up to 1024 vertices); a depth-first walk whose frames are
// the matched entries (at most n/2 deep, because the skip child of an entry is
// the walk's next node after it backtracks over that entry); rows without an
// available vertex are skipped with one bitmap search and a row's entries are
// read 32 at a time with one ballot.  Work moves through the bounded global
// ring of vc_search.cuh: a unit donates its shallowest untried skip child while
// more units wait than records are queued.  One addition leaves the answer
// unchanged: a subtree is cut when even matching every available vertex could
// not raise the maximum already found (count + 2 * floor(available / 2) <=
// maximum), since the answer is a maximum over leaves.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>

#include "vc_search.cuh"
#include "vc_host.h"
#include "vcgpu.h"

namespace vch {
extern std::atomic<uint64_t> g_launches;
}

namespace vcg {

constexpr uint32_t kMcmMaxN = 1024;
constexpr unsigned kMcmThreads = 256;  // 8 search units per CTA

struct McmArgs {
    uint32_t n, nw;
    unsigned long long node_limit;
};

// Frame depth of one unit: at most n/2 matched entries, plus one.
__host__ __device__ inline uint32_t mcm_depth(uint32_t n) { return n / 2 + 1; }

// The first available vertex >= r (kNone if none); `av` is word `lane` of the set.
__device__ __forceinline__ uint32_t mcm_next_row(uint32_t av, uint32_t r, uint32_t lane)
{
    const uint32_t wr = r >> 5;
    const uint32_t w = lane > wr ? av : (lane == wr ? av & (0xffffffffu << (r & 31u)) : 0u);
    const uint32_t b = __ballot_sync(0xffffffffu, w != 0u);
    if (!b) return kNone;
    const uint32_t l = __ffs(b) - 1;
    return 32u * l + (__ffs(__shfl_sync(0xffffffffu, w, l)) - 1);
}

// The first entry at or after (cr, ce) whose row and column vertices are both
// available (findNextEdgeByWarp's choice); false if none is left.
__device__ __forceinline__ bool mcm_next_entry(const uint32_t *rp, const uint32_t *cl, uint32_t n, uint32_t av,
                                               uint32_t lane, uint32_t cr, uint32_t ce, uint32_t &er, uint32_t &ee)
{
    uint32_t r = cr;
    for (;;) {
        const uint32_t nr = mcm_next_row(av, r, lane);
        if (nr == kNone || nr >= n) return false;
        const uint32_t e0 = nr == cr ? max(ce, __ldg(&rp[nr])) : __ldg(&rp[nr]);
        const uint32_t e1 = __ldg(&rp[nr + 1]);
        for (uint32_t eb = e0; eb < e1; eb += 32) {
            const uint32_t ei = eb + lane;
            const uint32_t u = ei < e1 ? __ldg(&cl[ei]) : 0u;
            const uint32_t word = __shfl_sync(0xffffffffu, av, u >> 5);
            const uint32_t b = __ballot_sync(0xffffffffu, ei < e1 && ((word >> (u & 31u)) & 1u));
            if (b) {
                er = nr;
                ee = eb + (__ffs(b) - 1);
                return true;
            }
        }
        r = nr + 1;
    }
}

// Gives the skip child of frame `bot` to the ring: the available set before
// that frame's entry was matched, and the cursor past it.
__device__ __forceinline__ bool mcm_donate(const Params &P, const McmArgs &A, InstState &st, const uint32_t *fe,
                                           const uint32_t *fp, uint32_t bot, uint32_t level, uint32_t av,
                                           uint32_t lane)
{
    unsigned long long qpos = 0;
    uint32_t ok = 0;
    if (lane == 0) {
        atomicAdd(&P.ctl[kState], 1ull << 32);
        if (ring_claim_enq(P, qpos)) ok = 1;
        else atomicAdd(&P.ctl[kState], 0xffffffff00000000ull);
    }
    if (!__shfl_sync(0xffffffffu, ok, 0)) return false;
    qpos = __shfl_sync(0xffffffffu, qpos, 0);
    uint32_t w = av;
    for (uint32_t f = bot; f < level; ++f) {
        const uint32_t pr = fp[f], r = pr & 0xffffu, u = pr >> 16;
        if ((r >> 5) == lane) w |= 1u << (r & 31u);
        if ((u >> 5) == lane) w |= 1u << (u & 31u);
    }
    uint32_t *slot = P.pool_data + (size_t)(qpos & P.q_mask) * P.stride;
    if (lane == 0) {
        atomicAdd(&st.act, 1u);
        __stcg(&slot[0], 0u);
        __stcg(&slot[1], fp[bot] & 0xffffu);
        __stcg(&slot[2], fe[bot] + 1u);
        __stcg(&slot[3], 0u);
    }
    if (lane < A.nw) __stcg(&slot[4 + lane], w);
    __threadfence();
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        st_release_u64(&P.pool_seq[qpos & P.q_mask], qpos + 1);
    }
    return true;
}

// Waits for a ring record (bounded by the launch's deadline).  False when the
// search is over: every token returned, a stop flag, or the time limit.
__device__ __forceinline__ bool mcm_acquire(const Params &P, const McmArgs &A, InstState &st,
                                            unsigned long long deadline, uint32_t lane, uint32_t &av, uint32_t &cr,
                                            uint32_t &ce)
{
    if (lane == 0) atomicAdd(&P.ctl[kState], 1ull);  // idle units + 1
    uint32_t nap = 64;
    for (;;) {
        uint32_t res = 0;  // 0 wait, 1 record, 2 over
        unsigned long long qpos = 0;
        if (lane == 0) {
            const unsigned long long stw = ld_relaxed_u64(&P.ctl[kState]);
            if (ld_relaxed_u64(&P.ctl[kAbort]) || ld_relaxed_u32(&st.act) == 0u ||
                (ld_relaxed_u32(&st.flags) & (kFound | kBudget | kError))) {
                res = 2;
            } else if ((stw >> 32) > 0 && ring_claim_deq(P, qpos)) {
                atomicAdd(&P.ctl[kState], 0xfffffffeffffffffull);  // pending - 1, idle units - 1
                res = 1;
            } else if (globaltimer() > deadline) {
                atomicExch(&P.ctl[kAbort], 1ull);
                res = 2;
            }
        }
        res = __shfl_sync(0xffffffffu, res, 0);
        if (res == 2) return false;
        if (res == 1) {
            qpos = __shfl_sync(0xffffffffu, qpos, 0);
            const uint32_t slot_i = (uint32_t)(qpos & P.q_mask);
            const uint32_t *g = P.pool_data + (size_t)slot_i * P.stride;
            __syncwarp();
            __threadfence();
            cr = __ldcg(&g[1]);
            ce = __ldcg(&g[2]);
            av = lane < A.nw ? __ldcg(&g[4 + lane]) : 0u;
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                st_release_u64(&P.pool_seq[slot_i], qpos + P.q_mask + 1);
            }
            return true;
        }
        if (lane == 0) __nanosleep(nap);
        nap = nap < 4096u ? nap * 2 : 4096u;
        __syncwarp();
    }
}

__global__ void k_mcm_init_ring(unsigned long long *seq, uint32_t q)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < q) seq[i] = i;
}

template <unsigned NT>
__global__ void __launch_bounds__(NT) k_mcm(Params P, McmArgs A)
{
    extern __shared__ __align__(16) uint32_t msm[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t depth = mcm_depth(A.n);
    uint32_t *fe = msm + (size_t)warp * 2u * depth;  // entry index of each matched pair
    uint32_t *fp = fe + depth;                       // its row | column << 16
    InstState &st = P.st[0];
    const uint32_t *rp = P.row_ptr, *cl = P.col;
    const unsigned long long deadline = globaltimer() + P.time_limit_ns;
    const uint32_t su = blockIdx.x * (NT / 32) + warp;
    if (su == 0 && lane == 0) atomicCAS(&P.ctl[kT0], 0ull, globaltimer());

    uint32_t av = 0, level = 0, bot = 0, cr = 0, ce = 0;
    bool have = false;
    if (su == 0) {  // the root: every vertex with a neighbour, cursor at entry 0
        for (uint32_t b = 0; b < 32; ++b) {
            const uint32_t v = 32u * lane + b;
            if (v < A.n && __ldg(&rp[v + 1]) > __ldg(&rp[v])) av |= 1u << b;
        }
        have = true;
    }
    uint32_t c_best = 0, c_flags = 0, ticks = 0;
    unsigned long long c_state = 0, local = 0;
    for (;;) {
        if (!have) {
            if (!mcm_acquire(P, A, st, deadline, lane, av, cr, ce)) break;
            level = bot = 0;
            have = true;
            ticks = 0;
        }
        if ((ticks & 7u) == 0u) {  // cached maximum, flags and ring state
            uint32_t b = 0, f = 0;
            unsigned long long w = 0;
            if (lane == 0) {
                b = ld_relaxed_u32(&st.best);
                f = ld_relaxed_u32(&st.flags);
                w = ld_relaxed_u64(&P.ctl[kState]);
                if ((ticks & 255u) == 0u) {
                    if (ld_relaxed_u64(&P.ctl[kAbort])) f |= kError;
                    else if (globaltimer() > deadline) { atomicExch(&P.ctl[kAbort], 1ull); f |= kError; }
                }
            }
            c_best = __shfl_sync(0xffffffffu, b, 0);
            c_flags = __shfl_sync(0xffffffffu, f, 0);
            c_state = __shfl_sync(0xffffffffu, w, 0);
        }
        ++ticks;
        if (c_flags & (kFound | kBudget | kError)) {  // stop: drop this record
            if (lane == 0) atomicSub(&st.act, 1u);
            have = false;
            continue;
        }
        // ---- one node
        if (++local == 128) {
            if (lane == 0) {
                const unsigned long long tot = atomicAdd(&st.nodes, local) + local;
                if (A.node_limit && tot >= A.node_limit) atomicOr(&st.flags, kBudget);
            }
            local = 0;
        }
        const uint32_t avc = __reduce_add_sync(0xffffffffu, __popc(av));
        const uint32_t cnt = A.n - avc;  // matched and isolated vertices (getMatchedVertices)
        uint32_t er = 0, ee = 0;
        bool descend = false;
        if (cnt < A.n && c_best < A.n && cnt + (avc & ~1u) > c_best)
            descend = mcm_next_entry(rp, cl, A.n, av, lane, cr, ce, er, ee);
        if (!descend && cnt > c_best) {
            // a leaf (every vertex unavailable, or no eligible entry left; a cut subtree
            // cannot count more than the maximum): raise the maximum
            uint32_t nb = cnt;
            if (lane == 0) {
                nb = max(atomicMax(&st.best, cnt), cnt);
                if (cnt == A.n) atomicOr(&st.flags, kFound);
            }
            c_best = __shfl_sync(0xffffffffu, nb, 0);
        }
        if (descend) {
            // share the shallowest untried skip child while more units wait than records are
            // queued, once a first leaf has set a maximum: the first descent is a greedy
            // matching, often already maximum, and runs fastest with the SMs to itself
            if (c_best > 0 && bot < level && (long long)(uint32_t)c_state - (long long)(c_state >> 32) > 0 &&
                mcm_donate(P, A, st, fe, fp, bot, level, av, lane)) {
                bot += 1;
                c_state += 1ull << 32;
            }
            const uint32_t u = __ldg(&cl[ee]);
            if (lane == 0) {
                fe[level] = ee;
                fp[level] = er | (u << 16);
            }
            level += 1;
            if (lane == (er >> 5)) av &= ~(1u << (er & 31u));
            if (lane == (u >> 5)) av &= ~(1u << (u & 31u));
            cr = er;
            ce = ee + 1;
            __syncwarp();
            continue;
        }
        // backtrack: the skip child of the deepest matched entry, or the end of this record
        if (level == bot) {
            if (lane == 0) atomicSub(&st.act, 1u);
            have = false;
            continue;
        }
        level -= 1;
        const uint32_t pr = fp[level], r = pr & 0xffffu, u = pr >> 16;
        if (lane == (r >> 5)) av |= 1u << (r & 31u);
        if (lane == (u >> 5)) av |= 1u << (u & 31u);
        cr = r;
        ce = fe[level] + 1;
    }
    if (lane == 0 && local) atomicAdd(&st.nodes, local);
}

}  // namespace vcg

using namespace vcg;
using namespace vch;

// The MCM mode (see the file comment).  out->size receives the launch's
// maximum: 2 * (maximum matching) + (isolated vertices) when the status is
// VC_OK, the largest count reached so far on VC_TIMEOUT / VC_BUDGET.
extern "C" vc_status vc_mcm(const vc_csr *g, const vc_request *req, vc_result *out)
{
    DeviceGuard dg;
    auto t0 = std::chrono::steady_clock::now();
    if (!g || !req || !out) return VC_ERR_INVALID;
    if (req->instance != VC_MVC) return VC_ERR_INVALID;
    if (req->flags & VC_FLAG_DEVICE_INPUT) return VC_ERR_INVALID;
    if (!(req->flags & VC_FLAG_NO_VALIDATE)) {
        const vc_status v = validate_csr(g);
        if (v != VC_OK) return v;
    } else if (!g->row_ptr || (g->m && !g->col)) {
        return VC_ERR_INVALID;
    }
    out->size = 0;
    out->decision = 1;
    out->has_cover = 0;
    out->tree_nodes = 0;
    out->kernel_ms = 0;
    out->done_ms = 0;
    if (g->n == 0) {
        out->status = VC_OK;
        out->total_ms = 0;
        return VC_OK;
    }
    if (g->n > kMcmMaxN) return VC_ERR_TOO_LARGE;
    vc_status err;
    Ctx *c = get_ctx(req->device, &err);
    if (!c) return err;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t stream = req->stream ? (cudaStream_t)req->stream : c->stream;

    const uint32_t n = g->n, nw = (n + 31) / 32, m2 = 2 * g->m;
    const uint32_t smem = (kMcmThreads / 32) * 2u * mcm_depth(n) * 4u;
    auto fn = k_mcm<kMcmThreads>;
    int per_sm = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)kMcmThreads, smem) != cudaSuccess ||
        per_sm <= 0)
        return VC_ERR_CUDA;
    const uint32_t grid = (uint32_t)per_sm * (uint32_t)c->sms;
    const uint32_t num_su = grid * (kMcmThreads / 32);
    uint32_t q = 1024;
    while (q < 2 * num_su) q <<= 1;
    const uint32_t stride = (4 + nw + 3) / 4 * 4;
    if (c->rp.ensure(4ull * (n + 1)) || c->col.ensure(4ull * std::max<uint32_t>(m2, 1)) ||
        c->st.ensure(sizeof(InstState)) || c->ctl.ensure(sizeof(unsigned long long) * kCtlWords) ||
        c->seq.ensure(sizeof(unsigned long long) * q) || c->data.ensure(4ull * q * stride))
        return VC_ERR_NOMEM;
    InstState s0;
    memset(&s0, 0, sizeof(s0));
    s0.act = 1;  // the root
    s0.cover_size = kNone;
    bool ok = cudaMemcpyAsync(c->rp.p, g->row_ptr, 4ull * (n + 1), cudaMemcpyHostToDevice, stream) == cudaSuccess &&
              (m2 == 0 || cudaMemcpyAsync(c->col.p, g->col, 4ull * m2, cudaMemcpyHostToDevice, stream) == cudaSuccess) &&
              cudaMemcpyAsync(c->st.p, &s0, sizeof(s0), cudaMemcpyHostToDevice, stream) == cudaSuccess &&
              cudaMemsetAsync(c->ctl.p, 0, sizeof(unsigned long long) * kCtlWords, stream) == cudaSuccess;
    if (!ok) {
        cudaStreamSynchronize(stream);
        return VC_ERR_CUDA;
    }
    // launches are checked by their own return codes: an error the caller left
    // pending is neither reported here nor cleared
    unsigned long long *seq = (unsigned long long *)c->seq.p;
    void *init_args[] = {&seq, &q};
    if (cudaLaunchKernel((const void *)k_mcm_init_ring, dim3((q + 255) / 256), dim3(256), init_args, 0, stream) !=
        cudaSuccess) {
        cudaStreamSynchronize(stream);
        return VC_ERR_CUDA;
    }
    Params P;
    memset(&P, 0, sizeof(P));
    P.row_ptr = (const uint32_t *)c->rp.p;
    P.col = (const uint32_t *)c->col.p;
    P.st = (InstState *)c->st.p;
    P.count = 1;
    P.num_su = num_su;
    P.ctl = (unsigned long long *)c->ctl.p;
    P.pool_seq = (unsigned long long *)c->seq.p;
    P.pool_data = (uint32_t *)c->data.p;
    P.q_mask = q - 1;
    P.stride = stride;
    const double tl = req->time_limit_s > 0 ? req->time_limit_s : 300.0;
    P.time_limit_ns = (unsigned long long)(tl * 1e9);
    McmArgs A;
    A.n = n;
    A.nw = nw;
    A.node_limit = req->node_limit;
    Plan pl;
    pl.fn = (const void *)fn;
    pl.block = kMcmThreads;
    pl.grid = grid;
    pl.smem = smem;
    pl.np = 32 * nw;
    pl.num_su = num_su;
    c->last_plan = pl;  // reported by vc_debug_stats
    c->last_num_su = 0;
    cudaEventRecord(c->ev0, stream);
    void *args[] = {&P, &A};
    const bool launched =
        cudaLaunchKernel((const void *)fn, dim3(grid), dim3(kMcmThreads), args, smem, stream) == cudaSuccess;
    cudaEventRecord(c->ev1, stream);
    g_launches += 2;
    InstState s1;
    unsigned long long abort_word = 0;
    ok = launched && cudaMemcpyAsync(&s1, c->st.p, sizeof(s1), cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
         cudaMemcpyAsync(&abort_word, (unsigned long long *)c->ctl.p + kAbort, sizeof(abort_word),
                         cudaMemcpyDeviceToHost, stream) == cudaSuccess;
    if (cudaStreamSynchronize(stream) != cudaSuccess || !ok) return VC_ERR_CUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    out->size = s1.best;
    out->tree_nodes = s1.nodes;
    out->kernel_ms = ms;
    if (s1.flags & kFound) out->status = VC_OK;  // every vertex matched or isolated: nothing can exceed it
    else if (s1.flags & kBudget) out->status = VC_BUDGET;
    else if (abort_word || (s1.flags & kError)) out->status = VC_TIMEOUT;
    else out->status = VC_OK;
    out->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return out->status;
}
