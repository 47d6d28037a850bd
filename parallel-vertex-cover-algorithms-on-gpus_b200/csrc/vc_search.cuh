// vc_search.cuh -- device side of the exact MVC / PVC branch-and-reduce search.
//
// What it computes is the reference's search (src/GlobalWorkList.cuh:16-200 for
// MVC, src/GlobalWorkListParameterized.cuh:13-202 for PVC): reduce a node with the
// degree-one, degree-two/triangle and high-degree rules, prune on
// del >= best or E >= (best-del-1)^2 + 1 (PVC: del > k or E >= (k-del)^2 + 1),
// branch on the max-degree vertex v into "take v" and "take N(v)".  How it is
// computed is B200-first rather than a translation:
//
//  * Search unit (SU) = one warp (graphs up to a few thousand vertices) or one
//    CTA (larger graphs).  An SU owns, in shared memory: the live-degree array
//    of its current node (int32; a deleted vertex holds a large negative value),
//    an undo trail of the vertices deleted below its starting node, and a frame
//    stack of pending "take N(v)" children (trail position + v).  Backtracking
//    restores the trail instead of copying whole degree arrays (the reference
//    copies (UB+1)*V ints per CTA, stack.cuh:10-47).
//  * One read-only scan per reduction pass decides all three rules from the same
//    snapshot and marks the vertices to take in a bitmap; an apply step then
//    takes them.  The final (mark-free) scan also yields sum of degrees, max
//    degree and its lowest-index argmax with warp redux instructions.  Taking a
//    set of vertices chosen from one snapshot equals taking them one rule at a
//    time (each choice stays valid or becomes a no-op after the others), so the
//    optimum is unchanged; only the order of deletions differs from the
//    reference's phase-by-phase loop (helperFunctions.cuh:229-447).
//  * Work sharing: a bounded lock-free MPMC ring in global memory (L2-resident)
//    holds donated subtrees as deleted-vertex bitmaps (n bits).  A busy SU
//    donates its shallowest pending child only while more SUs are idle than
//    items are queued.  Termination: one 64-bit word (pending<<32 | idle).
//    Every spin is bounded by a deadline read from %globaltimer.
//  * Many graphs run in one launch: SUs pull graph roots from a cursor first and
//    the ring carries (graph id, bitmap) records, so idle SUs help whichever
//    graph still has work.  Per-graph incumbent, token count and flags live in
//    InstState; the graph is finished when its token count reaches zero.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vc_types.h"

namespace vcg {
// ---------------------------------------------------------------- memory ops
__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Graph rows and offsets.  A batch launch's arena is read-only while it runs
// and goes through the non-coherent cache; a server launch's arena slots are
// reused for new requests while the kernel runs, so it reads around L1
// (ld.global.cg) and never sees a line of the slot's previous graph.
__device__ __forceinline__ uint32_t gld(bool cg, const uint32_t *p) { return cg ? __ldcg(p) : __ldg(p); }

// A graph descriptor read around L1 (server slots are rewritten during a launch).
__device__ __forceinline__ InstDesc load_desc(const InstDesc *p)
{
    InstDesc d;
    d.n = __ldcg(&p->n);
    d.nw = __ldcg(&p->nw);
    d.row_off = __ldcg(&p->row_off);
    d.col_off = __ldcg(&p->col_off);
    d.mode = __ldcg(&p->mode);
    d.k = __ldcg(&p->k);
    d.init_best = __ldcg(&p->init_best);
    d.cover_off = __ldcg(&p->cover_off);
    d.node_limit = __ldcg(&p->node_limit);
    d.key = __ldcg(&p->key);
    d.m2 = __ldcg(&p->m2);
    return d;
}

// Device-resident graphs: one CTA per graph checks the CSR layout the kernels
// rely on (row_ptr[0] = 0, row_ptr[n] = the 2m the caller stated, monotone
// offsets, ids < n, no self loops) and flags a graph that breaks it, so the
// search never reads or writes outside the caller's arrays.
template <int Unused>
__global__ void k_check_csr(const uint32_t *row_ptr, const uint32_t *col, const InstDesc *inst, InstState *st,
                            uint32_t count)
{
    for (uint32_t gi = blockIdx.x; gi < count; gi += gridDim.x) {
        const InstDesc d = inst[gi];
        const uint32_t *rp = row_ptr + d.row_off, *cl = col + d.col_off;
        const uint32_t m2 = rp[d.n];
        bool bad = rp[0] != 0u || (d.m2 != kNone && m2 != d.m2);
        if (!bad) {
            for (uint32_t v = threadIdx.x; v < d.n; v += blockDim.x) {
                const uint32_t e0 = rp[v], e1 = rp[v + 1];
                if (e1 < e0 || e1 > m2) { bad = true; break; }
                for (uint32_t e = e0; e < e1; ++e) {
                    const uint32_t u = cl[e];
                    if (u >= d.n || u == v) { bad = true; break; }
                }
            }
        }
        if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&st[gi].flags, kBadGraph);
    }
}

// Idle search units that wait for work from their CTA (all but the CTA's one
// ring poller) sleep with exponential back-off up to kIdleNapMax ns between
// looks at the CTA pool.  Each look costs a few dozen instructions; dozens of
// idle warps per SM looking every 256 ns took most of the SM's issue slots from
// the busy warps when one graph had the whole GPU.
#ifndef VC_IDLE_NAP_MAX
#define VC_IDLE_NAP_MAX 16384u
#endif
constexpr uint32_t kIdleNapMax = VC_IDLE_NAP_MAX;

// ---------------------------------------------------------------- groups
struct WarpG {
    static constexpr unsigned kSize = 32;
    __device__ __forceinline__ static unsigned rank() { return threadIdx.x & 31u; }
    __device__ __forceinline__ static void sync() { __syncwarp(); }
    __device__ __forceinline__ static bool any(bool p) { return __any_sync(0xffffffffu, p); }
    __device__ __forceinline__ static uint32_t sum(uint32_t x) { return __reduce_add_sync(0xffffffffu, x); }
    __device__ __forceinline__ static uint32_t max(uint32_t x) { return __reduce_max_sync(0xffffffffu, x); }
    __device__ __forceinline__ static uint32_t min(uint32_t x) { return __reduce_min_sync(0xffffffffu, x); }
    __device__ __forceinline__ static uint32_t bcast(uint32_t x) { return __shfl_sync(0xffffffffu, x, 0); }
    __device__ __forceinline__ static unsigned long long bcast64(unsigned long long x)
    {
        return __shfl_sync(0xffffffffu, x, 0);
    }
    __device__ __forceinline__ static unsigned su_local() { return threadIdx.x >> 5; }
    __device__ __forceinline__ static unsigned su_global() { return blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); }
    __device__ __forceinline__ static unsigned warp() { return 0; }
    static constexpr unsigned kWarps = 1;
    static constexpr bool kTeam = false;  // CSR rows walked one lane per row
};

template <unsigned NT>
struct BlockG {
    static constexpr unsigned kSize = NT;
    static constexpr unsigned kWarps = NT / 32;
    __device__ __forceinline__ static unsigned rank() { return threadIdx.x; }
    __device__ __forceinline__ static void sync() { __syncthreads(); }
    __device__ __forceinline__ static bool any(bool p) { return __syncthreads_or(p) != 0; }
    __device__ __forceinline__ static uint32_t reduce(uint32_t x, int op)
    {
        __shared__ uint32_t part[NT / 32];
        __shared__ uint32_t res;
        uint32_t w = op == 0 ? __reduce_add_sync(0xffffffffu, x)
                             : (op == 1 ? __reduce_max_sync(0xffffffffu, x) : __reduce_min_sync(0xffffffffu, x));
        if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = w;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint32_t ident = op == 2 ? 0xffffffffu : 0u;
            uint32_t v = threadIdx.x < NT / 32 ? part[threadIdx.x] : ident;
            v = op == 0 ? __reduce_add_sync(0xffffffffu, v)
                        : (op == 1 ? __reduce_max_sync(0xffffffffu, v) : __reduce_min_sync(0xffffffffu, v));
            if (threadIdx.x == 0) res = v;
        }
        __syncthreads();
        uint32_t r = res;
        __syncthreads();
        return r;
    }
    __device__ __forceinline__ static uint32_t sum(uint32_t x) { return reduce(x, 0); }
    __device__ __forceinline__ static uint32_t max(uint32_t x) { return reduce(x, 1); }
    __device__ __forceinline__ static uint32_t min(uint32_t x) { return reduce(x, 2); }
    __device__ __forceinline__ static uint32_t bcast(uint32_t x)
    {
        __shared__ uint32_t b;
        if (threadIdx.x == 0) b = x;
        __syncthreads();
        uint32_t r = b;
        __syncthreads();
        return r;
    }
    __device__ __forceinline__ static unsigned long long bcast64(unsigned long long x)
    {
        __shared__ unsigned long long b;
        if (threadIdx.x == 0) b = x;
        __syncthreads();
        unsigned long long r = b;
        __syncthreads();
        return r;
    }
    __device__ __forceinline__ static unsigned su_local() { return 0; }
    __device__ __forceinline__ static unsigned su_global() { return blockIdx.x; }
    __device__ __forceinline__ static unsigned warp() { return threadIdx.x >> 5; }
    static constexpr bool kTeam = false;
};

// The same group with CSR rows walked by teams of lanes (see Team): the choice
// for graphs whose average degree is 4 or more.
template <class Base>
struct TeamG : Base {
    static constexpr bool kTeam = true;
};

// ---------------------------------------------------------------- SU state
// Workspace layout (bytes), np = vertex capacity, nw = np/32:
//   deg[np] int32 | trail[np] u32 | fpos[np] u32 | fv[np] u32 | marks[nw] | bits[nw] | ctr[4] | cand[np] u32 |
//   aux[np] (np > 65536 only)

struct SUStat {
    unsigned long long passes, donations, donate_fail, receives, roots, busy, idle, polls, restored;
};

struct SU {
    SUStat stat;
    int32_t *deg;
    uint32_t *trail, *fpos, *fv, *marks, *bits, *ctr, *cand, *aux;
    // current graph
    const uint32_t *rp, *cl;
    uint32_t inst, n, nw, mode, k, cover_off;
    unsigned long long node_limit;
    uint32_t base_del;
    bool cg;          // graph reads around L1 (server launches)
    uint32_t c_best;  // cached incumbent (refreshed every few nodes; stale values only weaken pruning)
    uint32_t fr_bot, fr_top;
    uint32_t tlg;   // log2 of the lanes that walk one CSR row together (see Team)
    unsigned long long local_nodes;
    unsigned long long deadline;
};

// A team: 2^lg consecutive lanes of one warp that walk one CSR row together
// (coalesced loads, lane j reads entries j, j + w, ...), while the group's other
// teams work on other vertices.  The width follows the graph's average degree:
// one lane per row where rows are a few entries long, the whole warp where they
// are hundreds long.  Teams never straddle a warp, so their ballots, shuffles
// and reductions use the team's own lane mask.
// The members are recomputed from lg where used (a few integer operations) so
// that they hold no registers across the walks.
template <class G>
struct Team {
    uint32_t lg;
    __device__ __forceinline__ uint32_t w() const { return 1u << lg; }
    __device__ __forceinline__ uint32_t lane() const { return G::rank() & (w() - 1u); }
    __device__ __forceinline__ uint32_t id() const { return G::rank() >> lg; }
    __device__ __forceinline__ uint32_t T() const { return G::kSize >> lg; }
    __device__ __forceinline__ uint32_t src() const { return threadIdx.x & 31u & ~(w() - 1u); }
    __device__ __forceinline__ uint32_t mask() const
    {
        return lg == 5u ? 0xffffffffu : ((1u << w()) - 1u) << src();
    }
};

// Team width for a graph of n vertices and m2 = 2m CSR entries: one lane below
// an average degree of 4 (rows of two or three entries keep 32 vertices in
// flight per warp), else the largest power of two not above the average
// degree, up to the whole warp.
__device__ __forceinline__ uint32_t team_lg(uint32_t n, uint32_t m2)
{
    const uint32_t avg = n ? m2 / n : 0u;
    return avg < 4u ? 0u : min(5u, 31u - (uint32_t)__clz(avg));
}

// The record bitmap a search unit fills for donation (see donation_bits).
__device__ __forceinline__ uint32_t *rec_bits(SU &s) { return s.bits; }


__device__ __forceinline__ void su_bind(SU &s, uint8_t *ws, uint32_t np)
{
    uint32_t nw = np / 32;
    s.deg = reinterpret_cast<int32_t *>(ws);
    s.trail = reinterpret_cast<uint32_t *>(ws) + np;
    s.fpos = s.trail + np;
    s.fv = s.fpos + np;
    s.marks = s.fv + np;
    s.bits = s.marks + nw;
    s.ctr = s.bits + nw;
    s.cand = s.ctr + 4;
    s.aux = np > 65536u ? s.cand + np : nullptr;
}

__device__ __forceinline__ void mark(uint32_t *marks, uint32_t v) { atomicOr(&marks[v >> 5], 1u << (v & 31u)); }

__device__ __forceinline__ bool row_contains(bool cg, const uint32_t *rp, const uint32_t *cl, uint32_t row, uint32_t x)
{
    uint32_t lo = gld(cg, &rp[row]), hi = gld(cg, &rp[row + 1]);
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t c = gld(cg, &cl[mid]);
        if (c == x) return true;
        if (c < x) lo = mid + 1; else hi = mid;
    }
    return false;
}

// One thread takes v: claim it, log it on the trail, decrement live neighbours.
__device__ __forceinline__ void take_one_lane(SU &s, uint32_t v)
{
    const int32_t old = atomicExch(&s.deg[v], kDead);
    if (old < 0) return;
    s.trail[atomicAdd(&s.ctr[0], 1u)] = v;
    volatile int32_t *dv = s.deg;
    const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
    for (uint32_t e = gld(s.cg, &s.rp[v]); e < e1; ++e) {
        const uint32_t u = gld(s.cg, &s.cl[e]);
        if (dv[u] >= 0) atomicSub(&s.deg[u], 1);
    }
}

// One team takes v: its first lane claims v and logs it on the trail, then the
// team decrements v's live neighbours.
template <class G>
__device__ __forceinline__ void take_one(SU &s, uint32_t v, const Team<G> &t)
{
    uint32_t ok = 0;
    if (t.lane() == 0) {
        const int32_t old = atomicExch(&s.deg[v], kDead);
        if (old >= 0) {
            s.trail[atomicAdd(&s.ctr[0], 1u)] = v;
            ok = 1;
        }
    }
    if (!__shfl_sync(t.mask(), ok, t.src())) return;
    volatile int32_t *dv = s.deg;
    const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
    for (uint32_t e = gld(s.cg, &s.rp[v]) + t.lane(); e < e1; e += t.w()) {
        const uint32_t u = gld(s.cg, &s.cl[e]);
        if (dv[u] >= 0) atomicSub(&s.deg[u], 1);
    }
}

struct ScanOut {
    uint32_t sum, maxd, amax;
};

// One reduction pass.  Returns true if marks were found and applied (another
// pass is needed); otherwise fills `o` with the fixpoint's statistics.  A first
// sweep takes the statistics and the high-degree marks and gathers the degree-1/2
// vertices into a list; the list is then worked one vertex per thread, so the
// CSR row walks of the leaf and triangle rules run side by side instead of in
// one divergent round per vertex slot.
template <class G>
__device__ __forceinline__ bool reduce_pass(SU &s, uint32_t del, uint32_t bound, ScanOut &o)
{
    uint32_t sum = 0, maxd = 0, amax = kNone;
    bool marked = false;
    const int32_t *deg = s.deg;
    for (uint32_t v = G::rank(); v < s.n; v += G::kSize) {
        int32_t d = deg[v];
        if (d <= 0) continue;
        uint32_t ud = (uint32_t)d;
        sum += ud;
        if (ud > maxd) { maxd = ud; amax = v; }
        if (ud + del >= bound) {  // high-degree rule (helperFunctions.cuh:323-327)
            mark(s.marks, v);
            marked = true;
        } else if (d <= 2) {
            s.cand[atomicAdd(&s.ctr[1], 1u)] = v;
        }
    }
    G::sync();
    const uint32_t nc = s.ctr[1];
    G::sync();
    if (G::rank() == 0) s.ctr[1] = 0;
    const Team<G> t{s.tlg};
    if constexpr (!G::kTeam) {  // rows of a few entries: a lane per candidate
        for (uint32_t i = G::rank(); i < nc; i += G::kSize) {
            const uint32_t v = s.cand[i];
            if (deg[v] == 1) {        // degree-one rule (helperFunctions.cuh:252-265)
                const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
                for (uint32_t e = gld(s.cg, &s.rp[v]); e < e1; ++e) {
                    const uint32_t u = gld(s.cg, &s.cl[e]);
                    const int32_t du = deg[u];
                    if (du > 0) {
                        if (du > 1 || u < v) { mark(s.marks, u); marked = true; }
                        break;
                    }
                }
            } else {                  // degree-two triangle rule (helperFunctions.cuh:384-417)
                uint32_t n1 = kNone, n2 = kNone;
                bool keep = false;
                const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
                for (uint32_t e = gld(s.cg, &s.rp[v]); e < e1; ++e) {
                    const uint32_t u = gld(s.cg, &s.cl[e]);
                    const int32_t du = deg[u];
                    if (du > 0) {
                        if (du == 1 || (du == 2 && u < v)) { keep = true; break; }
                        if (n1 == kNone) n1 = u; else { n2 = u; break; }
                    }
                }
                if (!keep && n2 != kNone && row_contains(s.cg, s.rp, s.cl, n2, n1)) {
                    mark(s.marks, n1);
                    mark(s.marks, n2);
                    marked = true;
                }
            }
        }
    }
    // Otherwise a team per candidate finds its live neighbours in row order
    // (degrees do not change during this loop, so a degree-d vertex has exactly
    // d of them); the same rules on them.
    for (uint32_t i = G::kTeam ? t.id() : nc; i < nc; i += t.T()) {
        const uint32_t v = s.cand[i];
        const uint32_t dv0 = (uint32_t)deg[v];  // 1 or 2
        uint32_t got = 0, n1 = kNone, n2 = kNone;
        int32_t d1 = 0, d2 = 0;
        const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
        for (uint32_t eb = gld(s.cg, &s.rp[v]); eb < e1 && got < dv0; eb += t.w()) {
            const uint32_t e = eb + t.lane();
            uint32_t u = kNone;
            int32_t du = 0;
            if (e < e1) {
                u = gld(s.cg, &s.cl[e]);
                du = deg[u];
            }
            uint32_t live = __ballot_sync(t.mask(), du > 0) >> t.src();
            while (live && got < dv0) {
                const uint32_t b = __ffs(live) - 1;
                live &= live - 1;
                const uint32_t uu = __shfl_sync(t.mask(), u, t.src() + b);
                const int32_t dd = __shfl_sync(t.mask(), du, t.src() + b);
                if (got == 0) { n1 = uu; d1 = dd; } else { n2 = uu; d2 = dd; }
                ++got;
            }
        }
        if (t.lane() != 0 || n1 == kNone) continue;
        if (dv0 == 1) {           // degree-one rule (helperFunctions.cuh:252-265)
            if (d1 > 1 || n1 < v) { mark(s.marks, n1); marked = true; }
        } else if (n2 != kNone) { // degree-two triangle rule (helperFunctions.cuh:384-417)
            const bool keep = d1 == 1 || (d1 == 2 && n1 < v) || d2 == 1 || (d2 == 2 && n2 < v);
            if (!keep && row_contains(s.cg, s.rp, s.cl, n2, n1)) {
                mark(s.marks, n1);
                mark(s.marks, n2);
                marked = true;
            }
        }
    }
    s.stat.passes += 1;
    if (G::any(marked)) {
        G::sync();  // the vote is not a memory barrier: make every lane's marks visible
        if constexpr (!G::kTeam) {  // a lane per marks word takes its vertices
            for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) {
                uint32_t m = s.marks[w];
                if (!m) continue;
                s.marks[w] = 0;
                while (m) {
                    const uint32_t b = __ffs(m) - 1;
                    m &= m - 1;
                    take_one_lane(s, w * 32 + b);
                }
            }
            G::sync();
        } else {  // list the marked vertices (the candidate list is spent), then a team takes each
            for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) {
                uint32_t m = s.marks[w];
                if (!m) continue;
                s.marks[w] = 0;
                uint32_t at = atomicAdd(&s.ctr[3], (uint32_t)__popc(m));
                while (m) {
                    s.cand[at++] = w * 32 + __ffs(m) - 1;
                    m &= m - 1;
                }
            }
            G::sync();
            const uint32_t nm = s.ctr[3];
            for (uint32_t i = t.id(); i < nm; i += t.T()) take_one(s, s.cand[i], t);
            G::sync();
            if (G::rank() == 0) s.ctr[3] = 0;  // every thread read it before the barrier; the next use is a pass later
        }
        return true;
    }
    o.sum = G::sum(sum);
    o.maxd = G::max(maxd);
    o.amax = G::min((maxd == o.maxd && maxd > 0) ? amax : kNone);
    return false;
}

// Left child: take the branching vertex v (helperFunctions.cuh:200-215).
template <class G>
__device__ __forceinline__ void take_vertex(SU &s, uint32_t v)
{
    uint32_t ok = 0;
    if (G::rank() == 0) {
        int32_t old = atomicExch(&s.deg[v], kDead);
        if (old >= 0) {
            s.trail[s.ctr[0]] = v;
            s.ctr[0] += 1;
            ok = 1;
        }
    }
    ok = G::bcast(ok);
    if (ok) {
        volatile int32_t *dv = s.deg;
        uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
        for (uint32_t e = gld(s.cg, &s.rp[v]) + G::rank(); e < e1; e += G::kSize) {
            uint32_t u = gld(s.cg, &s.cl[e]);
            if (dv[u] >= 0) atomicSub(&s.deg[u], 1);
        }
    }
    G::sync();
}

// Right child: take every live neighbour of v (helperFunctions.cuh:156-184).
template <class G>
__device__ __forceinline__ void take_neighbours(SU &s, uint32_t v)
{
    const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
    if constexpr (G::kTeam) {
        const Team<G> t{s.tlg};
        for (uint32_t e = gld(s.cg, &s.rp[v]) + t.id(); e < e1; e += t.T()) take_one(s, gld(s.cg, &s.cl[e]), t);
    } else {
        for (uint32_t e = gld(s.cg, &s.rp[v]) + G::rank(); e < e1; e += G::kSize) take_one_lane(s, gld(s.cg, &s.cl[e]));
    }
    G::sync();
}

// Undo the trail back to position `pos` (vertices become live again with their
// exact live-neighbour counts).
template <class G>
__device__ __forceinline__ void restore_to(SU &s, uint32_t pos)
{
    uint32_t top = s.ctr[0];
    s.stat.restored += top - pos;
    for (uint32_t i = pos + G::rank(); i < top; i += G::kSize) s.deg[s.trail[i]] = kRestoring;
    G::sync();
    volatile int32_t *dv = s.deg;
    if constexpr (G::kTeam) {
        const Team<G> t{s.tlg};
        for (uint32_t i = pos + t.id(); i < top; i += t.T()) {  // a team per trail vertex
            const uint32_t v = s.trail[i];
            uint32_t c = 0;
            const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
            for (uint32_t e = gld(s.cg, &s.rp[v]) + t.lane(); e < e1; e += t.w()) {
                const uint32_t u = gld(s.cg, &s.cl[e]);
                const int32_t d = dv[u];
                if (d == kRestoring) ++c;
                else if (d >= 0) { atomicAdd(&s.deg[u], 1); ++c; }
            }
            c = __reduce_add_sync(t.mask(), c);  // every lane of the team has read trail[i]
            if (t.lane() == 0) {
                if (s.aux) s.aux[i] = c; else s.trail[i] = v | (c << 16);
            }
        }
    } else {
        for (uint32_t i = pos + G::rank(); i < top; i += G::kSize) {  // a lane per trail vertex
            const uint32_t v = s.trail[i];
            uint32_t c = 0;
            const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
            for (uint32_t e = gld(s.cg, &s.rp[v]); e < e1; ++e) {
                const uint32_t u = gld(s.cg, &s.cl[e]);
                const int32_t d = dv[u];
                if (d == kRestoring) ++c;
                else if (d >= 0) { atomicAdd(&s.deg[u], 1); ++c; }
            }
            if (s.aux) s.aux[i] = c; else s.trail[i] = v | (c << 16);
        }
    }
    G::sync();
    for (uint32_t i = pos + G::rank(); i < top; i += G::kSize) {
        uint32_t t = s.trail[i];
        if (s.aux) s.deg[t] = (int32_t)s.aux[i];
        else s.deg[t & 0xffffu] = (int32_t)(t >> 16);
    }
    G::sync();
    if (G::rank() == 0) s.ctr[0] = pos;
    G::sync();
}

// bits[w] = 1 for every deleted vertex of the current state (warp ballots).
template <class G>
__device__ __forceinline__ void dead_bits(SU &s, uint32_t *dst)
{
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t w = G::warp(); w < s.nw; w += G::kWarps) {
        uint32_t word = __ballot_sync(0xffffffffu, s.deg[w * 32 + lane] < 0);
        if (lane == 0) dst[w] = word;
    }
}

template <class G>
__device__ __forceinline__ void cover_bits(SU &s, uint32_t *dst) { dead_bits<G>(s, dst); }

// Rebuild the degree array from a deleted-vertex bitmap in s.bits.
template <class G>
__device__ __forceinline__ void rebuild(SU &s)
{
    uint32_t pad_end = s.nw * 32;
    const Team<G> t{G::kTeam ? s.tlg : 0u};  // a team (or a lane) per vertex
    for (uint32_t v = t.id(); v < pad_end; v += t.T()) {
        if (v >= s.n) { if (t.lane() == 0) s.deg[v] = 0; continue; }
        if ((s.bits[v >> 5] >> (v & 31u)) & 1u) { if (t.lane() == 0) s.deg[v] = kDead; continue; }
        uint32_t c = 0;
        const uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
        for (uint32_t e = gld(s.cg, &s.rp[v]) + t.lane(); e < e1; e += t.w()) {
            const uint32_t u = gld(s.cg, &s.cl[e]);
            c += ((s.bits[u >> 5] >> (u & 31u)) & 1u) ^ 1u;
        }
        if constexpr (G::kTeam) c = __reduce_add_sync(t.mask(), c);
        if (t.lane() == 0) s.deg[v] = (int32_t)c;
    }
    uint32_t pc = 0;
    for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) pc += __popc(s.bits[w]);
    for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) s.marks[w] = 0;
    s.base_del = G::sum(pc);
    if (G::rank() == 0) { s.ctr[0] = 0; s.ctr[1] = 0; s.ctr[3] = 0; }
    G::sync();
}

template <class G>
__device__ __forceinline__ void bind_graph(SU &s, const Params &P, uint32_t inst)
{
    const InstDesc d = load_desc(&P.inst[inst]);
    s.inst = inst;
    s.n = d.n;
    s.nw = d.nw;
    s.mode = d.mode;
    s.k = d.k;
    s.cover_off = d.cover_off;
    s.node_limit = d.node_limit;
    s.rp = P.row_ptr + d.row_off;
    s.cl = P.col + d.col_off;
    s.tlg = team_lg(d.n, gld(s.cg, &s.rp[d.n]));
    s.fr_bot = s.fr_top = 0;
    s.local_nodes = 0;
}

// Root of a graph: the input degrees.
template <class G>
__device__ __forceinline__ void load_root(SU &s)
{
    uint32_t pad_end = s.nw * 32;
    for (uint32_t v = G::rank(); v < pad_end; v += G::kSize)
        s.deg[v] = v < s.n ? (int32_t)(gld(s.cg, &s.rp[v + 1]) - gld(s.cg, &s.rp[v])) : 0;
    for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) s.marks[w] = 0;
    s.base_del = 0;
    if (G::rank() == 0) { s.ctr[0] = 0; s.ctr[1] = 0; s.ctr[3] = 0; }
    G::sync();
}

// ---------------------------------------------------------------- global ring
// Bounded MPMC ring (per-slot sequence numbers).  Both claims give up after a
// few attempts instead of spinning: a failed claim is retried by the caller
// after a back-off.
__device__ __forceinline__ bool ring_claim_enq(const Params &P, unsigned long long &pos_out)
{
    for (int it = 0; it < 8; ++it) {
        unsigned long long pos = ld_relaxed_u64(&P.ctl[kTail]);
        unsigned long long seq = ld_acquire_u64(&P.pool_seq[pos & P.q_mask]);
        long long dif = (long long)(seq - pos);
        if (dif == 0) {
            if (atomicCAS(&P.ctl[kTail], pos, pos + 1) == pos) { pos_out = pos; return true; }
        } else if (dif < 0) {
            return false;  // full
        }
    }
    return false;
}

__device__ __forceinline__ bool ring_claim_deq(const Params &P, unsigned long long &pos_out)
{
    for (int it = 0; it < 2; ++it) {
        unsigned long long pos = ld_relaxed_u64(&P.ctl[kHead]);
        unsigned long long seq = ld_acquire_u64(&P.pool_seq[pos & P.q_mask]);
        long long dif = (long long)(seq - (pos + 1));
        if (dif == 0) {
            if (atomicCAS(&P.ctl[kHead], pos, pos + 1) == pos) { pos_out = pos; return true; }
        } else if (dif < 0) {
            return false;  // empty, or the producer has not published yet
        }
    }
    return false;
}

// ---------------------------------------------------------------- CTA pool
// The warps of one CTA share work through shared memory; only fully idle CTAs
// take work from the global ring, and only one warp per CTA polls it.
enum : uint32_t { kCpIdle = 0, kCpCount, kCpPoller, kCpRegistered, kCpExit, kCpHdrWords = 8 };

struct CtaPool {
    uint32_t *hdr;        // kCpHdrWords control words (shared memory)
    uint32_t *state;      // [lp] 0 empty, 1 being written, 2 full, 3 being read
    uint32_t *data;       // [lp][stride]
    uint32_t lp, su;      // slots, search units in this CTA
};

__device__ __forceinline__ uint32_t vld(const uint32_t *p) { return *(volatile const uint32_t *)p; }

// Bitmap of the child to donate: frame state (dead now minus the trail above the
// frame) plus N(v).  Left in s.bits.
template <class G>
__device__ __forceinline__ void donation_bits(SU &s)
{
    uint32_t pos = s.fpos[s.fr_bot], v = s.fv[s.fr_bot];
    uint32_t top = s.ctr[0];
    dead_bits<G>(s, s.bits);
    G::sync();
    for (uint32_t i = pos + G::rank(); i < top; i += G::kSize) {
        uint32_t u = s.trail[i];
        atomicAnd(&s.bits[u >> 5], ~(1u << (u & 31u)));
    }
    G::sync();
    uint32_t e1 = gld(s.cg, &s.rp[v + 1]);
    for (uint32_t e = gld(s.cg, &s.rp[v]) + G::rank(); e < e1; e += G::kSize) {
        uint32_t u = gld(s.cg, &s.cl[e]);
        atomicOr(&s.bits[u >> 5], 1u << (u & 31u));
    }
    G::sync();
}

// Donate the shallowest pending child to a sibling warp of this CTA.
template <class G, class S>
__device__ bool donate_local(S &s, const Params &P, CtaPool &cp)
{
    uint32_t slot = kNone;
    if (G::rank() == 0) {
        for (uint32_t i = 0; i < cp.lp; ++i)
            if (atomicCAS(&cp.state[i], 0u, 1u) == 0u) { slot = i; break; }
    }
    slot = G::bcast(slot);
    if (slot == kNone) { s.stat.donate_fail += 1; return false; }
    donation_bits<G>(s);
    uint32_t *d = cp.data + (size_t)slot * P.stride;
    if (G::rank() == 0) {
        d[0] = s.inst;
        atomicAdd(&P.st[s.inst].act, 1u);
    }
    for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) d[4 + w] = rec_bits(s)[w];
    __threadfence_block();
    G::sync();
    if (G::rank() == 0) {
        __threadfence_block();
        atomicExch(&cp.state[slot], 2u);
        atomicAdd(&cp.hdr[kCpCount], 1u);
    }
    s.fr_bot += 1;
    s.stat.donations += 1;
    return true;
}

// Donate the shallowest pending child to the global ring (for idle CTAs).
template <class G, class S>
__device__ bool donate_global(S &s, const Params &P)
{
    unsigned long long qpos = 0;
    uint32_t ok = 0;
    if (G::rank() == 0) {
        atomicAdd(&P.ctl[kState], 1ull << 32);
        if (ring_claim_enq(P, qpos)) ok = 1;
        else atomicAdd(&P.ctl[kState], 0xffffffff00000000ull);
    }
    ok = G::bcast(ok);
    if (!ok) { s.stat.donate_fail += 1; return false; }
    qpos = G::bcast64(qpos);
    donation_bits<G>(s);
    uint32_t *slot = P.pool_data + (size_t)(qpos & P.q_mask) * P.stride;
    if (G::rank() == 0) {
        atomicAdd(&P.st[s.inst].act, 1u);
        __stcg(&slot[0], s.inst);
    }
    for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) __stcg(&slot[4 + w], rec_bits(s)[w]);
    __threadfence();
    G::sync();
    if (G::rank() == 0) {
        __threadfence();
        st_release_u64(&P.pool_seq[qpos & P.q_mask], qpos + 1);
    }
    s.fr_bot += 1;
    s.stat.donations += 1;
    return true;
}

// Claims the next graph root (one thread).  Batch launches walk a cursor over
// graphs 0..count-1; a server launch takes slot ids the host published on the
// submission queue and initialises the slot's state.
__device__ __forceinline__ bool claim_root(const Params &P, uint32_t &slot)
{
    if (!P.server) {
        const uint32_t i = (uint32_t)atomicAdd(&P.ctl[kCursor], 1ull);
        if (i < P.count) { slot = i; return true; }
        return false;
    }
    for (int it = 0; it < 4; ++it) {
        const unsigned long long c = ld_relaxed_u64(&P.ctl[kCursor]);
        const unsigned long long t = ld_acquire_u64(&P.ctl[kSubTail]);
        if (c >= t) return false;
        if (atomicCAS(&P.ctl[kCursor], c, c + 1) == c) {
            slot = __ldcg(&P.subq[c & P.subq_mask]);
            const InstDesc d = load_desc(&P.inst[slot]);
            InstState *st = &P.st[slot];
            st->best = d.init_best;
            st->act = 1;
            st->flags = 0;
            st->lock = 0;
            st->cover_size = kNone;
            st->nodes = 0;
            st->t_done = 0;
            __threadfence();
            atomicExch(&P.ctl[kLastWork], globaltimer());
            return true;
        }
    }
    return false;
}

// True when a server launch may stop: the host asked for shutdown, or nothing
// was submitted for idle_ns; and no published submission is unclaimed.
__device__ __forceinline__ bool server_may_stop(const Params &P)
{
    if (ld_relaxed_u64(&P.ctl[kCursor]) < ld_acquire_u64(&P.ctl[kSubTail])) return false;
    if (ld_relaxed_u64(&P.ctl[kShutdown])) return true;
    return globaltimer() > ld_relaxed_u64(&P.ctl[kLastWork]) + P.idle_ns;
}

// Server mode: the SU that returned a graph's last token copies its result
// and cover into the host-mapped record, then publishes the ticket.
template <class G>
__device__ __forceinline__ void publish_result(const Params &P, uint32_t slot)
{
    const InstDesc d = load_desc(&P.inst[slot]);
    InstState *st = &P.st[slot];
    HostResult *hr = reinterpret_cast<HostResult *>(P.hres + (size_t)slot * P.hres_words);
    uint32_t *hcover = reinterpret_cast<uint32_t *>(hr + 1);
    const uint32_t cs = ld_relaxed_u32(&st->cover_size);
    if (cs != kNone)
        for (uint32_t w = G::rank(); w < d.nw; w += G::kSize) hcover[w] = __ldcg(&P.covers[d.cover_off + w]);
    __threadfence_system();
    G::sync();
    if (G::rank() == 0) {
        hr->best = ld_relaxed_u32(&st->best);
        hr->flags = ld_relaxed_u32(&st->flags);
        hr->cover_size = cs;
        hr->nodes = ld_relaxed_u64(&st->nodes);
        hr->t_done = ld_relaxed_u64(&st->t_done);
        __threadfence_system();
        *reinterpret_cast<volatile unsigned long long *>(&hr->done) = d.key;
        __threadfence_system();
    }
    G::sync();
}

// Record a cover found at a leaf (MVC improvement or PVC success).
template <class G, class S>
__device__ void report_leaf(S &s, const Params &P, uint32_t del)
{
    InstState &st = P.st[s.inst];
    uint32_t write = 0;
    if (G::rank() == 0) {
        if (s.mode == kModeMVC) {
            uint32_t old = atomicMin(&st.best, del);
            if (del < old) {
                bool got = false;
                for (int it = 0; it < (1 << 20); ++it) {  // bounded lock acquisition
                    if (atomicCAS(&st.lock, 0u, 1u) == 0u) { got = true; break; }
                    __nanosleep(64);
                }
                if (!got) atomicOr(&st.flags, kError);
                else if (del < ld_relaxed_u32(&st.cover_size)) write = 1;
                else atomicExch(&st.lock, 0u);
            }
            s.c_best = min(old, del);
        } else {
            uint32_t old = atomicOr(&st.flags, kFound);
            if (!(old & kFound)) write = 2;
        }
    }
    s.c_best = G::bcast(s.c_best);
    write = G::bcast(write);
    if (!write) return;
    cover_bits<G>(s, P.covers + s.cover_off);
    __threadfence();
    G::sync();
    if (G::rank() == 0) {
        st.cover_size = del;
        if (write == 2) atomicMin(&st.best, del);
        __threadfence();
        if (write == 1) atomicExch(&st.lock, 0u);
    }
}

__device__ __forceinline__ bool old_act_pending(InstState &st) { return ld_relaxed_u32(&st.act) > 1u; }

// The SU leaves its current graph: return its token and node count.
template <class G, class S>
__device__ __forceinline__ void finish_stint(S &s, const Params &P)
{
    uint32_t last = 0;
    if (G::rank() == 0) {
        InstState &st = P.st[s.inst];
        atomicAdd(&st.nodes, s.local_nodes);
        __threadfence();
        if (s.node_limit) {
            const unsigned long long tot = ld_relaxed_u64(&st.nodes);
            if (tot >= s.node_limit && old_act_pending(st)) atomicOr(&st.flags, kBudget);
        }
        uint32_t old = atomicSub(&st.act, 1u);
        if (old == 1u) {
            st.t_done = globaltimer();
            __threadfence();
            atomicOr(&st.flags, kDone);
            last = 1;
        }
    }
    if (P.server) {
        last = G::bcast(last);
        if (last) publish_result<G>(P, s.inst);
    }
    s.local_nodes = 0;
    s.inst = kNone;
    s.fr_bot = s.fr_top = 0;
    G::sync();
}

// Starts work on a received record (bits already in s.bits, graph bound);
// returns false if its graph no longer needs work.
template <class G, class S>
__device__ __forceinline__ bool start_record(S &s, const Params &P)
{
    uint32_t fl = 0;
    if (G::rank() == 0) fl = ld_relaxed_u32(&P.st[s.inst].flags);
    fl = G::bcast(fl);
    if (fl & (kFound | kBudget | kError | kBadGraph)) {
        finish_stint<G, S>(s, P);
        return false;
    }
    rebuild<G>(s);
    s.stat.receives += 1;
    return true;
}

// Acquire work: a new graph root from the cursor, else a record from the CTA
// pool, else (fully idle CTA, one poller) from the global ring.  Returns false
// when the launch is over.
template <class G, class S>
__device__ bool acquire(S &s, const Params &P, CtaPool &cp, bool &cursor_open)
{
    if (cursor_open) {
        uint32_t i = kNone;
        if (G::rank() == 0 && !claim_root(P, i)) i = kNone;
        i = G::bcast(i);
        if (i != kNone) {
            bind_graph<G>(s, P, i);
            load_root<G>(s);
            s.stat.roots += 1;
            return true;
        }
        if (!P.server) cursor_open = false;
    }
    if (G::rank() == 0) {
        __threadfence_block();
        atomicAdd(&cp.hdr[kCpIdle], 1u);
    }
    bool poller = false;  // meaningful in rank 0 only
    uint32_t nap = 64;
    for (;;) {
        s.stat.polls += 1;
        // 0 wait, 1 local slot, 2 global record, 3 exit
        uint32_t res = 0, slot = 0;
        unsigned long long qpos = 0;
        if (G::rank() == 0) {
            if (vld(&cp.hdr[kCpExit])) {
                res = 3;
            } else if (vld(&cp.hdr[kCpCount]) > 0) {
                if (poller) { atomicExch(&cp.hdr[kCpPoller], 0u); poller = false; }
                atomicSub(&cp.hdr[kCpIdle], 1u);  // reserve before taking: the CTA never looks idle while work moves
                __threadfence_block();
                for (uint32_t i = 0; i < cp.lp; ++i)
                    if (atomicCAS(&cp.state[i], 2u, 3u) == 2u) { slot = i; res = 1; break; }
                if (res == 0) {
                    __threadfence_block();
                    atomicAdd(&cp.hdr[kCpIdle], 1u);
                }
            } else if (poller || atomicCAS(&cp.hdr[kCpPoller], 0u, 1u) == 0u) {
                poller = true;
                if (ld_relaxed_u64(&P.ctl[kAbort]) || ld_relaxed_u64(&P.ctl[kFinish])) {
                    atomicExch(&cp.hdr[kCpExit], 1u);
                    res = 3;
                } else {
                    unsigned long long stw = ld_relaxed_u64(&P.ctl[kState]);
                    uint32_t cnt = vld(&cp.hdr[kCpCount]);
                    __threadfence_block();
                    uint32_t idl = vld(&cp.hdr[kCpIdle]);
                    if (!vld(&cp.hdr[kCpRegistered]) && cnt == 0 && idl == cp.su) {
                        stw = atomicAdd(&P.ctl[kState], 1ull) + 1ull;  // this CTA is idle
                        cp.hdr[kCpRegistered] = 1u;
                    }
                    const bool reg = vld(&cp.hdr[kCpRegistered]) != 0;
                    uint32_t root = kNone;
                    if (P.server && claim_root(P, root)) {  // a new submission
                        if (reg) {
                            atomicAdd(&P.ctl[kState], 0xffffffffffffffffull);  // idle CTAs-1
                            cp.hdr[kCpRegistered] = 0u;
                        }
                        atomicSub(&cp.hdr[kCpIdle], 1u);
                        slot = root;
                        res = 4;
                    } else if ((stw >> 32) > 0 && ring_claim_deq(P, qpos)) {
                        if (reg) {
                            atomicAdd(&P.ctl[kState], 0xfffffffeffffffffull);  // pending-1, idle CTAs-1
                            cp.hdr[kCpRegistered] = 0u;
                        } else {
                            atomicAdd(&P.ctl[kState], 0xffffffff00000000ull);
                        }
                        atomicSub(&cp.hdr[kCpIdle], 1u);
                        res = 2;
                    } else if (reg && (uint32_t)stw == gridDim.x && (stw >> 32) == 0 &&
                               (!P.server || server_may_stop(P))) {
                        atomicExch(&P.ctl[kFinish], 1ull);
                        atomicExch(&cp.hdr[kCpExit], 1u);
                        res = 3;
                    } else if (globaltimer() > s.deadline) {
                        atomicExch(&P.ctl[kAbort], 1ull);
                        atomicExch(&cp.hdr[kCpExit], 1u);
                        res = 3;
                    }
                }
                if (res != 0) { atomicExch(&cp.hdr[kCpPoller], 0u); poller = false; }
            }
        }
        res = G::bcast(res);
        if (res == 3) return false;
        if (res == 4) {
            slot = G::bcast(slot);
            bind_graph<G>(s, P, slot);
            load_root<G>(s);
            s.stat.roots += 1;
            return true;
        }
        if (res == 1) {
            slot = G::bcast(slot);
            const uint32_t *d = cp.data + (size_t)slot * P.stride;
            __threadfence_block();
            uint32_t inst = vld(&d[0]);
            bind_graph<G>(s, P, inst);
            for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) s.bits[w] = vld(&d[4 + w]);
            G::sync();
            if (G::rank() == 0) {
                atomicSub(&cp.hdr[kCpCount], 1u);
                __threadfence_block();
                atomicExch(&cp.state[slot], 0u);
            }
            if (start_record<G, S>(s, P)) return true;
            if (G::rank() == 0) { __threadfence_block(); atomicAdd(&cp.hdr[kCpIdle], 1u); }
            continue;
        }
        if (res == 2) {
            qpos = G::bcast64(qpos);
            uint32_t slot_i = (uint32_t)(qpos & P.q_mask);
            const uint32_t *g = P.pool_data + (size_t)slot_i * P.stride;
            G::sync();
            __threadfence();
            uint32_t inst = __ldcg(&g[0]);
            bind_graph<G>(s, P, inst);
            for (uint32_t w = G::rank(); w < s.nw; w += G::kSize) s.bits[w] = __ldcg(&g[4 + w]);
            G::sync();
            if (G::rank() == 0) {
                __threadfence();
                st_release_u64(&P.pool_seq[slot_i], qpos + P.q_mask + 1);
            }
            if (start_record<G, S>(s, P)) return true;
            if (G::rank() == 0) { __threadfence_block(); atomicAdd(&cp.hdr[kCpIdle], 1u); }
            continue;
        }
        if (G::rank() == 0) __nanosleep(nap);
        nap = nap < (poller ? 4096u : kIdleNapMax) ? nap * 2 : (poller ? 4096u : kIdleNapMax);
        G::sync();
    }
}

template <class G>
__device__ void su_main(const Params &P, uint8_t *ws, CtaPool &cp)
{
    SU s;
    su_bind(s, ws, P.np);
    s.cg = P.server != 0;
    s.inst = kNone;
    s.fr_bot = s.fr_top = 0;
    s.local_nodes = 0;
    s.c_best = 0;
    s.deadline = globaltimer() + P.time_limit_ns;
    if (G::rank() == 0) atomicCAS(&P.ctl[kT0], 0ull, globaltimer());
    s.stat = SUStat{0, 0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long nodes_total = 0;
    long long t_mark = clock64();
    bool cursor_open = true;
    bool have = false;
    uint32_t ticks = 0, c_flags = 0;
    unsigned long long c_state = 0;

    for (;;) {
        if (!have) {
            if (s.inst != kNone && s.fr_top > s.fr_bot) {
                s.fr_top -= 1;
                restore_to<G>(s, s.fpos[s.fr_top]);
                take_neighbours<G>(s, s.fv[s.fr_top]);
                have = true;
            } else {
                if (s.inst != kNone) finish_stint<G, SU>(s, P);
                long long t0 = clock64();
                s.stat.busy += (unsigned long long)(t0 - t_mark);
                bool got = acquire<G, SU>(s, P, cp, cursor_open);
                t_mark = clock64();
                s.stat.idle += (unsigned long long)(t_mark - t0);
                if (!got) break;
                have = true;
                ticks = 0;  // refresh the cached graph state below
            }
        }
        // ---- one search-tree node
        InstState &st = P.st[s.inst];
        if ((ticks & 7u) == 0u) {  // refresh cached incumbent, flags and ring state
            uint32_t b = 0, f = 0;
            unsigned long long w = 0;
            if (G::rank() == 0) {
                b = ld_relaxed_u32(&st.best);
                f = ld_relaxed_u32(&st.flags);
                w = ld_relaxed_u64(&P.ctl[kState]);
                if ((ticks & 255u) == 0u) {
                    if (ld_relaxed_u64(&P.ctl[kAbort])) f |= kError;
                    else if (globaltimer() > s.deadline) { atomicExch(&P.ctl[kAbort], 1ull); f |= kError; }
                }
            }
            s.c_best = G::bcast(b);
            c_flags = G::bcast(f);
            c_state = G::bcast64(w);
        }
        ++ticks;
        if (c_flags & (kFound | kBudget | kError | kBadGraph)) {  // abandon this graph
            if (G::rank() == 0 && !(c_flags & (kFound | kBudget | kBadGraph))) atomicOr(&st.flags, kCut);
            s.fr_bot = s.fr_top = 0;
            have = false;
            continue;
        }
        s.local_nodes += 1;
        nodes_total += 1;
        if ((s.local_nodes & 127ull) == 0ull) {
            if (G::rank() == 0) {
                unsigned long long tot = atomicAdd(&st.nodes, s.local_nodes) + s.local_nodes;
                if (s.node_limit && tot >= s.node_limit) atomicOr(&st.flags, kBudget);
            }
            s.local_nodes = 0;
        }
        const uint32_t best = s.c_best;
        const uint32_t bound = s.mode == kModeMVC ? best : s.k + 1;
        ScanOut o = {0u, 0u, kNone};
        uint32_t del = s.base_del + s.ctr[0];
        for (int pass = 0; pass < (1 << 20); ++pass) {
            if (!reduce_pass<G>(s, del, bound, o)) break;
            del = s.base_del + s.ctr[0];
        }
        del = s.base_del + s.ctr[0];
        uint64_t edges = o.sum / 2;
        bool prune;
        if (s.mode == kModeMVC) {
            prune = del >= best;
            if (!prune) {
                uint64_t b = (uint64_t)(best - del - 1);
                prune = edges >= b * b + 1;
            }
        } else {
            prune = del > s.k;
            if (!prune) {
                uint64_t b = (uint64_t)(s.k - del);
                prune = edges >= b * b + 1;
            }
        }
        if (prune) { have = false; continue; }
        if (o.maxd == 0) {
            report_leaf<G, SU>(s, P, del);
            have = false;
            continue;
        }
        // branch: push the N(v) child, continue with the v child
        const uint32_t v = o.amax;
        if (G::rank() == 0) {
            s.fpos[s.fr_top] = s.ctr[0];
            s.fv[s.fr_top] = v;
        }
        s.fr_top += 1;
        G::sync();
        // share the shallowest pending child with starving siblings, else with idle CTAs
        uint32_t want = 0;
        if (G::rank() == 0) {
            uint32_t li = vld(&cp.hdr[kCpIdle]), lc = vld(&cp.hdr[kCpCount]);
            const bool local_need = li > lc;
            const bool ring_need = (long long)(uint32_t)c_state - (long long)(c_state >> 32) > (long long)P.ring_bias;
            // both a sibling warp and another CTA wait: the policy decides (local
            // first, ring first, or alternating)
            if (local_need && ring_need)
                want = (P.ring_first == 1 || (P.ring_first == 2 && (s.stat.donations & 1ull))) ? 2 : 1;
            else if (local_need) want = 1;
            else if (ring_need) want = 2;
        }
        want = G::bcast(want);
        if (want == 1) donate_local<G, SU>(s, P, cp);
        else if (want == 2 && donate_global<G, SU>(s, P)) c_state += 1ull << 32;
        take_vertex<G>(s, v);
    }
    if (P.stats && G::rank() == 0) {
        unsigned long long *o = P.stats + (size_t)G::su_global() * kStatWords;
        uint32_t smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        o[kStNodes] = nodes_total;
        o[kStPasses] = s.stat.passes;
        o[kStDonations] = s.stat.donations;
        o[kStDonateFail] = s.stat.donate_fail;
        o[kStReceives] = s.stat.receives;
        o[kStRoots] = s.stat.roots;
        o[kStBusyCycles] = s.stat.busy;
        o[kStIdleCycles] = s.stat.idle;
        o[kStPolls] = s.stat.polls;
        o[kStRestored] = s.stat.restored;
        o[kStSmid] = smid;
    }
}

}  // namespace vcg
