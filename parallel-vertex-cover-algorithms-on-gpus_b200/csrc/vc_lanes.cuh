// vc_lanes.cuh -- the throughput search for graphs of at most 255 vertices: one
// THREAD per search unit.
//
// Same search as vc_dense.cuh and vc_search.cuh (the reference's degree-one,
// degree-two/triangle and high-degree rules, the E > b^2 prune and max-degree
// branching: src/GlobalWorkList.cuh:108-190, src/helperFunctions.cuh:229-504),
// laid out so that a warp advances 32 search-tree nodes at once instead of one:
//
//  * a CTA works on one graph at a time; its adjacency is staged once into
//    shared memory as one bitmap row per vertex (as in vc_dense.cuh);
//  * every thread ("lane") is a search unit with its own depth-first search:
//      - the live set L and the pending removals P as bitmaps in registers;
//      - the live degrees as bytes in shared memory, interleaved by thread
//        (byte 4q+b of a lane's array is byte b of word q*NT + tid), so the
//        32 lanes of a warp scanning word q hit 32 distinct banks, and a lane
//        touching any vertex's byte stays in its own bank;
//      - an undo trail of removed vertices (bytes, same interleaving) with a
//        flag bit per position marking the branching vertex of a frame: a
//        backtrack pops and restores vertices one at a time (each restore adds
//        the vertex's live neighbours back to their degrees) down to the
//        newest flagged vertex v, whose "take N(v)" child comes next;
//      - the live edge count E, updated by each removal and restore;
//  * a warp runs its lanes in lock step: per iteration each lane does up to
//    kLaneOps vertex removals or restores, then, with nothing pending, one
//    reduction pass: a branch-free SWAR scan of its degree words (four
//    vertices per instruction) that marks the high-degree vertices and
//    gathers the degree-1 and degree-2-on-a-triangle candidates, whose
//    neighbours are read from the bitmap rows.  A pass without marks is the
//    node's fixpoint: a second scan finds the maximum degree and its lowest
//    vertex (one byte permute per vertex builds a (degree, -index) key);
//  * work sharing: a lane with a pending frame gives its OLDEST frame (the
//    largest subtree) away as a live bitmap: to a slot of the CTA's
//    shared-memory pool while lanes of the CTA are idle, else to the global
//    ring (bounded, lock-free, vc_search.cuh) while CTAs are idle.  A lane
//    that takes a record recounts its degrees from the bitmap.  Only a fully
//    idle CTA changes graphs: next root from the cursor, else a ring record;
//    termination is the (pending records, idle CTAs) word of vc_search.cuh;
//  * bounded waits only: ring claims give up, idle loops and the node loop
//    read %globaltimer against the launch's time limit.
#pragma once
#include "vc_dense.cuh"

namespace vcg {

constexpr uint32_t kLanePoolSlots = 32;  // CTA pool slots of the lane kernel
#ifndef VC_LANE_OPS
#define VC_LANE_OPS 4
#endif
constexpr int kLaneOps = VC_LANE_OPS;  // vertex removals / restores per lane per iteration
#ifndef VC_LANE_CAND_CAP
#define VC_LANE_CAND_CAP 8
#endif
constexpr uint32_t kLaneCandCap = VC_LANE_CAND_CAP;  // candidates examined per pass once a mark is found

// lane states
enum : uint32_t { kLsIdle = 0, kLsFresh = 1, kLsRun = 2, kLsRest = 3 };

// CTA control words of the lane kernel (static shared memory)
enum : uint32_t { kLhIdle = 0, kLhCount, kLhPoller, kLhReg, kLhExit, kLhGraph, kLhKey, kLhClosed, kLhWords = 8 };

// Shared-memory layout of a lane-kernel CTA in 32-bit words; nwc = words of a
// vertex set for the launch's largest graph (rows = 32 * nwc), NW = the
// kernel's register set width, NT = threads per CTA, PS = pool slots.
struct LaneLayout {
    uint32_t nwc, S, rows, tri, trim, sstate, sdata, claim, deg, trail, flg, words;
    VC_HD LaneLayout(uint32_t nwc_, uint32_t NW, uint32_t NT, uint32_t PS)
    {
        nwc = nwc_;
        S = NW == 8 ? 12u : NW;  // row stride: 16-byte row loads of 8 lanes in distinct banks
        rows = 32u * nwc;
        tri = rows * S;
        trim = tri + NW;
        sstate = trim + 8u * NW;
        sdata = sstate + PS;
        claim = sdata + PS * NW;
        deg = claim + NT;
        trail = deg + 8u * nwc * NT;
        flg = trail + 8u * nwc * NT;
        words = flg + nwc * NT;
    }
};

template <int NW>
__device__ __forceinline__ void lrow(const uint32_t *row, uint32_t (&r)[NW])
{
    if constexpr (NW % 4 == 0) {
#pragma unroll
        for (int w = 0; w < NW; w += 4) {
            const uint4 q = *reinterpret_cast<const uint4 *>(row + w);
            r[w] = q.x; r[w + 1] = q.y; r[w + 2] = q.z; r[w + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int w = 0; w < NW; w += 2) {
            const uint2 q = *reinterpret_cast<const uint2 *>(row + w);
            r[w] = q.x; r[w + 1] = q.y;
        }
    }
}

// Bit v of a register-held set.  The word is chosen by predicated selects
// written in PTX: written as a plain C++ select chain, the compiler turns it
// back into a dynamically indexed array, which lives in local memory.
template <int NW>
__device__ __forceinline__ void bit_set(uint32_t (&a)[NW], uint32_t v)
{
    const uint32_t b = 1u << (v & 31u), q = v >> 5;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t msk;
        asm("{.reg .pred p; setp.eq.u32 p, %1, %2; selp.b32 %0, %3, 0, p;}" : "=r"(msk) : "r"(q), "r"((uint32_t)w), "r"(b));
        a[w] |= msk;
    }
}

template <int NW>
__device__ __forceinline__ void bit_clear(uint32_t (&a)[NW], uint32_t v)
{
    const uint32_t b = 1u << (v & 31u), q = v >> 5;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t msk;
        asm("{.reg .pred p; setp.eq.u32 p, %1, %2; selp.b32 %0, %3, 0, p;}" : "=r"(msk) : "r"(q), "r"((uint32_t)w), "r"(b));
        a[w] &= ~msk;
    }
}

template <int NW>
__device__ __forceinline__ bool bit_test(const uint32_t (&a)[NW], uint32_t v)
{
    const uint32_t b = 1u << (v & 31u), q = v >> 5;
    uint32_t x = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t msk;
        asm("{.reg .pred p; setp.eq.u32 p, %1, %2; selp.b32 %0, %3, 0, p;}" : "=r"(msk) : "r"(q), "r"((uint32_t)w), "r"(b));
        x |= a[w] & msk;
    }
    return x != 0u;
}

template <int NW>
__device__ __forceinline__ bool any_bit(const uint32_t (&a)[NW])
{
    uint32_t x = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) x |= a[w];
    return x != 0u;
}

// Lowest set bit of a set (kNone if empty).
template <int NW>
__device__ __forceinline__ uint32_t lowest_bit(const uint32_t (&a)[NW])
{
    uint32_t r = kNone;
#pragma unroll
    for (int w = NW - 1; w >= 0; --w)
        if (a[w]) r = 32u * w + (__ffs(a[w]) - 1);
    return r;
}

template <int NW>
__device__ __forceinline__ uint32_t highest_bit(const uint32_t (&a)[NW])
{
    uint32_t r = kNone;
#pragma unroll
    for (int w = 0; w < NW; ++w)
        if (a[w]) r = 32u * w + (31u - __clz(a[w]));
    return r;
}

template <int NW>
__device__ __forceinline__ uint32_t popc_set(const uint32_t (&a)[NW])
{
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) c += __popc(a[w]);
    return c;
}

// One search unit's per-lane views of the CTA's shared memory.
template <int NW, unsigned NT>
struct LaneMem {
    const uint32_t *adj;  // [rows][S]
    uint32_t S;
    uint32_t *degw;  // word q of this lane at degw[q * NT]
    uint8_t *deg8;   // byte array base of all lanes' degree words
    uint8_t *trl8;   // byte array base of all lanes' trails
    uint32_t *flg;   // flag word w of this lane at flg[w * NT]
    uint32_t tid;
    __device__ __forceinline__ uint8_t *dbyte(uint32_t v) const { return deg8 + 4u * ((v >> 2) * NT + tid) + (v & 3u); }
    __device__ __forceinline__ uint8_t *tbyte(uint32_t i) const { return trl8 + 4u * ((i >> 2) * NT + tid) + (i & 3u); }
    __device__ __forceinline__ const uint32_t *row(uint32_t v) const { return adj + v * S; }
};

// Subtract (sign < 0) or add one to the degree byte of every vertex of x.
template <int NW, unsigned NT>
__device__ __forceinline__ void degree_step(const LaneMem<NW, NT> &m, uint32_t (&x)[NW], int sign)
{
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t xw = x[w];
        while (xw) {
            const uint32_t t = 32u * w + (__ffs(xw) - 1);
            xw &= xw - 1;
            uint8_t *p = m.dbyte(t);
            *p = (uint8_t)(*p + sign);
        }
    }
}

// Remove vertex u from L: its live neighbours lose one degree, its own byte
// becomes 0, it is logged on the trail (flagged if it is a frame's branching
// vertex).
template <int NW, unsigned NT>
__device__ __forceinline__ void lane_remove(const LaneMem<NW, NT> &m, uint32_t (&L)[NW], uint32_t u, bool flagged,
                                            uint32_t &top, uint32_t &E, uint32_t &fbot)
{
    bit_clear(L, u);
    uint32_t x[NW];
    lrow<NW>(m.row(u), x);
#pragma unroll
    for (int w = 0; w < NW; ++w) x[w] &= L[w];
    E -= popc_set(x);
    degree_step<NW, NT>(m, x, -1);
    *m.dbyte(u) = 0;
    *m.tbyte(top) = (uint8_t)u;
    if (flagged) {
        m.flg[(top >> 5) * NT] |= 1u << (top & 31u);
        if (fbot == kNone) fbot = top;
    }
    top += 1;
}

// Pop and restore the newest trail vertex.  Returns true (with N(v) & L in P)
// when it was a frame's branching vertex v.
template <int NW, unsigned NT>
__device__ __forceinline__ bool lane_restore(const LaneMem<NW, NT> &m, uint32_t (&L)[NW], uint32_t (&P)[NW],
                                             uint32_t &top, uint32_t &E, uint32_t &fbot, unsigned long long &restored)
{
    top -= 1;
    const uint32_t u = *m.tbyte(top);
    uint32_t *fp = m.flg + (top >> 5) * NT;
    const uint32_t fw = *fp;
    const bool fl = (fw >> (top & 31u)) & 1u;
    bit_set(L, u);
    uint32_t x[NW];
    lrow<NW>(m.row(u), x);
#pragma unroll
    for (int w = 0; w < NW; ++w) x[w] &= L[w];
    const uint32_t du = popc_set(x);
    E += du;
    degree_step<NW, NT>(m, x, +1);
    *m.dbyte(u) = (uint8_t)du;
    restored += 1;
    if (fl) {
        *fp = fw & ~(1u << (top & 31u));
        if (fbot == top) fbot = kNone;
#pragma unroll
        for (int w = 0; w < NW; ++w) P[w] = x[w];
    }
    return fl;
}

// Degrees of every live vertex from scratch (a received record or a root).
template <int NW, unsigned NT>
__device__ __forceinline__ void lane_recount(const LaneMem<NW, NT> &m, const uint32_t (&L)[NW], uint32_t gn,
                                             uint32_t gnw, uint32_t &E)
{
    uint32_t R[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) R[w] = L[w];
    uint32_t sum = 0;
#pragma unroll 1
    for (uint32_t w = 0; w < gnw; ++w) {
        const uint32_t lw = R[0];
#pragma unroll
        for (int i = 0; i < NW - 1; ++i) R[i] = R[i + 1];
        R[NW - 1] = 0;
#pragma unroll 1
        for (uint32_t j = 0; j < 8; ++j) {
            uint32_t word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const uint32_t v = 32u * w + 4u * j + b;
                if (((lw >> (4u * j + b)) & 1u) && v < gn) {
                    uint32_t r[NW];
                    lrow<NW>(m.row(v), r);
                    uint32_t c = 0;
#pragma unroll
                    for (int k = 0; k < NW; ++k) c += __popc(r[k] & L[k]);
                    word |= c << (8 * b);
                    sum += c;
                }
            }
            m.degw[(8u * w + j) * NT] = word;
        }
    }
    E = sum / 2;
}

// One reduction pass on the lane's degrees (same rules as dense_pass in
// vc_dense.cuh).  Returns true with the marks in P; otherwise the node is at
// its fixpoint and maxd / amax hold the maximum degree and its lowest vertex.
template <int NW, unsigned NT>
__device__ __forceinline__ bool lane_pass(const LaneMem<NW, NT> &m, const uint32_t *trim, const uint32_t (&L)[NW],
                                          uint32_t (&P)[NW], uint32_t gnw, uint32_t del, uint32_t bound,
                                          uint32_t &maxd, uint32_t &amax)
{
    const int tt = (int)bound - (int)del;  // the high-degree rule takes deg >= tt
    const uint32_t tl = (uint32_t)(tt & 0x7F) * 0x01010101u;
    uint32_t C[NW], M[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) C[w] = M[w] = 0u;
#pragma unroll 1
    for (uint32_t w = 0; w < (uint32_t)NW; ++w) {
        uint32_t cw = 0, mw = 0;
        if (w < gnw) {
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const uint32_t q = 8u * w + b;
                const uint32_t d = m.degw[q * NT];
                const uint32_t nz = ~bytes_zero(d) & 0x80808080u;
                const uint32_t lo = ((d | 0x80808080u) - tl) & 0x80808080u;  // low 7 bits >= tt's
                const uint32_t mid = tt < 128 ? ((d & 0x80808080u) | lo) : (d & lo);
                const uint32_t ge = tt <= 1 ? nz : (tt > 255 ? 0u : mid);
                const uint32_t c = (bytes_zero(d ^ 0x01010101u) | (bytes_zero(d ^ 0x02020202u) & trim[q])) & ~ge;
                cw |= gather4(c) << (4 * b);
                mw |= gather4(ge) << (4 * b);
            }
        }
#pragma unroll
        for (int i = 0; i < NW - 1; ++i) { C[i] = C[i + 1]; M[i] = M[i + 1]; }
        C[NW - 1] = cw;
        M[NW - 1] = mw;
    }
#pragma unroll
    for (int w = 0; w < NW; ++w) P[w] = M[w];
    bool marked = any_bit(M);
    uint32_t seen = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t cw = C[w];
        while (cw) {
            if (marked && seen >= kLaneCandCap) break;
            const uint32_t v = 32u * w + (__ffs(cw) - 1);
            cw &= cw - 1;
            ++seen;
            const uint32_t dv = *m.dbyte(v);
            uint32_t x[NW];
            lrow<NW>(m.row(v), x);
#pragma unroll
            for (int k = 0; k < NW; ++k) x[k] &= L[k];
            const uint32_t n1 = lowest_bit(x);
            if (n1 == kNone) continue;  // (degree bookkeeping guarantees a live neighbour)
            if (dv == 1) {  // degree-one rule (helperFunctions.cuh:252-265)
                const uint32_t du = *m.dbyte(n1);
                if (du > 1 || n1 < v) {
                    bit_set(P, n1);
                    marked = true;
                }
            } else {  // degree-two triangle rule (helperFunctions.cuh:384-417)
                const uint32_t n2 = highest_bit(x);
                if (n2 == n1) continue;
                const uint32_t d1 = *m.dbyte(n1), d2 = *m.dbyte(n2);
                const bool keep = d1 == 1 || d2 == 1 || (d1 == 2 && n1 < v) || (d2 == 2 && n2 < v);
                if (!keep && ((m.row(n2)[n1 >> 5] >> (n1 & 31u)) & 1u)) {
                    bit_set(P, n1);
                    bit_set(P, n2);
                    marked = true;
                }
            }
        }
    }
    if (marked) return true;
    // fixpoint: the largest (degree, -index) key over the live vertices
    uint32_t key = 0, idxw = 0xFCFDFEFFu;  // 255 - (4q + b) in byte b
#pragma unroll 4
    for (uint32_t q = 0; q < 8u * gnw; ++q) {
        const uint32_t d = m.degw[q * NT];
        const uint32_t k0 = __byte_perm(d, idxw, 0x0400u), k1 = __byte_perm(d, idxw, 0x1511u);
        const uint32_t k2 = __byte_perm(d, idxw, 0x2622u), k3 = __byte_perm(d, idxw, 0x3733u);
        key = max(key, max(max(k0, k1), max(k2, k3)));
        idxw -= 0x04040404u;
    }
    maxd = key >> 24;
    amax = 255u - ((key >> 16) & 0xFFu);
    return false;
}

// The lane's oldest frame as a record: the live set at that frame minus N(v)
// (written to dst[0..NW)), and the frame removed from the lane's stack.
template <int NW, unsigned NT>
__device__ __forceinline__ void lane_donate(const LaneMem<NW, NT> &m, const uint32_t (&L)[NW], uint32_t top,
                                            uint32_t &fbot, uint32_t gnw, uint32_t *dst, bool global_dst)
{
    const uint32_t p = fbot;
    const uint32_t v = *m.tbyte(p);
    uint32_t X[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) X[w] = L[w];
    for (uint32_t i = p; i < top; ++i) bit_set(X, (uint32_t)*m.tbyte(i));
    uint32_t r[NW];
    lrow<NW>(m.row(v), r);
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const uint32_t x = X[w] & ~r[w];
        if (global_dst) __stcg(&dst[w], x);
        else dst[w] = x;
    }
    // drop the frame: clear its flag, find the next flagged position
    m.flg[(p >> 5) * NT] &= ~(1u << (p & 31u));
    uint32_t nb = kNone;
    for (uint32_t w = p >> 5; w < gnw; ++w) {
        uint32_t fw = m.flg[w * NT];
        if (w == (p >> 5)) fw &= (p & 31u) == 31u ? 0u : ~((2u << (p & 31u)) - 1u);
        if (fw) { nb = 32u * w + (__ffs(fw) - 1); break; }
    }
    fbot = nb;
}

// Stage graph `inst` for the lane kernel (one warp): bitmap rows, the triangle
// bitmap and its byte masks.  Device-resident input is checked on the way:
// a decreasing or overlong row, a neighbour index out of range or a self loop
// marks the graph kBadGraph (and is skipped), so no write leaves the rows.
template <int NW>
__device__ __forceinline__ void stage_lanes(uint32_t *sm, const LaneLayout &lo, const Params &P, uint32_t inst)
{
    const unsigned lane = threadIdx.x & 31u;
    const InstDesc d = load_desc(&P.inst[inst]);
    const uint32_t *rp = P.row_ptr + d.row_off, *cl = P.col + d.col_off;
    uint32_t *adj = sm, *tri = sm + lo.tri, *trim = sm + lo.trim;
    for (uint32_t i = lane; i < lo.trim + 8u * NW; i += 32) sm[i] = 0;  // rows, tri and trim are contiguous
    __syncwarp();
    const uint32_t m2 = __ldcg(&rp[d.n]);
    bool bad = d.n > lo.rows || (d.m2 != kNone && m2 != d.m2) || __ldcg(&rp[0]) != 0u;
    if (!bad) {
        for (uint32_t v = lane; v < d.n; v += 32) {
            uint32_t *row = adj + v * lo.S;
            const uint32_t e0 = __ldcg(&rp[v]), e1 = __ldcg(&rp[v + 1]);
            if (e1 < e0 || e1 > m2) { bad = true; continue; }
            for (uint32_t e = e0; e < e1; ++e) {
                const uint32_t u = __ldcg(&cl[e]);
                if (u >= d.n || u == v) { bad = true; continue; }
                row[u >> 5] |= 1u << (u & 31u);
            }
        }
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) atomicOr(&P.st[inst].flags, kBadGraph);
    } else {
        // tri: v has a neighbour u with a common neighbour (only such a vertex
        // can ever meet the triangle rule)
        for (uint32_t v = lane; v < d.n; v += 32) {
            uint32_t r[NW];
            lrow<NW>(adj + v * lo.S, r);
            bool t = false;
#pragma unroll 1
            for (uint32_t w = 0; w < (uint32_t)NW && !t; ++w) {
                uint32_t x = adj[v * lo.S + w];
                while (x && !t) {
                    const uint32_t u = 32u * w + (__ffs(x) - 1);
                    x &= x - 1;
                    uint32_t c = 0;
#pragma unroll
                    for (int k = 0; k < NW; ++k) c |= adj[u * lo.S + k] & r[k];
                    t = c != 0u;
                }
            }
            if (t) atomicOr(&tri[v >> 5], 1u << (v & 31u));
        }
    }
    __syncwarp();
    for (uint32_t q = lane; q < 8u * NW; q += 32) trim[q] = spread4((tri[q >> 3] >> (4u * (q & 7u))) & 0xFu) << 7;
    __threadfence_block();
    __syncwarp();
}

// A fully idle CTA gives back its token of graph g (the last token marks the
// graph done).
__device__ __forceinline__ void lane_release(const Params &P, uint32_t g)
{
    InstState &st = P.st[g];
    const InstDesc d = load_desc(&P.inst[g]);
    __threadfence();
    if (d.node_limit) {
        const unsigned long long tot = ld_relaxed_u64(&st.nodes);
        if (tot >= d.node_limit && old_act_pending(st)) atomicOr(&st.flags, kBudget);
    }
    const uint32_t old = atomicSub(&st.act, 1u);
    if (old == 1u) {
        st.t_done = globaltimer();
        __threadfence();
        atomicOr(&st.flags, kDone);
    }
}

// A leaf (no edge left) of one lane: MVC improvement or PVC success.
template <int NW>
__device__ __forceinline__ void lane_leaf(const Params &P, uint32_t g, uint32_t mode, uint32_t gn, uint32_t gnw,
                                          uint32_t cover_off, const uint32_t (&L)[NW], uint32_t del, uint32_t &best)
{
    InstState &st = P.st[g];
    bool write = false;
    if (mode == kModeMVC) {
        const uint32_t old = atomicMin(&st.best, del);
        if (del < old) {
            bool got = false;
            for (int it = 0; it < (1 << 20); ++it) {  // bounded lock acquisition
                if (atomicCAS(&st.lock, 0u, 1u) == 0u) { got = true; break; }
                __nanosleep(64);
            }
            if (!got) atomicOr(&st.flags, kError);
            else if (del < ld_relaxed_u32(&st.cover_size)) write = true;
            else atomicExch(&st.lock, 0u);
        }
        best = min(old, del);
    } else {
        const uint32_t old = atomicOr(&st.flags, kFound);
        write = !(old & kFound);
    }
    if (!write) return;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if ((uint32_t)w < gnw) {
            const uint32_t lo = 32u * w;
            const uint32_t valid = lo + 32u <= gn ? 0xffffffffu : (1u << (gn - lo)) - 1u;
            P.covers[cover_off + w] = ~L[w] & valid;
        }
    }
    __threadfence();
    st.cover_size = del;
    if (mode != kModeMVC) atomicMin(&st.best, del);
    __threadfence();
    if (mode == kModeMVC) atomicExch(&st.lock, 0u);
}

template <int NW, unsigned NT>
__device__ void lanes_main(const Params &P, uint32_t *sm, uint32_t *hdr)
{
    constexpr uint32_t FULL = 0xffffffffu;
    const LaneLayout lo(P.np / 32u, NW, NT, P.cta_slots);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint32_t *trim = sm + lo.trim;
    uint32_t *sstate = sm + lo.sstate, *sdata = sm + lo.sdata, *claim = sm + lo.claim + 32u * warp;
    LaneMem<NW, NT> m;
    m.adj = sm;
    m.S = lo.S;
    m.degw = sm + lo.deg + tid;
    m.deg8 = reinterpret_cast<uint8_t *>(sm + lo.deg);
    m.trl8 = reinterpret_cast<uint8_t *>(sm + lo.trail);
    m.flg = sm + lo.flg + tid;
    m.tid = tid;

    // this lane's search
    uint32_t L[NW], Pn[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) L[w] = Pn[w] = 0u;
    uint32_t ls = kLsIdle, top = 0, base = 0, E = 0, fbot = kNone;
    bool brk = false;
    uint32_t lnodes = 0;  // since the last flush
    unsigned long long n_nodes = 0, n_passes = 0, n_don = 0, n_recv = 0, n_rest = 0;
    // the warp's view of its graph (uniform across the warp)
    uint32_t g = kNone, gn = 0, gnw = 0, gmode = 0, gk = 0, gcover = 0, gflags = 0;
    unsigned long long glimit = 0, stw = 0;
    uint32_t best = 0;  // per lane: the cached incumbent, lowered by the lane's own leaves
    bool poller = false;  // lane 0 only
    uint32_t nap = 64;
    const unsigned long long deadline = globaltimer() + P.time_limit_ns;
    if (tid == 0) atomicCAS(&P.ctl[kT0], 0ull, globaltimer());
    uint32_t aborted = 0;  // sticky: the launch hit its time limit
    unsigned long long busy = 0, idle_cyc = 0, polls = 0, roots = 0;
    // phase cycles / occupancy of the statistics mode (VC_PHASE_TIMERS=1 builds only)
    unsigned long long c_rec = 0, c_ops = 0, c_pass = 0, c_share = 0, it_held = 0, lanes_held = 0, it_rec = 0;

    auto bind = [&](uint32_t gg) {
        const InstDesc d = load_desc(&P.inst[gg]);
        g = gg;
        gn = d.n;
        gnw = d.nw;
        gmode = d.mode;
        gk = d.k;
        gcover = d.cover_off;
        glimit = d.node_limit;
        uint32_t b = 0, f = 0;
        if (lane == 0) {
            b = ld_relaxed_u32(&P.st[gg].best);
            f = ld_relaxed_u32(&P.st[gg].flags);
        }
        best = __shfl_sync(FULL, b, 0);
        gflags = __shfl_sync(FULL, f, 0);
    };
    // warp-wide: add the lanes' node counts to the graph and check its budget
    auto flush = [&]() {
        const uint32_t tot = __reduce_add_sync(FULL, lnodes);
        lnodes = 0;
        if (lane == 0 && tot && g != kNone) {
            const unsigned long long all = atomicAdd(&P.st[g].nodes, (unsigned long long)tot) + tot;
            if (glimit && all >= glimit) atomicOr(&P.st[g].flags, kBudget);
        }
    };

    for (uint32_t it = 0;; ++it) {
        uint32_t am = __ballot_sync(FULL, ls != kLsIdle);
        if (am == 0) {
            // ---- the whole warp is idle: CTA control (one poller per CTA) or a nap
            uint32_t res = 0, slot = 0;
            unsigned long long qpos = 0;
            polls += 1;
            if (lane == 0) {
                if (vld(&hdr[kLhExit])) {
                    res = 3;
                } else if (globaltimer() > deadline) {
                    atomicExch(&P.ctl[kAbort], 1ull);
                    atomicExch(&hdr[kLhExit], 1u);
                    res = 3;
                } else if (vld(&hdr[kLhCount]) > 0) {
                    if (poller) { atomicExch(&hdr[kLhPoller], 0u); poller = false; }
                    res = 1;
                } else if (poller || atomicCAS(&hdr[kLhPoller], 0u, 1u) == 0u) {
                    poller = true;
                    const uint32_t cnt = vld(&hdr[kLhCount]);
                    __threadfence_block();
                    const bool cta_idle = cnt == 0 && vld(&hdr[kLhIdle]) == NT;
                    if (ld_relaxed_u64(&P.ctl[kAbort]) || ld_relaxed_u64(&P.ctl[kFinish])) {
                        atomicExch(&hdr[kLhExit], 1u);
                        res = 3;
                    } else if (cta_idle) {
                        const uint32_t gc = vld(&hdr[kLhGraph]);
                        if (gc != kNone) {
                            lane_release(P, gc);
                            hdr[kLhGraph] = kNone;
                        }
                        if (!vld(&hdr[kLhClosed])) {
                            uint32_t i = kNone;
                            if (claim_root(P, i)) {
                                if (vld(&hdr[kLhReg])) {
                                    atomicAdd(&P.ctl[kState], 0xffffffffffffffffull);  // idle CTAs-1
                                    hdr[kLhReg] = 0u;
                                }
                                slot = i;
                                res = 4;
                            } else {
                                hdr[kLhClosed] = 1u;
                            }
                        }
                        if (res == 0 && vld(&hdr[kLhClosed])) {
                            unsigned long long w = ld_relaxed_u64(&P.ctl[kState]);
                            if (!vld(&hdr[kLhReg])) {
                                w = atomicAdd(&P.ctl[kState], 1ull) + 1ull;
                                hdr[kLhReg] = 1u;
                            }
                            if ((w >> 32) > 0 && ring_claim_deq(P, qpos)) {
                                atomicAdd(&P.ctl[kState], 0xfffffffeffffffffull);  // pending-1, idle CTAs-1
                                hdr[kLhReg] = 0u;
                                res = 2;
                            } else if ((uint32_t)w == gridDim.x && (w >> 32) == 0) {
                                atomicExch(&P.ctl[kFinish], 1ull);
                                atomicExch(&hdr[kLhExit], 1u);
                                res = 3;
                            }
                        }
                    }
                    // a new root or ring record keeps the poller role until it is
                    // published: no other warp may find the CTA idle meanwhile
                    if (res == 3) { atomicExch(&hdr[kLhPoller], 0u); poller = false; }
                }
            }
            res = __shfl_sync(FULL, res, 0);
            if (res == 3) break;
            if (res == 4 || res == 2) {
                // a new root, or a ring record, for this CTA: stage its graph,
                // publish the record in pool slot 0 (the pool is empty)
                slot = __shfl_sync(FULL, slot, 0);
                qpos = __shfl_sync(FULL, qpos, 0);
                const uint32_t *rg = P.pool_data + (size_t)(qpos & P.q_mask) * P.stride;
                if (res == 2) __threadfence();
                const uint32_t inst = res == 4 ? slot : __ldcg(&rg[0]);
                const uint32_t key = __ldcg(&P.inst[inst].key);
                if (vld(&hdr[kLhKey]) != key) {
                    stage_lanes<NW>(sm, lo, P, inst);
                    if (lane == 0) hdr[kLhKey] = key;
                }
                const InstDesc d = load_desc(&P.inst[inst]);
                if (lane < (uint32_t)NW) {
                    uint32_t x;
                    if (res == 4) {
                        const uint32_t lo32 = 32u * lane;
                        x = lo32 + 32u <= d.n ? 0xffffffffu : (lo32 < d.n ? (1u << (d.n - lo32)) - 1u : 0u);
                    } else {
                        x = lane < d.nw ? __ldcg(&rg[4 + lane]) : 0u;
                    }
                    sdata[lane] = x;
                }
                __syncwarp();
                if (lane == 0) {
                    if (res == 2) {
                        __threadfence();
                        st_release_u64(&P.pool_seq[qpos & P.q_mask], qpos + P.q_mask + 1);
                    } else {
                        roots += 1;
                    }
                    hdr[kLhGraph] = inst;
                    __threadfence_block();
                    atomicExch(&sstate[0], 2u);
                    atomicAdd(&hdr[kLhCount], 1u);
                    __threadfence_block();
                    atomicExch(&hdr[kLhPoller], 0u);
                    poller = false;
                }
                __syncwarp();
                nap = 64;
                continue;
            }
            if (res == 0) {
                if (lane == 0) __nanosleep(nap);
                nap = nap < (poller ? 4096u : kIdleNapMax) ? nap * 2 : (poller ? 4096u : kIdleNapMax);
                __syncwarp();
                continue;
            }
            nap = 64;
        }

        // ---- idle lanes take records from the CTA pool
        uint32_t taken = 0;
        const uint32_t idle = ~am;
        if (idle) {
            uint32_t cnt = 0;
            if (lane == 0) cnt = vld(&hdr[kLhCount]);
            cnt = __shfl_sync(FULL, cnt, 0);
            if (cnt) {
                const uint32_t want = __popc(idle);
                uint32_t got = 0, gg = kNone;
                if (lane == 0) {
                    if (poller) { atomicExch(&hdr[kLhPoller], 0u); poller = false; }
                    atomicSub(&hdr[kLhIdle], want);  // reserve first: the CTA never looks idle while work moves
                    __threadfence_block();
                    for (uint32_t i = 0; i < P.cta_slots && got < want; ++i)
                        if (atomicCAS(&sstate[i], 2u, 3u) == 2u) claim[got++] = i;
                    if (got) atomicSub(&hdr[kLhCount], got);
                    if (got < want) {
                        __threadfence_block();
                        atomicAdd(&hdr[kLhIdle], want - got);
                    }
                    gg = vld(&hdr[kLhGraph]);
                }
                got = __shfl_sync(FULL, got, 0);
                gg = __shfl_sync(FULL, gg, 0);
                __syncwarp();
                if (got) {
                    if (gg != g) {
                        flush();
                        bind(gg);
                    }
                    const uint32_t r = __popc(idle & ((1u << lane) - 1u));
                    if (((idle >> lane) & 1u) && r < got) {
                        const uint32_t s_ = claim[r];
                        const volatile uint32_t *d = sdata + s_ * NW;
#pragma unroll
                        for (int w = 0; w < NW; ++w) L[w] = d[w];
                        __threadfence_block();
                        atomicExch(&sstate[s_], 0u);
                        ls = kLsFresh;
                        n_recv += 1;
                    }
                    taken = __ballot_sync(FULL, ls == kLsFresh);
                }
            }
        }
        const uint32_t held = am | taken;  // lanes not counted idle in the CTA header
        if (held == 0) continue;

        // ---- the graph's state, every few iterations
        if ((it & 3u) == 0u) {
            uint32_t b = 0, f = 0;
            unsigned long long w = 0;
            if (lane == 0) {
                b = ld_relaxed_u32(&P.st[g].best);
                f = ld_relaxed_u32(&P.st[g].flags);
                w = ld_relaxed_u64(&P.ctl[kState]);
                if ((it & 255u) == 0u) {
                    if (ld_relaxed_u64(&P.ctl[kAbort])) aborted = kError;
                    else if (globaltimer() > deadline) { atomicExch(&P.ctl[kAbort], 1ull); aborted = kError; }
                }
                f |= aborted;
            }
            b = __shfl_sync(FULL, b, 0);
            best = min(best, b);
            gflags = __shfl_sync(FULL, f, 0);
            stw = __shfl_sync(FULL, w, 0);
        }
        if (gflags & (kFound | kBudget | kError | kBadGraph)) {
            // the graph needs no more work: drop it
            if (lane == 0 && !(gflags & (kFound | kBudget | kBadGraph))) atomicOr(&P.st[g].flags, kCut);
            ls = kLsIdle;
#pragma unroll
            for (int w = 0; w < NW; ++w) Pn[w] = 0u;
            fbot = kNone;
            flush();
            if (lane == 0) {
                __threadfence_block();
                atomicAdd(&hdr[kLhIdle], (uint32_t)__popc(held));
            }
            __syncwarp();
            continue;
        }

        const long long t0 = clock64();
        if (kPhaseTimers) {
            it_held += 1;
            lanes_held += __popc(held);
            it_rec += __any_sync(FULL, ls == kLsFresh) ? 1u : 0u;
        }
        // ---- a received record: degrees from scratch
        if (ls == kLsFresh) {
            lane_recount<NW, NT>(m, L, gn, gnw, E);
            top = 0;
            base = gn - popc_set(L);
            fbot = kNone;
            brk = false;
#pragma unroll
            for (int w = 0; w < NW; ++w) Pn[w] = 0u;
            for (uint32_t w = 0; w < gnw; ++w) m.flg[w * NT] = 0u;
            ls = kLsRun;
        }
        long long tp = 0;
        if (kPhaseTimers) { __syncwarp(); tp = clock64(); c_rec += (unsigned long long)(tp - t0); }
        // ---- vertex removals / restores.  A pending set of forced vertices (rule
        // marks, or N(v) of a right child) that already reaches the bound ends the
        // node as its reduction would (del >= best for MVC, del > k for PVC),
        // without removing them one by one.
        if (ls == kLsRun && !brk && any_bit(Pn)) {
            const uint32_t del_after = base + top + popc_set(Pn);
            if (gmode == kModeMVC ? del_after >= best : del_after > gk) {
#pragma unroll
                for (int w = 0; w < NW; ++w) Pn[w] = 0u;
                lnodes += 1;
                n_nodes += 1;
                ls = top == 0 ? kLsIdle : kLsRest;
            }
        }
#pragma unroll 1
        for (int r = 0; r < kLaneOps; ++r) {
            if (ls == kLsRest) {
                if (top == 0) { ls = kLsIdle; break; }
                if (lane_restore<NW, NT>(m, L, Pn, top, E, fbot, n_rest)) ls = kLsRun;
            } else if (ls == kLsRun && any_bit(Pn)) {
                const uint32_t u = lowest_bit(Pn);
                bit_clear(Pn, u);
                if (bit_test(L, u)) lane_remove<NW, NT>(m, L, u, brk, top, E, fbot);
                brk = false;
            } else {
                break;
            }
        }
        if (kPhaseTimers) { __syncwarp(); const long long t = clock64(); c_ops += (unsigned long long)(t - tp); tp = t; }
        // ---- one reduction pass, and the node's decision at its fixpoint
        if (ls == kLsRun && !any_bit(Pn)) {
            const uint32_t del = base + top;
            const uint32_t bound = gmode == kModeMVC ? best : gk + 1;
            uint32_t maxd = 0, amax = 0;
            n_passes += 1;
            if (!lane_pass<NW, NT>(m, trim, L, Pn, gnw, del, bound, maxd, amax)) {
                lnodes += 1;
                n_nodes += 1;
                bool prune;
                if (gmode == kModeMVC) {
                    prune = del >= best;
                    if (!prune) {
                        const uint64_t b = (uint64_t)(best - del - 1);
                        prune = (uint64_t)E >= b * b + 1;
                    }
                } else {
                    prune = del > gk;
                    if (!prune) {
                        const uint64_t b = (uint64_t)(gk - del);
                        prune = (uint64_t)E >= b * b + 1;
                    }
                }
                if (!prune && maxd == 0) {
                    lane_leaf<NW>(P, g, gmode, gn, gnw, gcover, L, del, best);
                    prune = true;
                }
                if (prune) {
                    ls = top == 0 ? kLsIdle : kLsRest;
                } else {
                    bit_set(Pn, amax);  // the "take v" child; the frame is its flagged trail entry
                    brk = true;
                }
            }
        }
        if (kPhaseTimers) __syncwarp();
        const long long t1 = clock64();
        busy += (unsigned long long)(t1 - t0);
        if (kPhaseTimers) c_pass += (unsigned long long)(t1 - tp);

        // ---- work sharing: the oldest frame of a lane, to idle lanes of the CTA or to idle CTAs
        const uint32_t cand = __ballot_sync(FULL, ls == kLsRun && fbot != kNone);
        if (cand) {
            uint32_t want = 0, ring = 0;
            if (lane == 0) {
                const uint32_t li = vld(&hdr[kLhIdle]), lc = vld(&hdr[kLhCount]);
                if (li > lc) want = min(li - lc, (uint32_t)__popc(cand));
                else if ((long long)(uint32_t)stw - (long long)(stw >> 32) > (long long)P.ring_bias) ring = 1;
            }
            want = __shfl_sync(FULL, want, 0);
            ring = __shfl_sync(FULL, ring, 0);
            if (want) {
                uint32_t got = 0;
                if (lane == 0) {
                    for (uint32_t i = 0; i < P.cta_slots && got < want; ++i)
                        if (atomicCAS(&sstate[i], 0u, 1u) == 0u) claim[got++] = i;
                }
                got = __shfl_sync(FULL, got, 0);
                __syncwarp();
                const uint32_t r = __popc(cand & ((1u << lane) - 1u));
                if (((cand >> lane) & 1u) && r < got) {
                    const uint32_t s_ = claim[r];
                    lane_donate<NW, NT>(m, L, top, fbot, gnw, sdata + s_ * NW, false);
                    __threadfence_block();
                    atomicExch(&sstate[s_], 2u);
                    n_don += 1;
                }
                __syncwarp();
                if (lane == 0 && got) atomicAdd(&hdr[kLhCount], got);
            } else if (ring) {
                unsigned long long qpos = 0;
                uint32_t ok = 0;
                if (lane == 0) {
                    atomicAdd(&P.ctl[kState], 1ull << 32);
                    if (ring_claim_enq(P, qpos)) ok = 1;
                    else atomicAdd(&P.ctl[kState], 0xffffffff00000000ull);
                }
                ok = __shfl_sync(FULL, ok, 0);
                if (ok) {
                    qpos = __shfl_sync(FULL, qpos, 0);
                    stw += 1ull << 32;
                    const uint32_t donor = __ffs(cand) - 1;
                    if (lane == donor) {
                        uint32_t *slot = P.pool_data + (size_t)(qpos & P.q_mask) * P.stride;
                        atomicAdd(&P.st[g].act, 1u);
                        __stcg(&slot[0], g);
                        lane_donate<NW, NT>(m, L, top, fbot, gnw, slot + 4, true);
                        __threadfence();
                        st_release_u64(&P.pool_seq[qpos & P.q_mask], qpos + 1);
                        n_don += 1;
                    }
                    __syncwarp();
                }
            }
        }

        // ---- lanes that ran out of work this iteration
        const uint32_t now_idle = held & ~__ballot_sync(FULL, ls != kLsIdle);
        if (now_idle || (it & 31u) == 0u) flush();
        if (now_idle && lane == 0) {
            __threadfence_block();
            atomicAdd(&hdr[kLhIdle], (uint32_t)__popc(now_idle));
        }
        const long long t2 = clock64();
        idle_cyc += (unsigned long long)(t2 - t1);
        if (kPhaseTimers) c_share += (unsigned long long)(t2 - t1);
    }
    if (P.stats) {
        unsigned long long *o = P.stats + ((size_t)blockIdx.x * NT + tid) * kStatWords;
        uint32_t smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        o[kStNodes] = n_nodes;
        o[kStPasses] = n_passes;
        o[kStDonations] = n_don;
        o[kStDonateFail] = 0;
        o[kStReceives] = n_recv;
        o[kStRoots] = roots;
        o[kStBusyCycles] = busy;
        o[kStIdleCycles] = idle_cyc;
        o[kStPolls] = polls;
        o[kStRestored] = n_rest;
        o[kStSmid] = smid;
        if (kPhaseTimers) {
            o[kStCycScan] = c_pass;
            o[kStCycApply] = c_ops;
            o[kStCycPop] = c_rec;
            o[kStCycBranch] = c_share;
            o[kStCycOther] = it_held;
            o[kStDonateFail] = lanes_held;
            o[kStRoots] = it_rec;
        }
    }
}

}  // namespace vcg
