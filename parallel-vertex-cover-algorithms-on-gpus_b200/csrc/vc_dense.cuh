// vc_dense.cuh -- the search for graphs of at most 255 vertices (the batched
// workload's G(n, p) instances, n in [30, 200], and the 60-vertex case), and,
// with 20-word rows, for graphs of up to 640 vertices whose degrees all fit a
// byte (at most 254); with 16- and 32-word rows and 16-bit degrees (two to a
// word, see "Half" below), for graphs of up to 512 and 1024 vertices of any
// degree -- the dense DIMACS-style graphs the CSR walks handle worst.
//
// Same search as vc_search.cuh (the reference's degree-one, triangle and
// high-degree rules, the E > b^2 prune and max-degree branching), with dense
// bitsets instead of CSR walks:
//
//  * a CTA works on one graph at a time: its adjacency is staged once into
//    shared memory as one NW-word bitmap per vertex (NW = 8: 8 KB) and shared
//    by the CTA's warps, which split the graph's search tree among themselves
//    through the CTA pool (vc_search.cuh);
//  * one warp is one search unit; its node state is the live-vertex set L (NW
//    words in shared memory, word w kept by lane w; copied into registers
//    where a whole row is masked with it); a vertex taken into the cover
//    leaves L, so del = n - |L| and the cover is the complement of L;
//  * deg(v) = popc(adj[v] & L), kept as bytes (0 = removed or isolated), four
//    to a 32-bit word: lane l holds words l and l + 32 in registers, so the
//    rule tests of a pass look at four vertices per instruction (SWAR byte
//    arithmetic).  When a set M leaves L, only the rows of M are read: each
//    lane subtracts the 4-bit slices of those rows that cover its vertices
//    (the adjacency is symmetric).  After a backtrack the degrees are
//    recounted, one vertex per lane;
//  * the triangle test of a degree-2 vertex is one bit test and the leaf
//    rule's neighbour one find-first-set: no serial CSR row walks;
//  * backtracking: an undo trail of removed ids (u16) and frames of (trail
//    position, branching vertex); restoring ORs bits back into L.
//
// Records exchanged through the CTA pool and the global ring are live bitmaps.
#pragma once
#include "vc_search.cuh"

namespace vcg {

template <int NW>
struct Rows {
    static constexpr bool kHalf = NW == 16 || NW == 32;  // 16-bit degrees (dense_half)
    static constexpr int kStride = NW == 8 ? 12 : (NW == 16 ? 20 : NW);  // dense_row_words
    static constexpr bool kSwz = NW == 32;  // 16-byte chunks of a row XOR-swizzled by the row's low 3 bits
    // Index of word w of row v.
    static __device__ __forceinline__ uint32_t at(uint32_t v, uint32_t w)
    {
        return v * kStride + (kSwz ? ((((w >> 2) ^ (v & 7u)) << 2) | (w & 3u)) : w);
    }
    static constexpr int kPer = kHalf ? 2 : 4;                             // degrees per word
    static constexpr int kJ = kHalf ? NW / 2 : (NW >= 8 ? NW / 4 : 1);     // degree words per lane
    // bits of a lane's candidate count (at most kPer * kJ)
    static constexpr int kCandBits = kPer * kJ >= 32 ? 6 : (kPer * kJ >= 16 ? 5 : (kPer * kJ >= 8 ? 4 : 3));
    static constexpr int kTri = 32 * NW * kStride;          // offset of the triangle bitmap
};

// 0x80 in every byte of x that is zero, 0 elsewhere.
__device__ __forceinline__ uint32_t bytes_zero(uint32_t x)
{
    return ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);
}

// 4 bits -> the low bit of each of 4 bytes (bit b to bit 8b).
__device__ __forceinline__ uint32_t spread4(uint32_t nib) { return (nib * 0x00204081u) & 0x01010101u; }

// The top bits of 4 bytes (bit 8b+7) -> 4 bits (bit b).
__device__ __forceinline__ uint32_t gather4(uint32_t hb) { return ((hb >> 7) * 0x01020408u) >> 24; }

// Half: the same tests on two 16-bit degrees per word (values below 2^15).
// 0x8000 in every halfword of x that is zero, 0 elsewhere.
__device__ __forceinline__ uint32_t halves_zero(uint32_t x)
{
    return ~(((x & 0x7FFF7FFFu) + 0x7FFF7FFFu) | x | 0x7FFF7FFFu);
}

// 2 bits -> the low bit of each halfword.
__device__ __forceinline__ uint32_t spread2(uint32_t b) { return (b & 1u) | ((b & 2u) << 15); }

// The top bits of 2 halfwords (bits 15, 31) -> 2 bits.
__device__ __forceinline__ uint32_t gather2(uint32_t hb) { return ((hb >> 15) & 1u) | ((hb >> 30) & 2u); }

// extra CTA header words used by the dense kernel
enum : uint32_t { kCpStaged = 5, kCpCursorClosed = 6 };

// Per-phase cycle counters of the statistics mode (vc_debug_stats) cost a
// clock read and a branch per phase even when off, so they are compiled in
// only with VC_PHASE_TIMERS=1.
#ifndef VC_PHASE_TIMERS
#define VC_PHASE_TIMERS 0
#endif
constexpr bool kPhaseTimers = VC_PHASE_TIMERS != 0;

struct PhaseCycles {
    unsigned long long scan, apply, pop, branch;
};

template <int NW>
struct DSU {
    SUStat stat;
    PhaseCycles cyc;
    bool timed;
    const uint32_t *adj;  // CTA-shared [32*NW][kStride] rows, then the triangle bitmap
    uint8_t *ws;          // this warp's workspace; the arrays below sit at fixed offsets
    __device__ __forceinline__ uint32_t *frames() const { return reinterpret_cast<uint32_t *>(ws); }  // [32*NW] (trail position << 16) | vertex
    __device__ __forceinline__ uint32_t *marks() const { return frames() + 32 * NW; }  // [NW]
    __device__ __forceinline__ uint32_t *bits() const { return marks() + NW; }         // [NW] record / scratch
    __device__ __forceinline__ uint32_t *lsm() const { return bits() + NW; }           // [NW] the live set L
    __device__ __forceinline__ uint16_t *trail() const { return reinterpret_cast<uint16_t *>(lsm() + NW); }  // [32*NW]
    __device__ __forceinline__ uint16_t *cand() const { return trail() + 32 * NW; }   // [32*NW] pass candidates
    __device__ __forceinline__ uint8_t *degs() const { return reinterpret_cast<uint8_t *>(cand() + 32 * NW); }  // [32*NW] staging copy of D
    __device__ __forceinline__ uint16_t *degs16() const { return reinterpret_cast<uint16_t *>(cand() + 32 * NW); }  // the same, Half
    uint32_t D[Rows<NW>::kJ];   // degree bytes of vertices 4q..4q+3, q = 32j + lane (Half: 16-bit degrees of 2q, 2q+1)
    uint32_t Ln[Rows<NW>::kJ];  // their live bits (4 per word; Half: 2)
    const uint32_t *rp, *cl;
    uint32_t inst, n, nw, mode, k, cover_off;
    unsigned long long node_limit;
    uint32_t base_del, top;
    uint32_t c_best;
    uint32_t fr_bot, fr_top;
    uint32_t pending;  // how the next node starts: kPendApply / kPendRecount with the set in marks
    unsigned long long local_nodes;
    unsigned long long deadline;
};

enum : uint32_t { kPendApply = 1, kPendRecount = 2 };

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <int NW>
__device__ __forceinline__ void dsu_bind(DSU<NW> &s, uint8_t *ws, const uint32_t *adj)
{
    s.adj = adj;
    s.ws = ws;
}

template <int NW>
__device__ __forceinline__ uint32_t *rec_bits(DSU<NW> &s) { return s.bits(); }

// Loads the first nw (runtime, uniform) words of a row; the rest read as 0.
template <int NW>
__device__ __forceinline__ void load_row(const uint32_t *row, uint32_t (&r)[NW], uint32_t nw)
{
    if constexpr (NW % 4 == 0) {
#pragma unroll
        for (int w = 0; w < NW; w += 4) {
            if ((uint32_t)w < nw) {
                const uint4 q = *reinterpret_cast<const uint4 *>(row + w);
                r[w] = q.x; r[w + 1] = q.y; r[w + 2] = q.z; r[w + 3] = q.w;
            } else {
                r[w] = r[w + 1] = r[w + 2] = r[w + 3] = 0u;
            }
        }
    } else {
#pragma unroll
        for (int w = 0; w < NW; w += 2) {
            const uint2 q = *reinterpret_cast<const uint2 *>(row + w);
            r[w] = q.x; r[w + 1] = q.y;
        }
    }
}

// Row v of the adjacency (logical word order) into registers.
template <int NW>
__device__ __forceinline__ void load_row_at(const uint32_t *adj, uint32_t v, uint32_t (&r)[NW])
{
    if constexpr (Rows<NW>::kSwz) {
        const uint32_t sw = v & 7u;
#pragma unroll
        for (int c = 0; c < NW / 4; ++c) {
            const uint4 q = *reinterpret_cast<const uint4 *>(adj + v * Rows<NW>::kStride + 4u * ((uint32_t)c ^ sw));
            r[4 * c] = q.x; r[4 * c + 1] = q.y; r[4 * c + 2] = q.z; r[4 * c + 3] = q.w;
        }
    } else {
        load_row<NW>(adj + v * Rows<NW>::kStride, r, NW);
    }
}

// All NW words of L into registers.
template <int NW>
__device__ __forceinline__ void load_L(const DSU<NW> &s, uint32_t (&L)[NW])
{
    load_row<NW>(s.lsm(), L, NW);
}

// The live bits of this lane's degree words (from the mirror of L).
template <int NW>
__device__ __forceinline__ void live_nibbles(DSU<NW> &s)
{
    const unsigned lane = lane_id();
#pragma unroll
    for (int j = 0; j < Rows<NW>::kJ; ++j) {
        const uint32_t q = 32u * j + lane;
        if constexpr (Rows<NW>::kHalf)
            s.Ln[j] = q < 16u * s.nw ? (s.lsm()[q >> 4] >> (2u * (lane & 15u))) & 0x3u : 0u;
        else
            s.Ln[j] = q < 8u * s.nw ? (s.lsm()[q >> 3] >> (4u * (lane & 7u))) & 0xFu : 0u;
    }
}

// Degrees from scratch into the staging array, then each lane picks up its
// words.  With 4-word row chunks (NW = 8, 16, 20, 32) only the live vertices
// are counted -- listed by a prefix sum over the words of L, then one per lane
// -- and only over the chunks of L that hold a live vertex; the staging array
// is zeroed first, so removed and padding vertices read 0.  Deep in a dense
// graph's tree most vertices are gone, and this is most of a node's work.
template <int NW>
__device__ __forceinline__ void dense_degrees(DSU<NW> &s)
{
    const unsigned lane = lane_id();
    uint32_t L[NW];
    load_L(s, L);
    if constexpr (NW % 4 == 0) {
        constexpr int C = NW / 4;
        uint32_t nzc = 0;  // chunks of L with a live vertex (the same in every lane)
#pragma unroll
        for (int c = 0; c < C; ++c) nzc |= (uint32_t)((L[4 * c] | L[4 * c + 1] | L[4 * c + 2] | L[4 * c + 3]) != 0u) << c;
        uint32_t *d32 = reinterpret_cast<uint32_t *>(s.degs());
        constexpr uint32_t kStageWords = 32u * NW / Rows<NW>::kPer;
        for (uint32_t i = lane; i < kStageWords; i += 32) d32[i] = 0u;
        const uint32_t x = lane < (uint32_t)NW ? s.lsm()[lane] : 0u;
        const uint32_t cnt = __popc(x);
        uint32_t off = cnt;  // inclusive prefix over the words of L
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, off, d);
            if (lane >= (unsigned)d) off += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, off, 31);
        uint16_t *list = s.cand();  // free while the degrees are recounted
        uint32_t pos = off - cnt, m = x;
        while (m) {
            list[pos++] = (uint16_t)(32u * lane + (__ffs(m) - 1));
            m &= m - 1;
        }
        __syncwarp();
        for (uint32_t i = lane; i < total; i += 32) {
            const uint32_t v = list[i];
            const uint4 *row = reinterpret_cast<const uint4 *>(s.adj + v * Rows<NW>::kStride);
            const uint32_t sw = Rows<NW>::kSwz ? (v & 7u) : 0u;
            uint32_t c = 0;
#pragma unroll
            for (int k = 0; k < C; ++k) {
                if ((nzc >> k) & 1u) {
                    const uint4 r = row[(uint32_t)k ^ sw];
                    c += __popc(r.x & L[4 * k]) + __popc(r.y & L[4 * k + 1]) + __popc(r.z & L[4 * k + 2]) +
                         __popc(r.w & L[4 * k + 3]);
                }
            }
            if constexpr (Rows<NW>::kHalf) s.degs16()[v] = (uint16_t)c;
            else s.degs()[v] = (uint8_t)c;
        }
    } else {  // 2- and 4-word graphs: one vertex per lane
        const int kmax = (int)s.nw;
#pragma unroll 1
        for (int k = 0; k < kmax; ++k) {
            const uint32_t v = lane + 32u * k;
            uint32_t c = 0;
            if (v < s.n && ((s.lsm()[k] >> lane) & 1u)) {
                uint32_t r[NW];
                load_row<NW>(s.adj + v * Rows<NW>::kStride, r, NW);
#pragma unroll
                for (int w = 0; w < NW; ++w) c += __popc(r[w] & L[w]);
            }
            s.degs()[v] = (uint8_t)c;
        }
    }
    __syncwarp();
    const uint32_t *d32 = reinterpret_cast<const uint32_t *>(s.degs());
    constexpr uint32_t kWordsPerLsm = 32u / Rows<NW>::kPer;  // degree words per word of L
#pragma unroll
    for (int j = 0; j < Rows<NW>::kJ; ++j) {
        const uint32_t q = 32u * j + lane;
        s.D[j] = q < kWordsPerLsm * s.nw ? d32[q] : 0u;
    }
    live_nibbles(s);
}

// Log the vertices of the set in s.marks() on the trail (ascending) and drop
// them from L; lane w handles word w.
template <int NW>
__device__ __forceinline__ void dense_push(DSU<NW> &s)
{
    const unsigned lane = lane_id();
    const uint32_t mw = lane < NW ? s.marks()[lane] : 0u;
    const uint32_t c = __popc(mw);
    uint32_t off = c;  // inclusive prefix over the words
#pragma unroll
    for (int d = 1; d < NW; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, off, d);
        if (lane >= (unsigned)d) off += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, off, NW - 1);
    uint32_t pos = s.top + off - c, m = mw;
    while (m) {
        s.trail()[pos++] = (uint16_t)(32u * lane + (__ffs(m) - 1));
        m &= m - 1;
    }
    if (lane < NW) s.lsm()[lane] &= ~mw;
    s.top += total;
    __syncwarp();
}

// Put the trail above `pos` back into L.
template <int NW>
__device__ __forceinline__ void dense_restore(DSU<NW> &s, uint32_t pos)
{
    const unsigned lane = lane_id();
    if (lane < NW) s.bits()[lane] = 0;
    __syncwarp();
    for (uint32_t i = pos + lane; i < s.top; i += 32) {
        uint32_t u = s.trail()[i];
        atomicOr(&s.bits()[u >> 5], 1u << (u & 31u));
    }
    __syncwarp();
    if (lane < NW) s.lsm()[lane] |= s.bits()[lane];
    s.stat.restored += s.top - pos;
    s.top = pos;
    __syncwarp();
}

// The set in s.marks() has just left L (trail, L and its mirror already
// updated): subtract its edges from the degrees of the live vertices and zero
// the bytes of the removed ones.
template <int NW>
__device__ __forceinline__ void dense_apply_half(DSU<NW> &s)
{
    constexpr int J = Rows<NW>::kJ;
    const unsigned lane = lane_id();
    live_nibbles(s);
    {
        // word 2j + lane/16 of a row holds the bits of this lane's vertices 2q, 2q+1
        const uint32_t sh = 2u * (lane & 15u);
        const uint32_t hl = lane >> 4;
        const uint32_t mw = lane < s.nw ? s.marks()[lane] : 0u;
        uint32_t wm = __ballot_sync(0xffffffffu, mw != 0u);
        uint32_t acc[J];
#pragma unroll
        for (int j = 0; j < J; ++j) acc[j] = 0u;
        while (wm) {
            const uint32_t w = __ffs(wm) - 1;
            wm &= wm - 1;
            uint32_t m = __shfl_sync(0xffffffffu, mw, w);
            while (m) {
                const uint32_t u = 32u * w + (__ffs(m) - 1);
                m &= m - 1;
#pragma unroll
                for (int j = 0; j < J; ++j) acc[j] += spread2((s.adj[Rows<NW>::at(u, 2u * j + hl)] >> sh) & s.Ln[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < J; ++j) s.D[j] = (s.D[j] - acc[j]) & (spread2(s.Ln[j]) * 0xFFFFu);
    }
}

template <int NW>
__device__ __forceinline__ void dense_apply(DSU<NW> &s)
{
    if constexpr (Rows<NW>::kHalf) {
        dense_apply_half(s);
        return;
    } else {
    constexpr int J = Rows<NW>::kJ;
    const unsigned lane = lane_id();
    live_nibbles(s);
    const uint32_t sh = 4u * (lane & 7u);
    const uint32_t *rows = s.adj + (lane >> 3);  // word 4j + lane/8 of a row holds this lane's bits
    const uint32_t mw = lane < s.nw ? s.marks()[lane] : 0u;  // lane w holds word w of the set
    uint32_t wm = __ballot_sync(0xffffffffu, mw != 0u);
    uint32_t acc[J];  // per-byte decrements (at most the degree, so no byte overflows)
#pragma unroll
    for (int j = 0; j < J; ++j) acc[j] = 0u;
    while (wm) {
        const uint32_t w = __ffs(wm) - 1;
        wm &= wm - 1;
        uint32_t m = __shfl_sync(0xffffffffu, mw, w);
        while (m) {  // two removed vertices per step
            const uint32_t u1 = 32u * w + (__ffs(m) - 1);
            m &= m - 1;
            const uint32_t *r1 = rows + u1 * Rows<NW>::kStride;
            if (m) {
                const uint32_t u2 = 32u * w + (__ffs(m) - 1);
                m &= m - 1;
                const uint32_t *r2 = rows + u2 * Rows<NW>::kStride;
#pragma unroll
                for (int j = 0; j < J; ++j)
                    acc[j] += spread4((r1[4 * j] >> sh) & s.Ln[j]) + spread4((r2[4 * j] >> sh) & s.Ln[j]);
            } else {
#pragma unroll
                for (int j = 0; j < J; ++j) acc[j] += spread4((r1[4 * j] >> sh) & s.Ln[j]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < J; ++j) s.D[j] = (s.D[j] - acc[j]) & (spread4(s.Ln[j]) * 0xFFu);
    }
}

// One reduction pass (same rules and semantics as reduce_pass in vc_search.cuh)
// on current degrees.  Byte tests over each lane's degree words find the
// high-degree vertices (marked at once) and the degree-1 ones and degree-2 ones
// on a triangle of the graph, which are gathered into a list and worked one
// vertex per lane.  Returns true if marks
// were made (left in s.marks()); otherwise fills o with the degree sum, the
// maximum degree and its lowest vertex.
template <int NW>
__device__ __forceinline__ bool dense_pass_byte(DSU<NW> &s, uint32_t del, uint32_t bound, ScanOut &o)
{
    constexpr int J = Rows<NW>::kJ;
    const unsigned lane = lane_id();
    const uint32_t sh = 4u * (lane & 7u);
    const int tt = (int)bound - (int)del;  // the high-degree rule takes deg >= tt
    const uint32_t tl = (uint32_t)(tt & 0x7F) * 0x01010101u;
    const uint32_t *tri = s.adj + Rows<NW>::kTri;
    bool marked = false;
    uint32_t cn[J], ctot = 0;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const uint32_t d = s.D[j];
        const uint32_t nz = ~bytes_zero(d) & 0x80808080u;
        const uint32_t lo = ((d | 0x80808080u) - tl) & 0x80808080u;  // low 7 bits >= tt's
        const uint32_t mid = tt < 128 ? ((d & 0x80808080u) | lo) : (d & lo);
        const uint32_t ge = tt <= 1 ? nz : (tt > 255 ? 0u : mid);
        // degree 1, or degree 2 on a triangle of the graph
        const uint32_t tn = (tri[(32u * j + lane) >> 3] >> sh) & 0xFu;
        const uint32_t d12 = bytes_zero(d ^ 0x01010101u) | (bytes_zero(d ^ 0x02020202u) & (spread4(tn) << 7));
        const uint32_t hn = gather4(ge);
        if (hn) {
            atomicOr(&s.marks()[(32u * j + lane) >> 3], hn << sh);
            marked = true;
        }
        cn[j] = gather4(d12 & ~ge);
        ctot += __popc(cn[j]);
    }
    // compact the degree-1/2 candidates (at most 4J per lane) into s.cand()
    // (one vote first: many passes have none)
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t pre = 0, total = 0;
    if (__any_sync(0xffffffffu, ctot != 0u)) {
#pragma unroll
        for (int b = 0; b < Rows<NW>::kCandBits; ++b) {
            const uint32_t bal = __ballot_sync(0xffffffffu, (ctot >> b) & 1u);
            pre += __popc(bal & lt) << b;
            total += __popc(bal) << b;
        }
    }
    if (total) {
        uint32_t *d32 = reinterpret_cast<uint32_t *>(s.degs());
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const uint32_t q = 32u * j + lane;
            if (q < 8u * s.nw) d32[q] = s.D[j];
            uint32_t m = cn[j];
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                s.cand()[pre++] = (uint16_t)(4u * q + b);
            }
        }
        uint32_t L[NW];
        load_L(s, L);
        __syncwarp();
        for (uint32_t i = lane; i < total; i += 32) {  // degree-one / degree-two triangle rules
            const uint32_t v = s.cand()[i];
            const uint32_t dv = s.degs()[v];
            uint32_t r[NW];
            load_row<NW>(s.adj + v * Rows<NW>::kStride, r, NW);
            // v has exactly dv (1 or 2) live neighbours: the lowest and the
            // highest set bit of row & L
            uint32_t n1 = kNone, hi = kNone;
#pragma unroll
            for (int w = NW - 1; w >= 0; --w) {
                const uint32_t x = r[w] & L[w];
                n1 = x ? 32u * w + (__ffs(x) - 1) : n1;
            }
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const uint32_t x = r[w] & L[w];
                hi = x ? 32u * w + (31u - __clz(x)) : hi;
            }
            const uint32_t n2 = dv == 2 ? hi : kNone;
            if (dv == 1) {
                const uint32_t du = s.degs()[n1];
                if (du > 1 || n1 < v) {
                    atomicOr(&s.marks()[n1 >> 5], 1u << (n1 & 31u));
                    marked = true;
                }
            } else if (n2 != kNone) {
                const uint32_t d1 = s.degs()[n1], d2 = s.degs()[n2];
                const bool keep = d1 == 1 || d2 == 1 || (d1 == 2 && n1 < v) || (d2 == 2 && n2 < v);
                if (!keep && ((s.adj[n2 * Rows<NW>::kStride + (n1 >> 5)] >> (n1 & 31u)) & 1u)) {
                    atomicOr(&s.marks()[n1 >> 5], 1u << (n1 & 31u));
                    atomicOr(&s.marks()[n2 >> 5], 1u << (n2 & 31u));
                    marked = true;
                }
            }
        }
    }
    s.stat.passes += 1;
    if (__any_sync(0xffffffffu, marked)) {
        __syncwarp();
        return true;
    }
    uint32_t acc = 0, mx = 0;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const uint32_t d = s.D[j];
        acc += (d & 0x00FF00FFu) + ((d >> 8) & 0x00FF00FFu);
        mx = max(mx, max(max(d & 0xFFu, (d >> 8) & 0xFFu), max((d >> 16) & 0xFFu, d >> 24)));
    }
    o.sum = __reduce_add_sync(0xffffffffu, (acc & 0xFFFFu) + (acc >> 16));
    o.maxd = __reduce_max_sync(0xffffffffu, mx);
    uint32_t first = kNone;
    if (o.maxd > 0) {
#pragma unroll
        for (int j = J - 1; j >= 0; --j) {
            const uint32_t e = bytes_zero(s.D[j] ^ (o.maxd * 0x01010101u));
            if (e) first = 4u * (32u * j + lane) + ((__ffs(e) >> 3) - 1);
        }
    }
    o.amax = __reduce_min_sync(0xffffffffu, first);
    return false;
}

// dense_pass on 16-bit degrees (Half): the same rules and results.
template <int NW>
__device__ __forceinline__ bool dense_pass_half(DSU<NW> &s, uint32_t del, uint32_t bound, ScanOut &o)
{
    constexpr int J = Rows<NW>::kJ;
    const unsigned lane = lane_id();
    const uint32_t sh = 2u * (lane & 15u);  // this lane's 2 bits in words of L, marks and tri
    const int tt = (int)bound - (int)del;  // the high-degree rule takes deg >= tt
    const uint32_t tl = (uint32_t)(tt > 0 ? min(tt, 0x7FFF) : 0) * 0x00010001u;
    const uint32_t *tri = s.adj + Rows<NW>::kTri;
    bool marked = false;
    uint32_t cn[J], ctot = 0;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const uint32_t d = s.D[j];
        const uint32_t q = 32u * j + lane;  // vertices 2q, 2q + 1
        const uint32_t nz = ~halves_zero(d) & 0x80008000u;
        // degrees are below 2^15, so 0x8000 + d - tt keeps its top bit iff d >= tt
        const uint32_t ge = tt <= 1 ? nz : (tt >= 0x7FFF ? 0u : ((d | 0x80008000u) - tl) & 0x80008000u);
        const uint32_t tn = (tri[q >> 4] >> sh) & 0x3u;
        const uint32_t d12 = halves_zero(d ^ 0x00010001u) | (halves_zero(d ^ 0x00020002u) & (spread2(tn) << 15));
        const uint32_t hn = gather2(ge);
        if (hn) {
            atomicOr(&s.marks()[q >> 4], hn << sh);
            marked = true;
        }
        cn[j] = gather2(d12 & ~ge);
        ctot += __popc(cn[j]);
    }
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t pre = 0, total = 0;
    if (__any_sync(0xffffffffu, ctot != 0u)) {
#pragma unroll
        for (int b = 0; b < Rows<NW>::kCandBits; ++b) {
            const uint32_t bal = __ballot_sync(0xffffffffu, (ctot >> b) & 1u);
            pre += __popc(bal & lt) << b;
            total += __popc(bal) << b;
        }
    }
    if (total) {
        uint32_t *d32 = reinterpret_cast<uint32_t *>(s.degs16());
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const uint32_t q = 32u * j + lane;
            if (q < 16u * s.nw) d32[q] = s.D[j];
            uint32_t m = cn[j];
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                s.cand()[pre++] = (uint16_t)(2u * q + b);
            }
        }
        uint32_t L[NW];
        load_L(s, L);
        __syncwarp();
        for (uint32_t i = lane; i < total; i += 32) {  // degree-one / degree-two triangle rules
            const uint32_t v = s.cand()[i];
            const uint32_t dv = s.degs16()[v];
            uint32_t r[NW];
            load_row_at<NW>(s.adj, v, r);
            uint32_t n1 = kNone, hi = kNone;  // lowest and highest live neighbour
#pragma unroll
            for (int w = NW - 1; w >= 0; --w) {
                const uint32_t x = r[w] & L[w];
                n1 = x ? 32u * w + (__ffs(x) - 1) : n1;
            }
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const uint32_t x = r[w] & L[w];
                hi = x ? 32u * w + (31u - __clz(x)) : hi;
            }
            const uint32_t n2 = dv == 2 ? hi : kNone;
            if (dv == 1) {
                const uint32_t du = s.degs16()[n1];
                if (du > 1 || n1 < v) {
                    atomicOr(&s.marks()[n1 >> 5], 1u << (n1 & 31u));
                    marked = true;
                }
            } else if (n2 != kNone) {
                const uint32_t d1 = s.degs16()[n1], d2 = s.degs16()[n2];
                const bool keep = d1 == 1 || d2 == 1 || (d1 == 2 && n1 < v) || (d2 == 2 && n2 < v);
                if (!keep && ((s.adj[Rows<NW>::at(n2, n1 >> 5)] >> (n1 & 31u)) & 1u)) {
                    atomicOr(&s.marks()[n1 >> 5], 1u << (n1 & 31u));
                    atomicOr(&s.marks()[n2 >> 5], 1u << (n2 & 31u));
                    marked = true;
                }
            }
        }
    }
    s.stat.passes += 1;
    if (__any_sync(0xffffffffu, marked)) {
        __syncwarp();
        return true;
    }
    uint32_t acc = 0, mx = 0;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const uint32_t d = s.D[j];
        acc += (d & 0xFFFFu) + (d >> 16);
        mx = max(mx, max(d & 0xFFFFu, d >> 16));
    }
    o.sum = __reduce_add_sync(0xffffffffu, acc);
    o.maxd = __reduce_max_sync(0xffffffffu, mx);
    uint32_t first = kNone;
    if (o.maxd > 0) {
#pragma unroll
        for (int j = J - 1; j >= 0; --j) {
            const uint32_t e = halves_zero(s.D[j] ^ (o.maxd * 0x00010001u));
            if (e) first = 2u * (32u * j + lane) + ((__ffs(e) >> 4) - 1);
        }
    }
    o.amax = __reduce_min_sync(0xffffffffu, first);
    return false;
}

template <int NW>
__device__ __forceinline__ bool dense_pass(DSU<NW> &s, uint32_t del, uint32_t bound, ScanOut &o)
{
    if constexpr (Rows<NW>::kHalf) return dense_pass_half(s, del, bound, o);
    else return dense_pass_byte(s, del, bound, o);
}

// A node's settling: the pending set in s.marks() leaves L and the degrees are
// brought up to date (subtracted, or recounted after a backtrack or a new
// record), then reduction passes run to a fixpoint, each pass's marks taking the
// same path.  One copy of the push / update code serves every caller.
template <int NW>
__device__ __forceinline__ void dense_settle(DSU<NW> &s, uint32_t bound, ScanOut &o)
{
    const unsigned lane = lane_id();
    uint32_t how = s.pending;
    s.pending = 0;
#pragma unroll 1
    for (int pass = 0; pass < 4 * 32 * NW; ++pass) {
        if (how) {
            const long long t0 = (kPhaseTimers && s.timed) ? clock64() : 0;
            dense_push(s);
            if (how == kPendRecount) dense_degrees(s);
            else dense_apply(s);
            __syncwarp();
            if (lane < NW) s.marks()[lane] = 0;
            __syncwarp();
            if (kPhaseTimers && s.timed) s.cyc.apply += (unsigned long long)(clock64() - t0);
        }
        if (!dense_pass(s, s.base_del + s.top, bound, o)) break;
        how = kPendApply;
    }
}

// ---- the overloads the shared work-sharing code (vc_search.cuh) calls
template <class G, int NW>
__device__ __forceinline__ void bind_graph(DSU<NW> &s, const Params &P, uint32_t inst)
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
    s.fr_bot = s.fr_top = 0;
    s.local_nodes = 0;
}

template <class G, int NW>
__device__ __forceinline__ void load_root(DSU<NW> &s)
{
    const unsigned w = lane_id();
    if (w < NW) {
        const uint32_t lo = 32u * w;
        s.lsm()[w] = lo + 32u <= s.n ? 0xffffffffu : (lo < s.n ? (1u << (s.n - lo)) - 1u : 0u);
        s.marks()[w] = 0;
    }
    s.top = 0;
    s.base_del = 0;
    __syncwarp();
    s.pending = kPendRecount;  // the node's settling counts the degrees
}

// From a received live bitmap in s.bits().
template <class G, int NW>
__device__ __forceinline__ void rebuild(DSU<NW> &s)
{
    const unsigned w = lane_id();
    const uint32_t x = w < s.nw ? s.bits()[w] : 0u;
    if (w < NW) {
        s.lsm()[w] = x;
        s.marks()[w] = 0;
    }
    const uint32_t live = __reduce_add_sync(0xffffffffu, __popc(x));
    s.top = 0;
    s.base_del = s.n - live;
    __syncwarp();
    s.pending = kPendRecount;  // the node's settling counts the degrees
}

// The bottom frame's pending child as a live bitmap in s.bits(): L at that frame
// (L now plus the trail above the frame) minus N(v).
template <class G, int NW>
__device__ __forceinline__ void donation_bits(DSU<NW> &s)
{
    const unsigned lane = lane_id();
    const uint32_t f = s.frames()[s.fr_bot];
    const uint32_t pos = f >> 16, v = f & 0xffffu;
    if (lane < NW) s.bits()[lane] = s.lsm()[lane];
    __syncwarp();
    for (uint32_t i = pos + lane; i < s.top; i += 32) {
        uint32_t u = s.trail()[i];
        atomicOr(&s.bits()[u >> 5], 1u << (u & 31u));
    }
    __syncwarp();
    if (lane < NW) s.bits()[lane] &= ~s.adj[Rows<NW>::at(v, lane)];
    __syncwarp();
}

template <class G, int NW>
__device__ __forceinline__ void cover_bits(DSU<NW> &s, uint32_t *dst)
{
    const unsigned lane = lane_id();
    if (lane < s.nw) {
        const uint32_t lo = 32u * lane;
        const uint32_t valid = lo + 32u <= s.n ? 0xffffffffu : (1u << (s.n - lo)) - 1u;
        dst[lane] = ~s.lsm()[lane] & valid;
    }
}

// Stage graph `inst`'s adjacency into the CTA's bitmaps (one warp; the CTA has
// no other active warp when this runs).
template <int NW>
__device__ __forceinline__ void stage_graph(uint32_t *adj, const Params &P, uint32_t inst)
{
    const unsigned lane = lane_id();
    const InstDesc d = load_desc(&P.inst[inst]);
    const uint32_t *rp = P.row_ptr + d.row_off, *cl = P.col + d.col_off;
    for (uint32_t i = lane; i < Rows<NW>::kTri + (uint32_t)NW; i += 32) adj[i] = 0;
    __syncwarp();
    // Entries that break the CSR layout (a row past row_ptr[n], an id out of
    // range, a self loop) are skipped, so no read or write leaves its array;
    // device-resident input is checked by k_check_csr before the search, which
    // drops a graph it flags.
    const uint32_t m2 = d.m2 != kNone ? min(__ldcg(&rp[d.n]), d.m2) : __ldcg(&rp[d.n]);
    for (uint32_t v = lane; v < d.n; v += 32) {  // row v belongs to lane v % 32
        const uint32_t e1 = min(__ldcg(&rp[v + 1]), m2);
        for (uint32_t e = __ldcg(&rp[v]); e < e1; ++e) {
            const uint32_t u = __ldcg(&cl[e]);
            if (u >= d.n || u == v) continue;
            adj[Rows<NW>::at(v, u >> 5)] |= 1u << (u & 31u);
        }
    }
    __syncwarp();
    // tri: v has a neighbour u with a common neighbour.  Only such a vertex can
    // ever meet the triangle rule (its two live neighbours adjacent), so the
    // passes look at degree-2 vertices in tri only.
    for (uint32_t v = lane; v < d.n; v += 32) {
        uint32_t r[NW];
        load_row_at<NW>(adj, v, r);
        bool t = false;
#pragma unroll 1
        for (uint32_t w = 0; w < (uint32_t)NW && !t; ++w) {
            uint32_t x = adj[Rows<NW>::at(v, w)];
            while (x && !t) {
                const uint32_t u = 32u * w + (__ffs(x) - 1);
                x &= x - 1;
                uint32_t c = 0;
#pragma unroll
                for (int k = 0; k < NW; ++k) c |= adj[Rows<NW>::at(u, k)] & r[k];
                t = c != 0u;
            }
        }
        if (t) atomicOr(&adj[Rows<NW>::kTri + (v >> 5)], 1u << (v & 31u));
    }
    __threadfence_block();
    __syncwarp();
}

// Acquire work for a dense search unit.  Local records always belong to the
// CTA's staged graph.  Only when the whole CTA is idle may the poller switch
// graphs: first to the next root from the cursor, then to records of any graph
// from the global ring.  Returns false when the launch is over.
template <int NW>
__device__ bool acquire_cta(DSU<NW> &s, const Params &P, CtaPool &cp, uint32_t *adj)
{
    using G = WarpG;
    using S = DSU<NW>;
    const unsigned lane = lane_id();
    if (lane == 0) {
        __threadfence_block();
        atomicAdd(&cp.hdr[kCpIdle], 1u);
    }
    bool poller = false;
    uint32_t nap = 64;
    for (;;) {
        s.stat.polls += 1;
        // 0 wait, 1 local slot, 2 global record, 3 exit, 4 new root
        uint32_t res = 0, slot = 0;
        unsigned long long qpos = 0;
        if (lane == 0) {
            if (vld(&cp.hdr[kCpExit])) {
                res = 3;
            } else if (vld(&cp.hdr[kCpCount]) > 0) {
                if (poller) { atomicExch(&cp.hdr[kCpPoller], 0u); poller = false; }
                atomicSub(&cp.hdr[kCpIdle], 1u);
                __threadfence_block();
                for (uint32_t i = 0; i < cp.lp; ++i)
                    if (atomicCAS(&cp.state[i], 2u, 3u) == 2u) { slot = i; res = 1; break; }
                if (res == 0) {
                    __threadfence_block();
                    atomicAdd(&cp.hdr[kCpIdle], 1u);
                }
            } else if (poller || atomicCAS(&cp.hdr[kCpPoller], 0u, 1u) == 0u) {
                poller = true;
                const uint32_t cnt = vld(&cp.hdr[kCpCount]);
                __threadfence_block();
                const bool cta_idle = cnt == 0 && vld(&cp.hdr[kCpIdle]) == cp.su;
                if (ld_relaxed_u64(&P.ctl[kAbort]) || ld_relaxed_u64(&P.ctl[kFinish])) {
                    atomicExch(&cp.hdr[kCpExit], 1u);
                    res = 3;
                } else if (cta_idle && !vld(&cp.hdr[kCpCursorClosed])) {
                    uint32_t i = kNone;
                    if (claim_root(P, i)) {
                        if (vld(&cp.hdr[kCpRegistered])) {
                            atomicAdd(&P.ctl[kState], 0xffffffffffffffffull);  // idle CTAs-1
                            cp.hdr[kCpRegistered] = 0u;
                        }
                        atomicSub(&cp.hdr[kCpIdle], 1u);
                        slot = i;
                        res = 4;
                    } else if (!P.server) {
                        cp.hdr[kCpCursorClosed] = 1u;
                    }
                }
                // one graph in the launch (a plain solve): every record is for the
                // graph this CTA already staged, so idle warps of a busy CTA may
                // take records from the ring too
                const bool single = P.count == 1 && !P.server;
                if (res == 0 && (P.server || single || vld(&cp.hdr[kCpCursorClosed]))) {
                    unsigned long long stw = ld_relaxed_u64(&P.ctl[kState]);
                    if (!vld(&cp.hdr[kCpRegistered]) && cta_idle) {
                        stw = atomicAdd(&P.ctl[kState], 1ull) + 1ull;
                        cp.hdr[kCpRegistered] = 1u;
                    }
                    const bool reg = vld(&cp.hdr[kCpRegistered]) != 0;
                    const bool staged = vld(&cp.hdr[kCpStaged]) != kNone;
                    // a registered CTA is fully idle, so the poller may switch graphs
                    if ((reg || (single && staged)) && (stw >> 32) > 0 && ring_claim_deq(P, qpos)) {
                        if (reg) {
                            atomicAdd(&P.ctl[kState], 0xfffffffeffffffffull);  // pending-1, idle CTAs-1
                            cp.hdr[kCpRegistered] = 0u;
                        } else {
                            atomicAdd(&P.ctl[kState], 0xffffffff00000000ull);  // pending-1
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
        if (res == 4) {  // a new graph root for the whole CTA
            slot = G::bcast(slot);
            const uint32_t key = __ldcg(&P.inst[slot].key);
            if (vld(&cp.hdr[kCpStaged]) != key) {
                stage_graph<NW>(adj, P, slot);
                if (lane == 0) cp.hdr[kCpStaged] = key;
            }
            bind_graph<G>(s, P, slot);
            load_root<G>(s);
            s.stat.roots += 1;
            return true;
        }
        if (res == 1) {
            slot = G::bcast(slot);
            const uint32_t *d = cp.data + (size_t)slot * P.stride;
            __threadfence_block();
            const uint32_t inst = vld(&d[0]);
            bind_graph<G>(s, P, inst);
            for (uint32_t w = lane; w < s.nw; w += 32) s.bits()[w] = vld(&d[4 + w]);
            __syncwarp();
            if (lane == 0) {
                atomicSub(&cp.hdr[kCpCount], 1u);
                __threadfence_block();
                atomicExch(&cp.state[slot], 0u);
            }
            if (start_record<G, S>(s, P)) return true;
            if (lane == 0) { __threadfence_block(); atomicAdd(&cp.hdr[kCpIdle], 1u); }
            continue;
        }
        if (res == 2) {
            qpos = G::bcast64(qpos);
            const uint32_t slot_i = (uint32_t)(qpos & P.q_mask);
            const uint32_t *g = P.pool_data + (size_t)slot_i * P.stride;
            __syncwarp();
            __threadfence();
            const uint32_t inst = __ldcg(&g[0]);
            const uint32_t key = __ldcg(&P.inst[inst].key);
            if (vld(&cp.hdr[kCpStaged]) != key) {
                stage_graph<NW>(adj, P, inst);
                if (lane == 0) cp.hdr[kCpStaged] = key;
            }
            bind_graph<G>(s, P, inst);
            for (uint32_t w = lane; w < s.nw; w += 32) s.bits()[w] = __ldcg(&g[4 + w]);
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                st_release_u64(&P.pool_seq[slot_i], qpos + P.q_mask + 1);
            }
            if (start_record<G, S>(s, P)) return true;
            if (lane == 0) { __threadfence_block(); atomicAdd(&cp.hdr[kCpIdle], 1u); }
            continue;
        }
        if (lane == 0) __nanosleep(nap);
        nap = nap < (poller ? 4096u : kIdleNapMax) ? nap * 2 : (poller ? 4096u : kIdleNapMax);
        __syncwarp();
    }
}

template <int NW>
__device__ void su_main_dense(const Params &P, uint8_t *ws, uint32_t *adj, CtaPool &cp)
{
    using G = WarpG;
    using S = DSU<NW>;
    S s;
    dsu_bind(s, ws, adj);
    s.inst = kNone;
    s.fr_bot = s.fr_top = 0;
    s.pending = 0;
    s.local_nodes = 0;
    s.c_best = 0;
    s.top = 0;
    s.deadline = globaltimer() + P.time_limit_ns;
    if (lane_id() == 0) atomicCAS(&P.ctl[kT0], 0ull, globaltimer());
    s.stat = SUStat{0, 0, 0, 0, 0, 0, 0, 0, 0};
    s.cyc = PhaseCycles{0, 0, 0, 0};
    s.timed = P.stats != nullptr;
    unsigned long long nodes_total = 0;
    long long t_mark = clock64();
    bool have = false;
    uint32_t ticks = 0, c_flags = 0;
    unsigned long long c_state = 0;
    const unsigned lane = lane_id();

    for (;;) {
        if (!have) {
            if (s.inst != kNone && s.fr_top > s.fr_bot) {
                const long long t_pop = (kPhaseTimers && s.timed) ? clock64() : 0;
                s.fr_top -= 1;
                const uint32_t f = s.frames()[s.fr_top];
                const uint32_t v = f & 0xffffu;
                dense_restore(s, f >> 16);
                if (lane < NW) s.marks()[lane] = s.adj[Rows<NW>::at(v, lane)] & s.lsm()[lane];
                __syncwarp();
                s.pending = kPendRecount;  // take N(v), then recount
                have = true;
                if (kPhaseTimers && s.timed) s.cyc.pop += (unsigned long long)(clock64() - t_pop);
            } else {
                if (s.inst != kNone) finish_stint<G, S>(s, P);
                long long t0 = clock64();
                s.stat.busy += (unsigned long long)(t0 - t_mark);
                bool got = acquire_cta<NW>(s, P, cp, adj);
                t_mark = clock64();
                s.stat.idle += (unsigned long long)(t_mark - t0);
                if (!got) break;
                have = true;  // load_root / rebuild counted the degrees
                ticks = 0;
            }
        }
        InstState &st = P.st[s.inst];
        if ((ticks & 7u) == 0u) {
            uint32_t b = 0, f = 0;
            unsigned long long w = 0;
            if (lane == 0) {
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
        if (c_flags & (kFound | kBudget | kError | kBadGraph)) {
            if (lane == 0 && !(c_flags & (kFound | kBudget | kBadGraph))) atomicOr(&st.flags, kCut);
            s.fr_bot = s.fr_top = 0;
            s.pending = 0;
            if (lane < NW) s.marks()[lane] = 0;
            __syncwarp();
            have = false;
            continue;
        }
        s.local_nodes += 1;
        nodes_total += 1;
        if ((s.local_nodes & 127ull) == 0ull) {
            if (lane == 0) {
                unsigned long long tot = atomicAdd(&st.nodes, s.local_nodes) + s.local_nodes;
                if (s.node_limit && tot >= s.node_limit) atomicOr(&st.flags, kBudget);
            }
            s.local_nodes = 0;
        }
        const uint32_t best = s.c_best;
        const uint32_t bound = s.mode == kModeMVC ? best : s.k + 1;
        ScanOut o = {0u, 0u, kNone};
        const long long t_scan = (kPhaseTimers && s.timed) ? clock64() : 0;
        const unsigned long long apply0 = s.cyc.apply;
        dense_settle(s, bound, o);
        if (kPhaseTimers && s.timed) s.cyc.scan += (unsigned long long)(clock64() - t_scan) - (s.cyc.apply - apply0);
        const uint32_t del = s.base_del + s.top;
        const uint64_t edges = o.sum / 2;
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
            report_leaf<G, S>(s, P, del);
            have = false;
            continue;
        }
        const long long t_br = (kPhaseTimers && s.timed) ? clock64() : 0;
        const uint32_t v = o.amax;
        if (lane == 0) s.frames()[s.fr_top] = (s.top << 16) | v;
        s.fr_top += 1;
        __syncwarp();
        uint32_t want = 0;
        if (lane == 0) {
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
        if (want == 1) donate_local<G, S>(s, P, cp);
        else if (want == 2 && donate_global<G, S>(s, P)) c_state += 1ull << 32;
        if (lane == 0) s.marks()[v >> 5] = 1u << (v & 31u);  // marks are clear after a settled node
        __syncwarp();
        s.pending = kPendApply;  // the child takes v
        if (kPhaseTimers && s.timed) s.cyc.branch += (unsigned long long)(clock64() - t_br);
    }
    if (P.stats && lane == 0) {
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
        o[kStCycScan] = s.cyc.scan;
        o[kStCycApply] = s.cyc.apply;
        o[kStCycPop] = s.cyc.pop;
        o[kStCycBranch] = s.cyc.branch;
        o[kStCycOther] = s.stat.busy - s.cyc.scan - s.cyc.apply - s.cyc.pop - s.cyc.branch;
    }
}

}  // namespace vcg
