// vc_types.h -- plain data shared by the search kernels and the host code.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define VC_HD __host__ __device__
#else
#define VC_HD
#endif

namespace vcg {


constexpr int32_t kDead = -(1 << 30);
constexpr int32_t kRestoring = -1;
constexpr uint32_t kNone = 0xffffffffu;

// InstState.flags
constexpr uint32_t kFound = 1u;   // PVC: a cover of size <= k was found
constexpr uint32_t kBudget = 2u;  // node limit reached
constexpr uint32_t kDone = 4u;    // every token of the graph returned
constexpr uint32_t kError = 8u;   // a bounded wait gave up
constexpr uint32_t kCut = 16u;    // work was dropped at the launch's time limit
constexpr uint32_t kBadGraph = 32u;  // device-resident CSR failed the kernel's staging checks

// control words, each on its own 128-byte line (index in u64 units)
enum : uint32_t {
    kHead = 0, kTail = 16, kState = 32, kCursor = 48, kAbort = 64, kFinish = 80, kT0 = 96,
    kSubTail = 112,   // server: submissions published by the host
    kShutdown = 128,  // server: the host asks the kernel to exit once idle
    kLastWork = 144,  // server: %globaltimer of the last claimed submission
    kStarted = 160,   // server: CTAs of the launch that have started
    kCtlWords = 176
};

enum : uint32_t { kModeMVC = 0, kModePVC = 1 };

// Per-SU counters (the role of the reference's Counters.cuh phase timers and
// NODES_PER_SM histogram), written once when an SU exits, only when enabled.
enum : uint32_t {
    kStNodes = 0, kStPasses, kStDonations, kStDonateFail, kStReceives, kStRoots, kStBusyCycles, kStIdleCycles,
    kStPolls, kStRestored, kStSmid,
    kStCycScan, kStCycApply, kStCycPop, kStCycBranch, kStCycOther,  // dense search phases (clock64)
    kStatWords = 16
};

struct InstDesc {
    uint32_t n, nw;            // vertices, 32-bit words of an n-bit set
    uint64_t row_off, col_off; // offsets of this graph's row_ptr / col in the arena
    uint32_t mode, k;          // kModeMVC / kModePVC, PVC parameter
    uint32_t init_best;        // MVC: look for covers smaller than this
    uint32_t cover_off;        // word offset of this graph's cover bitmap
    uint64_t node_limit;       // 0 = none
    uint32_t key;              // unique per graph (batch index / server ticket)
    uint32_t m2;               // row_ptr[n] (2m) as the host knows it, kNone = unknown
};

struct InstState {
    uint32_t best;        // MVC incumbent (init_best until a cover is found)
    uint32_t act;         // outstanding work tokens (SU stints + queued records)
    uint32_t flags;
    uint32_t lock;        // guards the cover bitmap
    uint32_t cover_size;  // size of the cover in the bitmap, kNone = none
    uint32_t pad;
    unsigned long long nodes;
    unsigned long long t_done;  // %globaltimer when the last token returned
};

struct Params {
    const uint32_t *row_ptr;
    const uint32_t *col;
    const InstDesc *inst;
    InstState *st;
    uint32_t *covers;
    uint32_t count;
    uint32_t num_su;
    unsigned long long *ctl;
    unsigned long long *pool_seq;
    uint32_t *pool_data;
    uint32_t q_mask;
    uint32_t stride;      // u32 words per ring slot (4 header words + nw)
    uint32_t np;          // per-SU vertex capacity (multiple of 32)
    uint32_t su_bytes;    // per-SU workspace bytes
    uint32_t cta_slots;   // CTA pool slots (0 when a CTA holds one SU)
    uint8_t *gws;         // global workspace (CTA SUs on large graphs), else null
    unsigned long long *stats;    // per-SU counters (kStatWords each), null = off
    unsigned long long time_limit_ns;
    int32_t ring_bias;  // give work to the global ring while idle CTAs minus queued records exceed this (< 0: keep a surplus queued)
    uint32_t ring_first;  // when both idle sibling warps and idle CTAs wait: 0 local pool first, 1 ring first, 2 alternate
    // server mode (persistent kernel fed by the host)
    uint32_t server;
    uint32_t subq_mask;
    const uint32_t *subq;         // slot ids in submission order
    uint32_t *hres;               // host-mapped result records, hres_words u32 each
    uint32_t hres_words;
    unsigned long long idle_ns;   // exit after this long without any work
};

// Result record written by the device into host-mapped memory (server mode).
struct HostResult {
    unsigned long long done;      // ticket of the finished request (0 = none yet)
    uint32_t best, flags, cover_size, pad;
    unsigned long long nodes, t_done;
    // followed by the cover bitmap words
};

// Workspace layout (bytes), np = vertex capacity, nw = np/32:
//   deg[np] int32 | trail[np] u32 | fpos[np] u32 | fv[np] u32 | marks[nw] | bits[nw] | ctr[4] | cand[np] u32 |
//   aux[np] (np > 65536 only)
VC_HD inline uint32_t su_workspace_bytes(uint32_t np)
{
    uint32_t nw = np / 32;
    uint32_t b = 20u * np + 8u * nw + 16u;
    if (np > 65536u) b += 4u * np;
    return (b + 15u) & ~15u;
}

// Dense-bitset search unit (nw = 2, 4 or 8 words: graphs of at most 255
// vertices; nw = 20: up to 640 vertices whose degrees are all at most 254;
// nw = 16 and 32: up to 512 and 1024 vertices of any degree, with 16-bit
// degrees): per CTA adj[32*nw][dense_row_words(nw)] u32, then tri[nw] u32 (the
// vertices that lie on a triangle of the staged graph); per warp
//   frames[32*nw] u32 | marks[nw] | bits[nw] | lsm[nw] | trail[32*nw] u16 |
//   cand[32*nw] u16 | degs[32*nw] u8 (u16 with 16-bit degrees)
// Row stride in words: 8- and 16-word rows are padded to 12 and 20 so that the
// 16-byte row loads of eight consecutive lanes fall in distinct shared-memory
// banks (20-word rows already do); 32-word rows are not padded (a 1024-vertex
// adjacency is 128 KB) but their eight 16-byte chunks are stored XOR-swizzled
// by the row's low three bits, which spreads the same loads as well.
VC_HD inline bool dense_half(uint32_t nw) { return nw == 16 || nw == 32; }
VC_HD inline uint32_t dense_row_words(uint32_t nw) { return nw == 8 ? 12u : (nw == 16 ? 20u : nw); }
VC_HD inline uint32_t dense_adj_bytes(uint32_t nw) { return 4u * 32u * nw * dense_row_words(nw) + 128u; }
VC_HD inline uint32_t dense_workspace_bytes(uint32_t nw)
{
    uint32_t b = 4u * (32u * nw + 3u * nw) + 2u * 32u * nw + 2u * 32u * nw + (dense_half(nw) ? 2u : 1u) * 32u * nw;
    return (b + 15u) & ~15u;
}

}  // namespace vcg
