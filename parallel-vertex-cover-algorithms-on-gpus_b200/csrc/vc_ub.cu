// vc_ub.cu -- the reference's two upper-bound heuristics on the GPU
// (vc_remove_max_ub / vc_remove_edge_ub in include/vcgpu.h).
//
// RemoveMaxApproximateMVC (src/auxFunctions.cpp:211-256) and
// RemoveEdgeApproximateMVC (:258-306) are greedy and order dependent: their
// results depend on the exact sequence of deletions, on the order in which the
// leaf and triangle rules visit the vertices (:44-127), and on the row order that
// CSRGraph::deleteVertex (CSRGraphRep.cpp:44-62) leaves behind, since it compacts
// each neighbour's row by copying the last live entry over the deleted one and
// the triangle test binary-searches those unsorted rows.  This kernel keeps that
// exact sequence and parallelises each step instead: one CTA per graph; a
// deletion updates all neighbours' rows at once (the rows are disjoint); the
// rules find "the next vertex in index order" with block-wide searches over
// bitmaps instead of full sweeps.
//
// Incremental bookkeeping that leaves the sequence unchanged:
//  * deg1: the vertices of degree 1 (bitmap + count).  A leaf-rule pass visits
//    them in index order from where the pass stands, exactly the vertices the
//    reference's sweep would act on; with none left no pass can act.
//  * dirty: every vertex whose triangle test may have changed since it last
//    failed.  The test of a degree-2 vertex i reads deg(i), i's live prefix,
//    the degrees of its two live neighbours and the second neighbour's row;
//    deleting x changes those only for i within two hops of x, so a deletion
//    marks x's live neighbours and theirs.  A full pass that finds no triangle
//    clears the bitmap; the next pass only looks at marked vertices, and the
//    first firing vertex in index order is the one the reference's restart-
//    from-zero sweep would reach first.
// The reference's binary search (auxFunctions.cpp:25-42) steps an unsigned
// index below zero (and reads out of bounds) in one corner case; there this
// search stops with "not found".
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <vector>

#include "vc_host.h"
#include "vcgpu.h"

using namespace vcg;

namespace vch {
extern std::atomic<uint64_t> g_launches;
}
using namespace vch;

namespace {

constexpr unsigned kUbThreads = 1024;
constexpr uint32_t kInf = 0xffffffffu;

struct UbParams {
    const uint32_t *n;         // [count]
    const uint64_t *row_off;   // [count] into row_ptr / deg
    const uint64_t *col_off;   // [count] into col / dst
    const uint64_t *bits_off;  // [count] into bits: deg1 words, then dirty words
    const uint32_t *row_ptr;
    const uint32_t *col;
    uint32_t *dst;     // working copy of col, compacted by deletions
    int32_t *deg;      // working degrees, -1 = in the cover
    uint32_t *bits;
    uint32_t *ub;      // [count] results
    uint32_t mode;     // 0 RemoveMax, 1 RemoveEdge
    uint32_t r;        // RemoveEdge: the value of rand() the reference's draws used
};

constexpr uint32_t kHubDeg = 128;  // rows longer than this are updated by the whole block
constexpr uint32_t kHubList = 2048;

struct UbShared {
    uint32_t found;      // block search result
    uint32_t cnt1;       // vertices of degree 1
    uint32_t dirty_any;  // dirty bitmap not empty
    uint32_t nhub;       // long rows left for the block in this deletion
    unsigned long long amax;  // argmax key: degree << 32 | ~index
    uint32_t hub[kHubList];
};

// Bookkeeping after w lost one live neighbour (its degree went from dw to dw-1).
__device__ __forceinline__ void ub_lost_one(uint32_t *d1, UbShared &sh, uint32_t w, int dw)
{
    if (dw - 1 == 1) {
        atomicOr(&d1[w >> 5], 1u << (w & 31u));
        atomicAdd(&sh.cnt1, 1u);
    } else if (dw == 1) {
        atomicAnd(&d1[w >> 5], ~(1u << (w & 31u)));
        atomicSub(&sh.cnt1, 1u);
    }
}

// Deletes live vertex x (CSRGraph::deleteVertex): each live neighbour w takes
// x out of its live prefix by moving its last live entry over it.  One thread
// per neighbour; the rows are disjoint.
__device__ void ub_delete(const uint32_t *rp, uint32_t *dst, int32_t *deg, uint32_t *d1, uint32_t *dt, UbShared &sh,
                          uint32_t x)
{
    __syncthreads();  // sh.nhub is 0 here: set at the end of the previous deletion and at the start
    const int dx = deg[x];
    for (int t = (int)threadIdx.x; t < dx; t += (int)blockDim.x) {
        const uint32_t w = dst[rp[x] + (uint32_t)t];
        const int dw = deg[w];
        if ((uint32_t)dw > kHubDeg) {  // a long row: the whole block takes it below
            const uint32_t slot = atomicAdd(&sh.nhub, 1u);
            if (slot < kHubList) {
                sh.hub[slot] = w;
                continue;
            }
        }
        const uint32_t last = rp[w] + (uint32_t)dw;
        for (uint32_t j = rp[w]; j < last; ++j)
            if (dst[j] == x) dst[j] = dst[last - 1];
        const int nd = dw - 1;
        deg[w] = nd;
        ub_lost_one(d1, sh, w, dw);
        atomicOr(&dt[w >> 5], 1u << (w & 31u));
        for (uint32_t k = rp[w]; k < rp[w] + (uint32_t)nd; ++k) {
            const uint32_t y = dst[k];
            atomicOr(&dt[y >> 5], 1u << (y & 31u));
        }
        sh.dirty_any = 1u;
    }
    __syncthreads();
    // Long rows, one at a time: the block finds x in w's live prefix, one
    // thread moves the last live entry over it, the block marks w's neighbours.
    // Each row is changed exactly as the serial loop above would change it.
    const uint32_t nhub = min(sh.nhub, kHubList);
    for (uint32_t h = 0; h < nhub; ++h) {
        const uint32_t w = sh.hub[h];
        const int dw = deg[w];
        const uint32_t b = rp[w], last = b + (uint32_t)dw;
        if (threadIdx.x == 0) sh.found = kInf;
        __syncthreads();
        for (uint32_t j = b + threadIdx.x; j < last; j += blockDim.x)
            if (dst[j] == x) atomicMin(&sh.found, j);
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t j = sh.found;
            if (j != kInf) dst[j] = dst[last - 1];
            deg[w] = dw - 1;
            ub_lost_one(d1, sh, w, dw);
            atomicOr(&dt[w >> 5], 1u << (w & 31u));
            sh.dirty_any = 1u;
        }
        __syncthreads();
        for (uint32_t k = b + threadIdx.x; k < b + (uint32_t)(dw - 1); k += blockDim.x) {
            const uint32_t y = dst[k];
            atomicOr(&dt[y >> 5], 1u << (y & 31u));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (deg[x] == 1) {
            atomicAnd(&d1[x >> 5], ~(1u << (x & 31u)));
            sh.cnt1 -= 1u;
        }
        deg[x] = -1;
        sh.nhub = 0;
    }
    __syncthreads();
}

// The first set bit at index >= p of a bitmap of nw words, or kInf.
__device__ uint32_t ub_next_bit(const uint32_t *bm, uint32_t nw, uint32_t p, UbShared &sh)
{
    for (uint32_t base = p >> 5; base < nw; base += blockDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) sh.found = kInf;
        __syncthreads();
        const uint32_t wi = base + threadIdx.x;
        if (wi < nw) {
            uint32_t x = bm[wi];
            if (wi == (p >> 5)) x &= ~0u << (p & 31u);
            if (x) atomicMin(&sh.found, 32u * wi + (uint32_t)(__ffs(x) - 1));
        }
        __syncthreads();
        const uint32_t f = sh.found;
        if (f != kInf) return f;
    }
    return kInf;
}

// auxBinarySearch over a (compacted, possibly unsorted) row, stopping where
// the reference's unsigned index would go below zero.
__device__ bool ub_search(const uint32_t *arr, long l, long r, uint32_t x)
{
    while (l <= r) {
        const long m = l + (r - l) / 2;
        const uint32_t a = arr[m];
        if (a == x) return true;
        if (a < x) l = m + 1;
        else r = m - 1;
    }
    return false;
}

// The triangle test of vertex i (auxFunctions.cpp:79-121): its two live
// neighbours are the first two entries of its compacted row.
__device__ bool ub_fires(const uint32_t *rp, const uint32_t *dst, const int32_t *deg, uint32_t i, uint32_t *n1,
                         uint32_t *n2)
{
    if (deg[i] != 2) return false;
    const uint32_t a = dst[rp[i]], b = dst[rp[i] + 1];
    const int da = deg[a], db = deg[b];
    if (da == 1 || (da == 2 && a < i)) return false;
    if (db == 1 || (db == 2 && b < i)) return false;
    if (!ub_search(dst, (long)rp[b], (long)rp[b + 1] - 1, a)) return false;
    *n1 = a;
    *n2 = b;
    return true;
}

__global__ void __launch_bounds__(kUbThreads) k_ub(UbParams P)
{
    __shared__ UbShared sh;
    const uint32_t g = blockIdx.x;
    const uint32_t n = P.n[g];
    const uint32_t nw = (n + 31) / 32;
    const uint32_t *rp = P.row_ptr + P.row_off[g];
    const uint32_t *col = P.col + P.col_off[g];
    uint32_t *dst = P.dst + P.col_off[g];
    int32_t *deg = P.deg + P.row_off[g];
    uint32_t *d1 = P.bits + P.bits_off[g];
    uint32_t *dt = d1 + nw;
    const uint32_t m2 = n ? rp[n] : 0u;
    if (threadIdx.x == 0) {
        sh.cnt1 = 0;
        sh.dirty_any = 1;
        sh.nhub = 0;
    }
    for (uint32_t e = threadIdx.x; e < m2; e += blockDim.x) dst[e] = col[e];
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        d1[w] = 0;
        dt[w] = (32u * w + 32u <= n) ? ~0u : ((1u << (n - 32u * w)) - 1u);
    }
    __syncthreads();
    for (uint32_t v = threadIdx.x; v < n; v += blockDim.x) {
        const int d = (int)(rp[v + 1] - rp[v]);
        deg[v] = d;
        if (d == 1) {
            atomicOr(&d1[v >> 5], 1u << (v & 31u));
            atomicAdd(&sh.cnt1, 1u);
        }
    }
    __syncthreads();
    uint32_t minimum = 0;           // uniform across the block
    uint32_t remaining = m2 / 2;    // RemoveEdge's edge count
    uint32_t vertex = 0;            // RemoveEdge's loop index
    for (;;) {
        if (P.mode == 1 && !(vertex < n && remaining > 0)) break;
        // leaf rule to its fixpoint: passes in index order while a pass acts
        {
            uint32_t p = 0;
            bool changed = false;
            for (;;) {
                __syncthreads();
                if (sh.cnt1 == 0) break;  // no pass can act any more
                const uint32_t i = ub_next_bit(d1, nw, p, sh);
                if (i == kInf) {
                    if (!changed) break;
                    p = 0;
                    changed = false;
                    continue;
                }
                changed = true;
                ub_delete(rp, dst, deg, d1, dt, sh, dst[rp[i]]);  // its only live neighbour
                minimum += 1;
                p = i + 1;
            }
        }
        // triangle rule to its fixpoint: the first firing vertex, then restart
        for (;;) {
            __syncthreads();
            if (!sh.dirty_any) break;
            uint32_t fire = kInf;
            for (uint32_t base = 0; base < nw && fire == kInf; base += blockDim.x) {
                __syncthreads();
                if (threadIdx.x == 0) sh.found = kInf;
                __syncthreads();
                const uint32_t wi = base + threadIdx.x;
                if (wi < nw) {
                    uint32_t x = dt[wi];
                    while (x) {
                        const uint32_t i = 32u * wi + (uint32_t)(__ffs(x) - 1);
                        x &= x - 1;
                        uint32_t a, b;
                        if (ub_fires(rp, dst, deg, i, &a, &b)) {
                            atomicMin(&sh.found, i);
                            break;
                        }
                    }
                }
                __syncthreads();
                fire = sh.found;
            }
            if (fire == kInf) {  // a full pass without a triangle: every marked vertex fails
                __syncthreads();
                for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) dt[w] = 0;
                if (threadIdx.x == 0) sh.dirty_any = 0;
                __syncthreads();
                break;
            }
            uint32_t a = 0, b = 0;
            ub_fires(rp, dst, deg, fire, &a, &b);
            ub_delete(rp, dst, deg, d1, dt, sh, a);
            ub_delete(rp, dst, deg, d1, dt, sh, b);
            minimum += 2;
        }
        if (P.mode == 0) {
            // the lowest-index vertex of maximum degree
            __syncthreads();
            if (threadIdx.x == 0) sh.amax = 0;
            __syncthreads();
            unsigned long long best = 0;
            for (uint32_t v = threadIdx.x; v < n; v += blockDim.x) {
                const int d = deg[v];
                if (d > 0) {
                    const unsigned long long key = ((unsigned long long)(uint32_t)d << 32) | (uint32_t)(~v);
                    best = key > best ? key : best;
                }
            }
            if (best) atomicMax(&sh.amax, best);
            __syncthreads();
            const unsigned long long k = sh.amax;
            if (k == 0) break;
            ub_delete(rp, dst, deg, d1, dt, sh, ~(uint32_t)k);
            minimum += 1;
        } else {
            const int dv = deg[vertex];
            if (dv > 0) {
                const uint32_t u = dst[rp[vertex] + P.r % (uint32_t)dv];
                remaining -= (uint32_t)dv;
                remaining -= (uint32_t)deg[u];
                ++remaining;
                ub_delete(rp, dst, deg, d1, dt, sh, vertex);
                ub_delete(rp, dst, deg, d1, dt, sh, u);
                minimum += 2;
            }
            ++vertex;
        }
    }
    if (threadIdx.x == 0) P.ub[g] = minimum;
}

// Device buffers of one call, freed when it returns (after the stream is idle).
struct UbBufs {
    DevBuf n, ro, co, bo, rp, col, dst, deg, bits, ub;
    ~UbBufs()
    {
        for (DevBuf *b : {&n, &ro, &co, &bo, &rp, &col, &dst, &deg, &bits, &ub}) b->release();
    }
};

vc_status ub_run(const vc_csr_arena *a, uint32_t mode, uint32_t r, int32_t device, uint32_t *ub, uint8_t *cover,
                 float *kernel_ms)
{
    if (!a || !ub || (a->count && (!a->n || !a->row_off || !a->col_off || !a->row_ptr))) return VC_ERR_INVALID;
    const uint32_t count = a->count;
    if (count == 0) return VC_OK;
    uint64_t rows = 0, cols = 0, bits = 0;
    std::vector<uint64_t> boff(count);
    for (uint32_t i = 0; i < count; ++i) {
        if (a->n[i] > kMaxVertices) return VC_ERR_TOO_LARGE;
        const uint32_t *rp = a->row_ptr + a->row_off[i];
        rows = std::max<uint64_t>(rows, a->row_off[i] + a->n[i] + 1);
        cols = std::max<uint64_t>(cols, a->col_off[i] + rp[a->n[i]]);
        boff[i] = bits;
        bits += 2ull * ((a->n[i] + 31) / 32);
        vc_csr g;
        g.n = a->n[i];
        g.m = rp[g.n] / 2;
        g.row_ptr = rp;
        g.col = a->col + a->col_off[i];
        g.degree = nullptr;
        vc_status v = validate_csr(&g);
        if (v != VC_OK) return v;
    }
    vc_status err;
    Ctx *c = get_ctx(device, &err);
    if (!c) return err;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t st = c->stream;
    UbBufs B;
    DevBuf &d_n = B.n, &d_ro = B.ro, &d_co = B.co, &d_bo = B.bo, &d_rp = B.rp, &d_col = B.col, &d_dst = B.dst,
           &d_deg = B.deg, &d_bits = B.bits, &d_ub = B.ub;
    if (d_n.ensure(4ull * count) || d_ro.ensure(8ull * count) || d_co.ensure(8ull * count) ||
        d_bo.ensure(8ull * count) || d_rp.ensure(4ull * rows) || d_col.ensure(4ull * std::max<uint64_t>(cols, 1)) ||
        d_dst.ensure(4ull * std::max<uint64_t>(cols, 1)) || d_deg.ensure(4ull * rows) ||
        d_bits.ensure(4ull * std::max<uint64_t>(bits, 1)) || d_ub.ensure(4ull * count))
        return VC_ERR_NOMEM;
    bool ok = cudaMemcpyAsync(d_n.p, a->n, 4ull * count, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(d_ro.p, a->row_off, 8ull * count, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(d_co.p, a->col_off, 8ull * count, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(d_bo.p, boff.data(), 8ull * count, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(d_rp.p, a->row_ptr, 4ull * rows, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              (cols == 0 || cudaMemcpyAsync(d_col.p, a->col, 4ull * cols, cudaMemcpyHostToDevice, st) == cudaSuccess);
    if (!ok) {
        cudaStreamSynchronize(st);
        return VC_ERR_CUDA;
    }
    UbParams P;
    P.n = (const uint32_t *)d_n.p;
    P.row_off = (const uint64_t *)d_ro.p;
    P.col_off = (const uint64_t *)d_co.p;
    P.bits_off = (const uint64_t *)d_bo.p;
    P.row_ptr = (const uint32_t *)d_rp.p;
    P.col = (const uint32_t *)d_col.p;
    P.dst = (uint32_t *)d_dst.p;
    P.deg = (int32_t *)d_deg.p;
    P.bits = (uint32_t *)d_bits.p;
    P.ub = (uint32_t *)d_ub.p;
    P.mode = mode;
    P.r = r;
    cudaEventRecord(c->ev0, st);
    void *args[] = {&P};
    // checked by its own return code: an error the caller left pending is neither reported nor cleared
    bool good = cudaLaunchKernel((const void *)k_ub, dim3(count), dim3(kUbThreads), args, 0, st) == cudaSuccess;
    cudaEventRecord(c->ev1, st);
    g_launches += 1;
    good = good && cudaMemcpyAsync(ub, d_ub.p, 4ull * count, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    std::vector<int32_t> deg;
    if (cover && good) {
        deg.resize(rows);
        good = cudaMemcpyAsync(deg.data(), d_deg.p, 4ull * rows, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    }
    // the buffers are freed on return: the stream must be idle on every path
    if (cudaStreamSynchronize(st) != cudaSuccess || !good) return VC_ERR_CUDA;
    if (kernel_ms) cudaEventElapsedTime(kernel_ms, c->ev0, c->ev1);
    if (cover) {
        uint64_t k = 0;
        for (uint32_t i = 0; i < count; ++i)
            for (uint32_t v = 0; v < a->n[i]; ++v) cover[k++] = deg[a->row_off[i] + v] == -1;
    }
    return VC_OK;
}

}  // namespace

extern "C" vc_status vc_remove_max_ub(const vc_csr_arena *a, int32_t device, uint32_t *ub, uint8_t *cover,
                                     float *kernel_ms)
{
    vch::DeviceGuard dg;
    return ub_run(a, 0u, 0u, device, ub, cover, kernel_ms);
}

extern "C" vc_status vc_remove_edge_ub(const vc_csr_arena *a, uint32_t r, int32_t device, uint32_t *ub,
                                      uint8_t *cover, float *kernel_ms)
{
    vch::DeviceGuard dg;
    return ub_run(a, 1u, r, device, ub, cover, kernel_ms);
}
