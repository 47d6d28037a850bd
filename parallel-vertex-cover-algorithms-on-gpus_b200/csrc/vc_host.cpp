// vc_host.cpp -- host-side graph checks.
//
// The reference rejects duplicate edges and self-loops with an O(V^2)
// adjacency matrix (src/auxFunctions.cpp:308-354, asserted at :358).  The same
// conditions are checked here in O(m log d) on the CSR itself, plus the layout
// the kernels rely on: monotone offsets, ids < n, sorted rows, symmetry.
#include <algorithm>
#include <cstdint>

#include "vc_host.h"

namespace vch {

static bool row_has(const uint32_t *rp, const uint32_t *col, uint32_t row, uint32_t x)
{
    const uint32_t *b = col + rp[row], *e = col + rp[row + 1];
    return std::binary_search(b, e, x);
}

vc_status validate_csr(const vc_csr *g)
{
    if (!g->row_ptr) return VC_ERR_INVALID;
    const uint32_t n = g->n;
    const uint32_t *rp = g->row_ptr, *col = g->col;
    if (rp[0] != 0) return VC_ERR_INVALID;
    if ((uint64_t)rp[n] != 2ull * g->m) return VC_ERR_INVALID;
    if (g->m && !col) return VC_ERR_INVALID;
    for (uint32_t v = 0; v < n; ++v) {
        if (rp[v + 1] < rp[v]) return VC_ERR_INVALID;
        if (g->degree && (uint32_t)g->degree[v] != rp[v + 1] - rp[v]) return VC_ERR_INVALID;
        for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) {
            uint32_t u = col[e];
            if (u >= n || u == v) return VC_ERR_INVALID;                    // id range, self-loop
            if (e > rp[v] && col[e - 1] >= u) return VC_ERR_INVALID;       // sorted, no duplicate
        }
    }
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t e = rp[v]; e < rp[v + 1]; ++e)
            if (!row_has(rp, col, col[e], v)) return VC_ERR_INVALID;        // symmetric
    return VC_OK;
}

}  // namespace vch
