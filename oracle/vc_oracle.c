/*
 * vc_oracle.c -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * A plain-C restatement of the reference's sequential branch-and-reduce solver
 * for Minimum Vertex Cover (MVC) and Parameterized Vertex Cover (PVC).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this
 * file's library, and only as the checker: the product (libvcgpu.so and the
 * `output` CLI) never links or calls it.
 *
 * What it restates (reference paths are inside the reference project):
 *   oracle_mvc  -> src/Sequential.cpp:3-104            (Sequential)
 *   oracle_pvc  -> src/SequentialParameterized.cpp:4-110 (SequentialParameterized,
 *                  called as (graph, k+1, k, &kFound), the way the GPU kernels
 *                  bound the high-degree rule: GlobalWorkListParameterized.cuh:127)
 *   rules       -> src/helperFunctions.cpp:27-155
 *                  (deleteVertex :27-47, leafReductionRule :49-75,
 *                   highDegreeReductionRule :77-96, triangleReductionRule :98-155)
 *   greedy UB   -> the "always take the max-degree vertex" descent of
 *                  src/auxFunctions.cpp:211-256 (RemoveMaxApproximateMVC), stated on
 *                  the degree-array state (see oracle_greedy_ub below).
 *   oracle_remove_max_ub -> RemoveMaxApproximateMVC exactly (src/auxFunctions.cpp:
 *                  44-127, 211-256 with CSRGraph::deleteVertex, CSRGraphRep.cpp:44-62):
 *                  rows are compacted on deletion and the triangle test binary-searches
 *                  the compacted (unsorted) row, as the reference does.
 *   oracle_remove_edge_ub -> RemoveEdgeApproximateMVC exactly (auxFunctions.cpp:258-306),
 *                  with the value rand() returns after srand(time(0)) as a parameter.
 *   oracle_mcm  -> the edge-branching search of the reference's default build
 *                  (`#define VC 0`: GlobalWorkList_MCM.cuh:13-190), see below.
 *
 * Same rules, same order (leaf, triangle, high-degree; repeat while triangle or
 * high-degree changed), same branching (max-degree vertex, lowest index on ties;
 * the N(v) child is pushed and the v child is continued), same prune
 * (del >= best  or  E >= (best-del-1)^2 + 1).  Differences, all value-neutral:
 *   - the stack of full degree arrays grows on demand instead of being
 *     preallocated at (V+1)*V ints (Sequential.cpp:6-9);
 *   - (best-del-1)^2 is computed in 64-bit; the reference's int multiply
 *     (helperFunctions.cpp:3-6) overflows only above 46340, which no test reaches;
 *   - it counts tree nodes (one per computed reduction fixpoint), records the
 *     cover at each improving leaf (vertices whose degree is -1), and can stop at
 *     a node budget (status ORACLE_BUDGET).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_BUDGET 1
#define ORACLE_NOMEM 2

typedef struct {
    uint32_t n;
    const uint32_t *row_ptr; /* n+1 offsets into col */
    const uint32_t *col;     /* 2m neighbour ids, each row sorted ascending */
} og_graph;

/* helperFunctions.cpp:27-47 */
static void og_delete_vertex(const og_graph *g, uint32_t v, int32_t *deg, uint32_t *del)
{
    if (deg[v] < 0) return;
    for (uint32_t e = g->row_ptr[v]; e < g->row_ptr[v + 1]; ++e) {
        uint32_t u = g->col[e];
        if (deg[u] != -1) --deg[u];
    }
    deg[v] = -1;
    ++*del;
}

/* helperFunctions.cpp:49-75: sweep until no degree-1 vertex is found. */
static int og_leaf_rule(const og_graph *g, int32_t *deg, uint32_t *del)
{
    int deleted = 0, changed;
    do {
        changed = 0;
        for (uint32_t i = 0; i < g->n; ++i) {
            if (deg[i] == 1) {
                changed = 1;
                for (uint32_t e = g->row_ptr[i]; e < g->row_ptr[i + 1]; ++e) {
                    uint32_t u = g->col[e];
                    if (deg[u] != -1) {
                        deleted = 1;
                        og_delete_vertex(g, u, deg, del);
                    }
                }
            }
        }
    } while (changed);
    return deleted;
}

/* helperFunctions.cpp:77-96 */
static int og_high_degree_rule(const og_graph *g, int32_t *deg, uint32_t *del, uint32_t bound)
{
    int deleted = 0, changed;
    do {
        changed = 0;
        for (uint32_t i = 0; i < g->n; ++i) {
            if (deg[i] > 0 && (uint64_t)deg[i] + *del >= bound) {
                changed = deleted = 1;
                og_delete_vertex(g, i, deg, del);
            }
        }
    } while (changed);
    return deleted;
}

static int og_row_contains(const og_graph *g, uint32_t row, uint32_t x)
{
    uint32_t lo = g->row_ptr[row], hi = g->row_ptr[row + 1];
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (g->col[mid] == x) return 1;
        if (g->col[mid] < x) lo = mid + 1; else hi = mid;
    }
    return 0;
}

/* helperFunctions.cpp:98-155: a degree-2 vertex whose two live neighbours are
 * adjacent puts both neighbours in the cover; a degree-1 neighbour, or a
 * degree-2 neighbour with a smaller id, defers the vertex.  After one triangle
 * the sweep restarts from vertex 0 (the `break` at :150). */
static int og_triangle_rule(const og_graph *g, int32_t *deg, uint32_t *del)
{
    int deleted = 0, changed;
    do {
        changed = 0;
        for (uint32_t i = 0; i < g->n; ++i) {
            if (deg[i] != 2) continue;
            uint32_t n1 = 0, n2 = 0;
            int found1 = 0, keep = 0;
            for (uint32_t e = g->row_ptr[i]; e < g->row_ptr[i + 1]; ++e) {
                uint32_t u = g->col[e];
                int32_t du = deg[u];
                if (du > 0) {
                    if (du == 1 || (du == 2 && u < i)) { keep = 1; break; }
                    else if (!found1) { found1 = 1; n1 = u; }
                    else { n2 = u; break; }
                }
            }
            if (!keep && og_row_contains(g, n2, n1)) {
                changed = deleted = 1;
                og_delete_vertex(g, n1, deg, del);
                og_delete_vertex(g, n2, deg, del);
                break;
            }
        }
    } while (changed);
    return deleted;
}

typedef struct {
    int32_t *frames;   /* cap * n degree arrays */
    uint32_t *ndel;
    size_t cap;
    long top;
} og_stack;

static int og_push(og_stack *s, uint32_t n, const int32_t *deg, uint32_t del)
{
    if ((size_t)(s->top + 1) >= s->cap) {
        size_t nc = s->cap ? s->cap * 2 : 16;
        int32_t *f = (int32_t *)realloc(s->frames, nc * (size_t)(n ? n : 1) * sizeof(int32_t));
        if (!f) return 0;
        s->frames = f;
        uint32_t *d = (uint32_t *)realloc(s->ndel, nc * sizeof(uint32_t));
        if (!d) return 0;
        s->ndel = d;
        s->cap = nc;
    }
    ++s->top;
    memcpy(s->frames + (size_t)s->top * n, deg, (size_t)n * sizeof(int32_t));
    s->ndel[s->top] = del;
    return 1;
}

static void og_degrees(const og_graph *g, int32_t *deg)
{
    for (uint32_t v = 0; v < g->n; ++v) deg[v] = (int32_t)(g->row_ptr[v + 1] - g->row_ptr[v]);
}

/*
 * One search over the tree of Sequential.cpp:22-97 (mode 0, MVC) or
 * SequentialParameterized.cpp:25-104 (mode 1, PVC).
 *   MVC: `best` starts at `ub` and the return value is min(ub, OPT) exactly like
 *        Sequential(graph, ub); *improved says whether cover_out was written.
 *   PVC: high-degree bound k+1, prune del > k or E >= (k-del)^2 + 1, stop at the
 *        first leaf with del <= k; the return value is kFound.
 */
static int og_search(const og_graph *g, int mode, uint32_t ub, uint32_t k, uint8_t *cover_out,
                     uint64_t *nodes_out, uint64_t node_limit, uint32_t *result, int *improved)
{
    const uint32_t n = g->n;
    og_stack st = {0};
    st.top = -1;
    int32_t *deg = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    if (!deg) return ORACLE_NOMEM;
    og_degrees(g, deg);
    if (!og_push(&st, n, deg, 0)) { free(deg); return ORACLE_NOMEM; }

    uint32_t best = ub, del = 0, found = 0;
    uint64_t nodes = 0;
    int pop_next = 1, status = ORACLE_OK;
    *improved = 0;
    const uint32_t hd_bound = mode == 0 ? 0 : k + 1;

    while (st.top != -1 || !pop_next) {
        if (pop_next) {
            memcpy(deg, st.frames + (size_t)st.top * n, (size_t)n * sizeof(int32_t));
            del = st.ndel[st.top];
            --st.top;
        }
        if (node_limit && nodes >= node_limit) { status = ORACLE_BUDGET; break; }
        ++nodes;
        int tri, high;
        do {
            og_leaf_rule(g, deg, &del);
            tri = og_triangle_rule(g, deg, &del);
            high = og_high_degree_rule(g, deg, &del, mode == 0 ? best : hd_bound);
        } while (tri || high);

        uint32_t maxv = 0;
        int32_t maxd = 0;
        uint64_t sum = 0;
        for (uint32_t i = 0; i < n; ++i) {
            int32_t d = deg[i];
            if (d > maxd) { maxd = d; maxv = i; }
            if (d > 0) sum += (uint64_t)d;
        }
        uint64_t edges = sum / 2;

        int prune;
        if (mode == 0) {
            prune = del >= best;
            if (!prune) { uint64_t b = (uint64_t)(best - del - 1); prune = edges >= b * b + 1; }
        } else {
            prune = del > k;
            if (!prune) { uint64_t b = (uint64_t)(k - del); prune = edges >= b * b + 1; }
        }
        if (prune) { pop_next = 1; continue; }
        if (maxd == 0) {
            if (cover_out) for (uint32_t i = 0; i < n; ++i) cover_out[i] = deg[i] == -1;
            *improved = 1;
            if (mode == 0) { best = del; pop_next = 1; continue; }
            found = 1;
            break;
        }
        /* push the child that takes N(maxv), continue with the child that takes maxv */
        if (!og_push(&st, n, deg, del)) { status = ORACLE_NOMEM; break; }
        int32_t *right = st.frames + (size_t)st.top * n;
        for (uint32_t e = g->row_ptr[maxv]; e < g->row_ptr[maxv + 1]; ++e)
            og_delete_vertex(g, g->col[e], right, &st.ndel[st.top]);
        og_delete_vertex(g, maxv, deg, &del);
        pop_next = 0;
    }
    free(deg);
    free(st.frames);
    free(st.ndel);
    if (nodes_out) *nodes_out = nodes;
    *result = mode == 0 ? best : found;
    return status;
}

/* MVC: returns status; *size = min(ub, OPT).  cover_out (n bytes, 1 = in cover)
 * is written when the search found a cover smaller than ub (*improved = 1). */
int oracle_mvc(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t ub,
               uint32_t *size, uint8_t *cover_out, int *improved, uint64_t *nodes, uint64_t node_limit)
{
    og_graph g = {n, row_ptr, col};
    return og_search(&g, 0, ub, 0, cover_out, nodes, node_limit, size, improved);
}

/* PVC: returns status; *k_found = 1 iff the graph has a cover of size <= k
 * (cover_out then holds one). */
int oracle_pvc(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t k,
               uint32_t *k_found, uint8_t *cover_out, uint64_t *nodes, uint64_t node_limit)
{
    og_graph g = {n, row_ptr, col};
    int improved = 0;
    return og_search(&g, 1, 0, k, cover_out, nodes, node_limit, k_found, &improved);
}

/* A valid upper bound with its cover: leaf and triangle rules to a fixpoint,
 * then take the max-degree vertex, until no edge is left (the shape of
 * auxFunctions.cpp:211-256, stated on the degree-array state rather than on the
 * mutated CSR copy the reference uses). */
uint32_t oracle_greedy_ub(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint8_t *cover_out)
{
    og_graph g = {n, row_ptr, col};
    int32_t *deg = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    if (!deg) return n;
    og_degrees(&g, deg);
    uint32_t del = 0;
    for (;;) {
        int tri;
        do {
            og_leaf_rule(&g, deg, &del);
            tri = og_triangle_rule(&g, deg, &del);
        } while (tri);
        uint32_t maxv = 0;
        int32_t maxd = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (deg[i] > maxd) { maxd = deg[i]; maxv = i; }
        if (maxd == 0) break;
        og_delete_vertex(&g, maxv, deg, &del);
    }
    if (cover_out) for (uint32_t i = 0; i < n; ++i) cover_out[i] = deg[i] == -1;
    free(deg);
    return del;
}

/* RemoveMaxApproximateMVC (src/auxFunctions.cpp:211-256) restated exactly on a
 * working copy of the CSR that deletions compact, as CSRGraph::deleteVertex
 * does (CSRGraphRep.cpp:44-62): deleting v takes v out of the live prefix of
 * each live neighbour's row by copying that row's last live entry over it.
 * One iteration runs the leaf rule to a fixpoint (auxFunctions.cpp:44-69: passes
 * over the vertices in index order while a pass met a degree-1 vertex), then
 * the triangle rule to a fixpoint (:71-127: the first degree-2 vertex whose two
 * live neighbours pass the keep test and are found adjacent by a binary search
 * of the second neighbour's whole, compacted row; restart from vertex 0), then
 * deletes the lowest-index vertex of maximum degree; both rules return false, so
 * the do-while of :222-231 runs once.  The binary search (:25-42) is the same
 * except that where the reference's unsigned index would step below 0 (and read
 * out of bounds) this one stops with "not found".  Returns the cover size; the
 * cover (vertices deleted) goes to cover_out when non-null. */
static void rm_delete(const uint32_t *rp, uint32_t *dst, int32_t *deg, uint32_t v)
{
    const uint32_t b = rp[v], e = b + (uint32_t)deg[v];
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t w = dst[i];
        const uint32_t last = rp[w] + (uint32_t)deg[w];
        for (uint32_t j = rp[w]; j < last; ++j) {
            if (dst[j] == v) {
                dst[j] = dst[last - 1];
                if (deg[w] != -1) --deg[w];
            }
        }
    }
    deg[v] = -1;
}

static int rm_search(const uint32_t *arr, long l, long r, uint32_t x)
{
    while (l <= r) {
        const long m = l + (r - l) / 2;
        if (arr[m] == x) return 1;
        if (arr[m] < x) l = m + 1;
        else r = m - 1;
    }
    return 0;
}

uint32_t oracle_remove_max_ub(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint8_t *cover_out)
{
    const uint32_t m2 = row_ptr[n];
    uint32_t *dst = (uint32_t *)malloc((size_t)(m2 ? m2 : 1) * sizeof(uint32_t));
    int32_t *deg = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    if (!dst || !deg) { free(dst); free(deg); return n; }
    memcpy(dst, col, (size_t)m2 * sizeof(uint32_t));
    for (uint32_t v = 0; v < n; ++v) deg[v] = (int32_t)(row_ptr[v + 1] - row_ptr[v]);
    uint32_t minimum = 0;
    for (;;) {
        int changed;
        do {  /* leaf rule */
            changed = 0;
            for (uint32_t i = 0; i < n; ++i) {
                if (deg[i] != 1) continue;
                changed = 1;
                for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j)
                    if (deg[dst[j]] != -1) { rm_delete(row_ptr, dst, deg, dst[j]); ++minimum; }
            }
        } while (changed);
        do {  /* triangle rule */
            changed = 0;
            for (uint32_t i = 0; i < n; ++i) {
                if (deg[i] != 2) continue;
                uint32_t n1 = 0, n2 = 0;
                int found1 = 0, keep = 0;
                for (uint32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                    const uint32_t u = dst[e];
                    const int32_t du = deg[u];
                    if (du > 0) {
                        if (du == 1 || (du == 2 && u < i)) { keep = 1; break; }
                        else if (!found1) { found1 = 1; n1 = u; }
                        else { n2 = u; break; }
                    }
                }
                if (!keep && rm_search(dst, (long)row_ptr[n2], (long)row_ptr[n2 + 1] - 1, n1)) {
                    rm_delete(row_ptr, dst, deg, n1);
                    rm_delete(row_ptr, dst, deg, n2);
                    minimum += 2;
                    changed = 1;
                    break;
                }
            }
        } while (changed);
        uint32_t maxv = 0;
        int32_t maxd = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (deg[i] > maxd) { maxv = i; maxd = deg[i]; }
        if (maxd == 0) break;
        rm_delete(row_ptr, dst, deg, maxv);
        ++minimum;
    }
    if (cover_out) for (uint32_t i = 0; i < n; ++i) cover_out[i] = deg[i] == -1;
    free(dst);
    free(deg);
    return minimum;
}

/* RemoveEdgeApproximateMVC (src/auxFunctions.cpp:258-306) restated exactly,
 * on the same compacting CSR copy as oracle_remove_max_ub.  For each vertex in
 * index order, while the running edge count is positive: the leaf rule and the
 * triangle rule to their fixpoints (the do-while runs once, both rules return
 * false), then, if the vertex still has live neighbours, it and the neighbour at
 * row position (r mod degree) of its compacted row go into the cover.  The
 * reference draws that position with srand(time(0)); rand() on every call
 * (getRandom, :251-256), i.e. one value r for all calls within one second; here r
 * is a parameter.  The edge count is decremented only for the pair taken, as in
 * the reference (unsigned arithmetic).  Returns the cover size. */
uint32_t oracle_remove_edge_ub(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t r,
                               uint8_t *cover_out)
{
    const uint32_t m2 = row_ptr[n];
    uint32_t *dst = (uint32_t *)malloc((size_t)(m2 ? m2 : 1) * sizeof(uint32_t));
    int32_t *deg = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
    if (!dst || !deg) { free(dst); free(deg); return n; }
    memcpy(dst, col, (size_t)m2 * sizeof(uint32_t));
    for (uint32_t v = 0; v < n; ++v) deg[v] = (int32_t)(row_ptr[v + 1] - row_ptr[v]);
    uint32_t minimum = 0, remaining = m2 / 2;
    for (uint32_t vertex = 0; vertex < n && remaining > 0; ++vertex) {
        int changed;
        do {  /* leaf rule */
            changed = 0;
            for (uint32_t i = 0; i < n; ++i) {
                if (deg[i] != 1) continue;
                changed = 1;
                for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j)
                    if (deg[dst[j]] != -1) { rm_delete(row_ptr, dst, deg, dst[j]); ++minimum; }
            }
        } while (changed);
        do {  /* triangle rule */
            changed = 0;
            for (uint32_t i = 0; i < n; ++i) {
                if (deg[i] != 2) continue;
                uint32_t n1 = 0, n2 = 0;
                int found1 = 0, keep = 0;
                for (uint32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                    const uint32_t u = dst[e];
                    const int32_t du = deg[u];
                    if (du > 0) {
                        if (du == 1 || (du == 2 && u < i)) { keep = 1; break; }
                        else if (!found1) { found1 = 1; n1 = u; }
                        else { n2 = u; break; }
                    }
                }
                if (!keep && rm_search(dst, (long)row_ptr[n2], (long)row_ptr[n2 + 1] - 1, n1)) {
                    rm_delete(row_ptr, dst, deg, n1);
                    rm_delete(row_ptr, dst, deg, n2);
                    minimum += 2;
                    changed = 1;
                    break;
                }
            }
        } while (changed);
        if (deg[vertex] > 0) {
            const uint32_t e = row_ptr[vertex] + r % (uint32_t)deg[vertex];
            const uint32_t u = dst[e];
            remaining -= (uint32_t)deg[vertex];
            remaining -= (uint32_t)deg[u];
            ++remaining;
            rm_delete(row_ptr, dst, deg, vertex);
            rm_delete(row_ptr, dst, deg, u);
            minimum += 2;
        }
    }
    if (cover_out) for (uint32_t i = 0; i < n; ++i) cover_out[i] = deg[i] == -1;
    free(dst);
    free(deg);
    return minimum;
}

/* Edge-by-edge check: 1 iff every edge has an endpoint with cover[v] != 0. */
int oracle_is_cover(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint8_t *cover)
{
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t e = row_ptr[v]; e < row_ptr[v + 1]; ++e)
            if (!cover[v] && !cover[col[e]]) return 0;
    return 1;
}

/* oracle_mcm -> the search of the reference's default build (`#define VC 0`,
 * src/main.cu:9-36): GlobalWorkList_MCM.cuh:13-190 with findNextEdge
 * (helperFunctions.cuh:86-102), skipEdge (:188-195), deleteNextEdge (:218-225)
 * and getMatchedVertices (:532-553).  Depth first with the "match" child first
 * and no pruning beyond the reference's own (a node whose every vertex is
 * matched or isolated, or a maximum already equal to n, is a leaf).  A vertex
 * is available while unmatched with degree > 0; a node counts the unavailable
 * ones, takes the first CSR entry at or after its cursor whose row and column
 * vertices are both available, and branches into "match both" (cursor stays at
 * the entry, which is now ineligible) and "skip it" (cursor past the entry).
 * Returns ORACLE_OK or ORACLE_BUDGET; *best_out = the maximum count over leaves
 * (2 * maximum matching + isolated vertices on a finished tree). */
int oracle_mcm(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint64_t node_limit, uint32_t *best_out,
               uint64_t *nodes_out)
{
    const uint32_t m2 = row_ptr[n];
    uint32_t *src = (uint32_t *)malloc(sizeof(uint32_t) * (m2 ? m2 : 1));
    uint8_t *avail = (uint8_t *)malloc(n ? n : 1);
    uint32_t *frame = (uint32_t *)malloc(sizeof(uint32_t) * (n / 2 + 1));
    uint32_t avc = 0, best = 0, level = 0, cursor = 0;
    uint64_t nodes = 0;
    int status = ORACLE_OK;
    for (uint32_t v = 0; v < n; ++v) {
        for (uint32_t e = row_ptr[v]; e < row_ptr[v + 1]; ++e) src[e] = v;
        avail[v] = row_ptr[v + 1] > row_ptr[v];
        avc += avail[v];
    }
    for (;;) {
        ++nodes;
        if (node_limit && nodes > node_limit) {
            status = ORACLE_BUDGET;
            break;
        }
        const uint32_t cnt = n - avc;
        uint32_t next = m2;
        if (cnt < n && best < n)
            for (uint32_t e = cursor; e < m2; ++e)
                if (avail[src[e]] && avail[col[e]]) {
                    next = e;
                    break;
                }
        if (next < m2) {  /* match the entry's two vertices; the skip child waits on the frame */
            frame[level++] = next;
            avail[src[next]] = avail[col[next]] = 0;
            avc -= 2;
            cursor = next;
            continue;
        }
        if (cnt > best) best = cnt;  /* a leaf */
        if (level == 0) break;
        const uint32_t e = frame[--level];  /* the skip child of the deepest matched entry */
        avail[src[e]] = avail[col[e]] = 1;
        avc += 2;
        cursor = e + 1;
    }
    free(src);
    free(avail);
    free(frame);
    *best_out = best;
    if (nodes_out) *nodes_out = nodes;
    return status;
}
