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

/* Edge-by-edge check: 1 iff every edge has an endpoint with cover[v] != 0. */
int oracle_is_cover(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint8_t *cover)
{
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t e = row_ptr[v]; e < row_ptr[v + 1]; ++e)
            if (!cover[v] && !cover[col[e]]) return 0;
    return 1;
}
