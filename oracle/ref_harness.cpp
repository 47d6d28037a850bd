// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own CPU solver, compiled from the reference
// sources where they lie (see oracle/Makefile; nothing from the reference is
// copied into this repository).  It lets the tests and bench.py's reference arm
// call, through ctypes:
//   ref_mvc           -> Sequential(graph, ub)                  src/Sequential.cpp:3
//   ref_pvc           -> SequentialParameterized(graph, k+1, k) src/SequentialParameterized.cpp:4
//                        (high-degree bound k+1 as in GlobalWorkListParameterized.cuh:127)
//   ref_remove_max_ub -> RemoveMaxApproximateMVC(graph)         src/auxFunctions.cpp:211
//   ref_load          -> createCSRGraphFromFile(path)           src/auxFunctions.cpp:129
// Sequential* free the graph they are given (Sequential.cpp:99), so every call
// builds a fresh CSRGraph from the caller's arrays.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include "CSRGraphRep.h"
#include "Sequential.h"
#include "SequentialParameterized.h"
#include "auxFunctions.h"

static CSRGraph make_graph(uint32_t n, const uint32_t *row_ptr, const uint32_t *col)
{
    CSRGraph g;
    g.vertexNum = n;
    g.edgeNum = row_ptr[n] / 2;
    g.srcPtr = (unsigned int *)malloc(sizeof(unsigned int) * (n + 1));
    g.dst = (unsigned int *)malloc(sizeof(unsigned int) * (row_ptr[n] ? row_ptr[n] : 1));
    g.degree = (int *)malloc(sizeof(int) * (n ? n : 1));
    g.srcPtrUncompressed = nullptr;
    memcpy(g.srcPtr, row_ptr, sizeof(unsigned int) * (n + 1));
    memcpy(g.dst, col, sizeof(unsigned int) * row_ptr[n]);
    for (uint32_t v = 0; v < n; ++v) g.degree[v] = (int)(row_ptr[v + 1] - row_ptr[v]);
    return g;
}

extern "C" uint32_t ref_mvc(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t ub)
{
    return Sequential(make_graph(n, row_ptr, col), ub);
}

extern "C" uint32_t ref_pvc(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t k)
{
    unsigned int k_found = 0;
    SequentialParameterized(make_graph(n, row_ptr, col), k + 1, k, &k_found);
    return k_found;
}

extern "C" uint32_t ref_remove_max_ub(uint32_t n, const uint32_t *row_ptr, const uint32_t *col)
{
    CSRGraph g = make_graph(n, row_ptr, col);
    uint32_t ub = RemoveMaxApproximateMVC(g);
    g.del();
    return ub;
}

// RemoveEdgeApproximateMVC(graph) (src/auxFunctions.cpp:258), which draws its
// edges with srand(time(0)); rand() on every call.  When the run starts and ends
// in the same second, *r_out receives the value those calls returned and the
// bound is returned; otherwise UINT32_MAX.
extern "C" uint32_t ref_remove_edge_ub(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t *r_out)
{
    CSRGraph g = make_graph(n, row_ptr, col);
    const time_t t0 = time(0);
    uint32_t ub = RemoveEdgeApproximateMVC(g);
    const time_t t1 = time(0);
    g.del();
    if (t0 != t1) return UINT32_MAX;
    srand((unsigned)t0);
    *r_out = (uint32_t)rand();
    return ub;
}

// Loads a reference-format graph file; the caller frees *row_ptr and *col with
// ref_free.  Returns 0 on success.
extern "C" int ref_load(const char *path, uint32_t *n, uint32_t *m, uint32_t **row_ptr, uint32_t **col)
{
    CSRGraph g = createCSRGraphFromFile(path);
    *n = g.vertexNum;
    *m = g.edgeNum;
    *row_ptr = g.srcPtr;
    *col = g.dst;
    free(g.degree);
    free(g.srcPtrUncompressed);
    return 0;
}

extern "C" void ref_free(void *p) { free(p); }
