/*
 * vcgpu.h -- C ABI of the B200 exact vertex-cover solver (libvcgpu.so).
 *
 * The reference (GregorySchwing/Parallel-Vertex-Cover-Algorithms-on-GPUs) has no
 * library API: its boundary is the `./output` command line plus one kernel
 * launch per solve.  Each entry point below names the reference interface it
 * replaces.  Plain pointers and sizes only; no CUDA or torch types appear in
 * the signatures (a stream is passed as `void*`, a cudaStream_t).
 *
 * Ownership: every input is borrowed and never freed; outputs are caller-owned.
 * Errors are returned as vc_status codes -- nothing here calls exit().
 * Threading: calls are serialised per device inside the library; a server
 * handle (vc_server_*) is used by one host thread at a time.
 */
#ifndef VCGPU_H
#define VCGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vc_status {
    VC_OK = 0,
    VC_ERR_INVALID = 1,   /* bad argument or malformed graph */
    VC_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    VC_ERR_NOMEM = 3,     /* device memory or the admission budget is exhausted */
    VC_ERR_TOO_LARGE = 4, /* the graph exceeds what the kernels support */
    VC_TIMEOUT = 5,       /* stopped at the time limit: size is an upper bound */
    VC_BUDGET = 6,        /* stopped at the node limit: size is an upper bound */
    VC_ERR_INTERNAL = 7,  /* a device-side consistency check failed */
    VC_ERR_NO_DEVICE = 8, /* no usable CUDA device */
    VC_PENDING = 9        /* server: the request is still running */
} vc_status;

typedef enum vc_instance {
    VC_MVC = 0, /* minimum vertex cover (reference `-i mvc`, config.h:125-129) */
    VC_PVC = 1  /* parameterized vertex cover, decision size <= k (`-i pvc -k K`) */
} vc_instance;

/* vc_request.flags.  Host-resident graphs are checked on the host (monotone
 * offsets, ids < n, no self loop or duplicate, sorted symmetric rows) unless
 * VC_FLAG_NO_VALIDATE.  Device-resident graphs (VC_FLAG_DEVICE_INPUT, and
 * vc_solve_batch_device) cannot be read by the host: a kernel checks the layout
 * the search relies on for memory safety -- row_ptr[0] = 0, row_ptr[n] = 2m as
 * stated by the caller, monotone offsets, ids < n, no self loop -- and a graph
 * that fails is reported VC_ERR_INVALID without being searched.  Sortedness,
 * duplicates and symmetry of device-resident rows are trusted: a graph that
 * breaks them gets a wrong answer, never an access outside its arrays. */
#define VC_FLAG_DEVICE_INPUT 0x1u /* vc_csr / arena pointers are device pointers */
#define VC_FLAG_NO_VALIDATE 0x2u  /* skip the host-side CSR checks */

/* One undirected simple graph in the reference's CSRGraph layout
 * (src/CSRGraphRep.h:4-18): row_ptr = srcPtr[n+1], col = dst[2m] with every
 * edge stored in both directions and each row sorted ascending
 * (src/auxFunctions.cpp:203-206); degree (optional, may be NULL) must equal
 * row_ptr[v+1]-row_ptr[v].  Ids are 0-based. */
typedef struct vc_csr {
    uint32_t n;
    uint32_t m;
    const uint32_t *row_ptr;
    const uint32_t *col;
    const int32_t *degree;
} vc_csr;

/* Many graphs packed into one arena: graph i has n[i] vertices, its n[i]+1
 * local row offsets start at row_ptr[row_off[i]] and its neighbour ids at
 * col[col_off[i]]. */
typedef struct vc_csr_arena {
    uint32_t count;
    const uint32_t *n;
    const uint64_t *row_off;
    const uint64_t *col_off;
    const uint32_t *row_ptr;
    const uint32_t *col;
} vc_csr_arena;

/* What to solve.  `ub` plays the role of the reference's `minimum` argument
 * (main.cu:73 / Sequential(graph, minimum)): when nonzero the search only looks
 * for covers of size <= ub, and size = min(ub, OPT) like the reference returns;
 * 0 means no bound.  node_limit / time_limit_s stop a search early (status
 * VC_BUDGET / VC_TIMEOUT); 0 means unlimited / the library default (300 s). */
typedef struct vc_request {
    uint32_t instance;   /* vc_instance */
    uint32_t k;          /* PVC parameter (reference -k) */
    uint32_t ub;
    uint32_t flags;      /* VC_FLAG_* */
    uint64_t node_limit;
    double time_limit_s;
    int32_t device;      /* CUDA ordinal, -1 = current device */
    uint32_t reserved;
    void *stream;        /* cudaStream_t to run on, NULL = the library's stream */
} vc_request;

/* Result of one graph.  For MVC `size` is the minimum cover size (upper bound on
 * VC_TIMEOUT / VC_BUDGET) and `decision` is 1; for PVC `decision` is 1 iff a
 * cover of size <= k exists (the reference's kFound, main.cu:355-356) and
 * `size` is the size of the cover returned.  `cover_mask` (caller-owned, n
 * bytes, may be NULL) receives 1 for every vertex in the returned cover; when
 * no cover of size <= ub was found (MVC with ub < OPT+... or PVC "no") it is
 * left zeroed and has_cover is 0. */
typedef struct vc_result {
    uint32_t size;
    uint32_t decision;
    uint32_t has_cover;
    vc_status status;
    uint8_t *cover_mask;
    uint64_t tree_nodes;  /* search-tree nodes whose reduction fixpoint was computed */
    float kernel_ms;      /* device time of the search launch */
    float total_ms;       /* wall time of the call, copies included */
    float done_ms;        /* from the launch's start until this graph finished */
    uint32_t reserved;
} vc_result;

/* Plain one-graph solve; replaces the host path of main.cu:101-359 (device
 * query, sizing, allocation, the GlobalWorkList / GlobalWorkListParameterized
 * kernel launch at main.cu:302-314 and the read-back of minimum / kFound). */
vc_status vc_solve(const vc_csr *g, const vc_request *req, vc_result *out);

/* Batched solve: every graph of the arena in one persistent launch with a
 * shared device worklist (no counterpart in the reference, which launches one
 * graph per process).  reqs has `arena->count` entries; out likewise (each
 * out[i].cover_mask, if non-NULL, holds n[i] bytes).  Returns the first
 * non-OK per-graph status, or VC_OK. */
vc_status vc_solve_batch(const vc_csr_arena *arena, const vc_request *reqs, vc_result *out);

/* The same over an arena already resident on the device: `arena` holds the
 * host copies (n, row_off, col_off, row_ptr are read on the host to size the
 * launch), d_row_ptr / d_col the device copies the kernels read. */
vc_status vc_solve_batch_device(const vc_csr_arena *arena, const uint32_t *d_row_ptr, const uint32_t *d_col,
                                const vc_request *reqs, vc_result *out);

/* The reference's upper-bound heuristics on the GPU, one CTA per graph of the
 * arena (any sizes; host arrays, copied by the call).
 * vc_remove_max_ub replaces RemoveMaxApproximateMVC (src/auxFunctions.cpp:211-256),
 * vc_remove_edge_ub replaces RemoveEdgeApproximateMVC (:258-306).  Both return the
 * same bound as the reference on the same graph: the kernel keeps the reference's
 * order of deletions, its rule sweeps and the row order its deleteVertex leaves
 * (CSRGraphRep.cpp:44-62).  The reference draws RemoveEdge's edges with
 * srand(time(0)); rand(), one value per second of wall time: r is that value.
 * ub[i] receives graph i's bound; cover (optional) receives n_i bytes per graph,
 * in arena order, 1 = in the cover; kernel_ms (optional) the kernel time. */
vc_status vc_remove_max_ub(const vc_csr_arena *arena, int32_t device, uint32_t *ub, uint8_t *cover, float *kernel_ms);
vc_status vc_remove_edge_ub(const vc_csr_arena *arena, uint32_t r, int32_t device, uint32_t *ub, uint8_t *cover,
                            float *kernel_ms);

/* The MCM mode: the search the reference's default build runs (`#define VC 0`,
 * src/main.cu:9-36; GlobalWorkList_MCM.cuh:13-190 replaces the hybrid MVC
 * kernel there).  An edge-branching search in CSR entry order: a node counts
 * its matched and isolated vertices, takes the first entry at or after its
 * cursor whose two vertices are unmatched and non-isolated, and branches into
 * "match it" and "skip it"; a leaf raises the launch's maximum.  out->size
 * receives that maximum -- 2 * (maximum matching) + (isolated vertices) once the
 * tree is finished, the `minimum` field of the reference's Results.csv row; its
 * CLI prints half of it as "Size of maximum matching" -- and tree_nodes /
 * kernel_ms as vc_solve.  req->instance must be VC_MVC (the reference's MCM
 * build refuses PVC, main.cu:155-189); graphs of up to 1024 vertices
 * (VC_ERR_TOO_LARGE above); host input only.  VC_TIMEOUT / VC_BUDGET leave the
 * largest count reached so far. */
vc_status vc_mcm(const vc_csr *g, const vc_request *req, vc_result *out);

/* The autotuner (replaces the reference's fixed launch-sizing rule,
 * setBlockDimAndUseGlobalMemoryAutoWorkListSize, src/auxFunctions.cpp:469-578):
 * for each size class of graphs (dense n <= 64, <= 128, <= 255; wide dense
 * n <= 640; 16-bit dense n <= 1024; CSR larger) it times candidate launch shapes -- warp
 * or CTA search units, warps per CTA, CTA pool slots (the shared-memory stack
 * of donated subtrees) per warp, the global-ring donation threshold and the
 * donation order -- on seeded calibration graphs of the class for slice_s
 * seconds each (0 = 0.3 s; about 15 s in all) and installs the fastest for the
 * device's later solves.  table (optional, at least 42 words) receives per
 * class: set, cta_units, warps, pool slots per warp, ring threshold (int32),
 * tree nodes/s (float bits), ring first.
 * vc_set_tuning installs such a table (e.g. saved from an earlier run); a class
 * with set = 0 uses the built-in rules. */
vc_status vc_autotune(int32_t device, double slice_s, uint32_t *table, uint32_t max_words);
vc_status vc_set_tuning(int32_t device, const uint32_t *table, uint32_t words);

/* Continuous-batching server (no counterpart in the reference).  Persistent
 * kernels admit requests while others run; graphs and search state stay on the
 * device.  mem_budget_bytes bounds the device arenas holding admitted graphs
 * (0 = 1 GiB); max_requests is the number of device slots per lane (0 = 1024);
 * max_vertices is the largest graph accepted (0 = 1024).  With max_vertices <=
 * 255 there is one lane, the dense-bitset kernel on the whole device.  Above
 * that there are three lanes side by side on every SM: requests of at most
 * 255 vertices run in the dense lane, requests of 256..640 vertices whose
 * degrees are all at most 254 in the wide dense lane, the rest in a CSR lane;
 * the two dense lanes' kernels stay resident while the server lives.  A
 * request is admitted when a slot and arena room for its CSR are free in its
 * lane.  submit validates and copies the graph and returns a ticket (its lane
 * in the low two bits); poll returns VC_PENDING until the ticket's result is
 * ready, then fills *out (out->cover_mask, if non-NULL, receives n bytes;
 * total_ms is the time from submit to completion) and releases the ticket.
 * While a server runs on a device, its kernels hold that device's SMs. */
typedef struct vc_server vc_server;
vc_status vc_server_create(int32_t device, uint64_t mem_budget_bytes, uint32_t max_requests, uint32_t max_vertices,
                           vc_server **out);
vc_status vc_server_submit(vc_server *s, const vc_csr *g, const vc_request *req, uint64_t *ticket);
vc_status vc_server_poll(vc_server *s, uint64_t ticket, vc_result *out);
/* Tickets finished since the last call and not yet collected by vc_server_poll
 * (at most max_tickets, oldest first): lets a caller with many requests in
 * flight poll only the finished ones. No counterpart in the reference. */
vc_status vc_server_completed(vc_server *s, uint64_t *tickets, uint32_t max_tickets, uint32_t *count);
/* The server's lanes (1 to 3) into shape[6*i..]: largest request (vertices),
 * grid, block, search units, dynamic shared memory per CTA, dense (1) or CSR
 * (0) kernel; *lanes receives the lane count.  A diagnostic without a
 * counterpart in the reference. */
vc_status vc_server_shape(vc_server *s, uint32_t *shape, uint32_t max_lanes, uint32_t *lanes);
vc_status vc_server_destroy(vc_server *s);

/* Solve one graph of at most 255 vertices without allocating any memory (no
 * counterpart in the reference).  For callers that may not call cudaMalloc --
 * code whose device memory is owned by a framework's pool, hosts that forbid
 * allocation after start-up, callers that cannot afford an allocation's
 * implicit synchronisation.  The graph (g->row_ptr, g->col) must be in device
 * memory and req->flags must include VC_FLAG_DEVICE_INPUT.  Runs asynchronously
 * on req->stream; writes 8 words to the caller's device buffer d_result
 * (status, size, decision, has_cover, tree nodes low, tree nodes high, 0, 0)
 * and, if d_cover is not NULL, the cover as ceil(n/32) bitmap words.  All
 * scratch lives in one fixed 256 KiB device array per GPU (held until the
 * process exits) that every call shares: calls that overlap on the GPU race and
 * must be serialised by the caller.  The first call on a device does that
 * device's set-up and should come before any stream capture.  Larger graphs
 * return VC_ERR_TOO_LARGE. */
vc_status vc_solve_noalloc(const vc_csr *g, const vc_request *req, uint32_t *d_result, uint32_t *d_cover);

/* Diagnostics: the kernels launched by this library since load (for checking
 * that the device path ran), and a static status string. */
uint64_t vc_kernel_launches(void);
const char *vc_status_string(vc_status s);

#ifdef __cplusplus
}
#endif
#endif
