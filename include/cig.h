/*
 * cig.h - C ABI of libcig, the B200 (sm_100a) incremental streaming-graph engine.
 *
 * The reference has no plugin or FFI layer: its boundary is the command line
 * and text files of four executables (CMakeLists.txt:52-90), built on the
 * compile-time operator concept AppBase (include/framework/variants/api.cuh:
 * 22-174) and the Engine methods the samples call.  This header is the thin
 * C layer under our drop-in hybrid_bfs / hybrid_sssp / hybrid_cc / hybrid_pr
 * tools; each entry point names the reference interface it replaces.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative cig_status code.
 *     cig_last_error(h) describes the most recent failure on that handle.
 *     No C++ exception crosses this boundary.
 *   - Host pointers passed in are borrowed for the duration of the call.
 *     Outputs are caller-allocated.  Entry points ending in _device take
 *     device pointers (CUDA global memory on the handle's device).
 *   - A handle is used by one host thread at a time; different handles may be
 *     used concurrently.  After an error reported as CIG_ERR_DEVICE the
 *     handle's device state is undefined and the handle should be destroyed.
 *   - Vertex ids are uint32; distances/labels use 0xFFFFFFFF as "unreached".
 */
#ifndef CIG_H
#define CIG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cig_handle cig_handle;

typedef enum {
    CIG_OK = 0,
    CIG_ERR_ARG = -1,       /* invalid argument or call order */
    CIG_ERR_NOMEM = -2,     /* host or device allocation failed */
    CIG_ERR_DEVICE = -3,    /* CUDA error */
    CIG_ERR_ARENA = -4,     /* adjacency arena exhausted */
    CIG_ERR_LIMIT = -5,     /* a round/iteration bound or a device wait limit was hit */
    CIG_ERR_STATE = -6,     /* handle unusable after an earlier device error */
    CIG_ERR_NOTIMPL = -7
} cig_status;

/* Algorithms of the four reference samples (samples/hybrid_{bfs,sssp,cc,pr}). */
typedef enum { CIG_BFS = 0, CIG_SSSP = 1, CIG_CC = 2, CIG_PR = 3 } cig_algo;

typedef struct {
    int32_t algo;            /* cig_algo */
    int32_t device;          /* CUDA device ordinal */
    uint32_t source;         /* --source_node (clamped to [0, n-1] at load) */
    int32_t cache_compat;    /* 1: reference --cache table (include/framework/graph_datum.cuh:158-170) */
    double cache_gib;        /* --cache: HBM edge-cache budget in GiB of uint32 slots */
    double pr_epsilon;       /* --error: absolute per-vertex residual threshold */
    int32_t pr_max_rounds;   /* --pr_max_rounds (1..100 in the reference; any >0 here) */
    uint32_t max_batch;      /* largest deletion or insertion phase to size buffers for (0: grow) */
    uint32_t arena_headroom_pct; /* extra arena capacity in percent (0: default 12.5%) */
    uint32_t flags;          /* CIG_FLAG_* */
    double index_budget_gib; /* device bytes for the two position-index tables, GiB (0: a quarter of the
                                free device memory per table); the indexed row-class threshold rises until
                                the tables fit, and rows of smaller classes fall back to the row scan */
} cig_options;

#define CIG_FLAG_NO_CACHE_REFRESH 0x1u /* keep the segment residency chosen at load */
#define CIG_FLAG_PR_FP64 0x2u          /* PR ranks/residuals in FP64 (default: FP32 + Kahan) */
#define CIG_FLAG_NO_GRAPHS 0x8u         /* launch every batch kernel directly (default: a batch shape seen twice
                                          is captured into CUDA graphs and replayed) */
#define CIG_FLAG_WEIGHT_U255 0x4u      /* SSSP weights uniform in [1, 255]: 1 + lowbias32(u*0x9E3779B1 +
                                          v*0x85EBCA77) mod 255 (an extension; the reference's SSSP
                                          weight is (u+v)%128+1 whatever the file holds) */

typedef struct {
    uint64_t requested_deletes;
    uint64_t missing_deletes;    /* as ChunkStoreBatchMetrics::missing_deletes (source_local_chunk_store.h:36-40) */
    uint64_t requested_additions;
    uint64_t invalid_additions;  /* out-of-range source or destination */
    uint64_t changed_sources;
    uint64_t relocated_rows;     /* rows moved to a larger block */
    uint64_t affected;           /* vertices invalidated by deletions (BFS/SSSP/CC) */
    uint64_t seeds;              /* vertices improved directly by inserted edges */
    uint64_t rounds;             /* traversal rounds (all closures of the batch) */
    uint64_t edges_scanned;      /* forward + reverse adjacency entries read by traversal */
    uint64_t edges_scanned_cached; /* of which read from the HBM edge cache or device arena */
    uint64_t vertices_expanded;
    uint64_t cache_segments_loaded;
    uint64_t cache_segments_evicted;
    double ms_delete;            /* device time of the deletion phase */
    double ms_insert;            /* device time of the insertion phase */
    double ms_cache;             /* device time of cache maintenance */
    uint64_t pr_rounds;
    double pr_residual_l1;       /* FP64 L1 norm of the PR residual after the batch */
    uint64_t kernel_launches;    /* engine kernels launched by the call (library sort kernels excluded),
                                    directly or as nodes of a replayed graph */
    uint64_t graph_replays;      /* captured batch graphs launched by the call (0: direct launches) */
} cig_batch_stats;

typedef struct {
    uint32_t n;
    uint64_t m;
    uint64_t arena_capacity_edges;
    uint64_t arena_used_edges;
    uint64_t segment_edges;
    uint64_t segments_total;
    uint64_t segments_resident;
    uint64_t cache_capacity_segments;
    uint64_t device_bytes;
    uint64_t pinned_bytes;
} cig_graph_info;

/* Device memory held by a handle, by part (bytes).  No reference
 * counterpart (the reference sizes its cache in graph_datum.cuh:158-176 and
 * keeps its reverse index in host memory). */
typedef struct {
    uint64_t total;          /* sum of the parts below */
    uint64_t edge_cache;     /* HBM edge cache (the --cache budget, whole 64 KiB segments) */
    uint64_t segment_table;  /* segment -> cache-slot map, dirty flags, scores, free stack */
    uint64_t descriptors;    /* forward row descriptors (16 B per vertex) */
    uint64_t reverse_arena;  /* device-only in-edge arena and its descriptors */
    uint64_t position_index; /* both position-index tables and row bitmaps */
    uint64_t vertex_state;   /* values/parents, stamps, frontier queues, PR arrays */
    uint64_t batch_buffers;  /* per-batch update, key, group and sort scratch buffers */
    uint64_t query_buffers;  /* multi-source query buffers (allocated on first query) */
    uint64_t pinned_host;    /* pinned mapped host arena + staging (host memory, not in total) */
} cig_memory_info;

int cig_memory_info_get(cig_handle *h, cig_memory_info *out);

/* Fill `o` with the reference's defaults (app_skeleton.h:42-90 and the
 * per-sample flags). */
int cig_options_default(cig_options *o);

/* Replaces Engine construction (include/framework/framework.cuh:545-563). */
int cig_create(const cig_options *o, cig_handle **out);
int cig_destroy(cig_handle *h);
const char *cig_last_error(const cig_handle *h);

/* Replaces traversal::Context / ReadGraphMarket_bigdata + LoadGraph
 * (src/utils/parser.cpp:292-402, include/framework/framework.cuh:800-986):
 * builds the adjacency from a CSR whose rows are in stored ("file") order. */
int cig_load_csr(cig_handle *h, uint32_t n, const uint64_t *xadj, const uint32_t *adj);

/* Same, from an edge list in file order (rows keep file order). */
int cig_load_edges(cig_handle *h, uint32_t n, const uint32_t *src, const uint32_t *dst, uint64_t m);

/* Replaces InitGraph + Start / StartPageRank (framework.cuh:991-1041,
 * 1151-1182, 1649-1658): the static solve from scratch. */
int cig_init(cig_handle *h);

/* Replaces del_edge -> update_tree_del (framework.cuh:1564-1586, 2752-2894):
 * the deletion phase of one batch (topology + incremental repair). */
int cig_delete_phase(cig_handle *h, const uint32_t *u, const uint32_t *v, uint64_t count,
                     cig_batch_stats *stats);

/* Replaces add_edge -> update_tree_add (framework.cuh:1397-1401, 2139-2348)
 * followed by the per-batch cache maintenance (samples/hybrid_sssp/
 * hybrid_sssp.cu:476-497). */
int cig_insert_phase(cig_handle *h, const uint32_t *u, const uint32_t *v, uint64_t count,
                     cig_batch_stats *stats);

/* One whole batch: deletion phase then insertion phase (PR: UpdatePageRank,
 * framework.cuh:1660-1704).  Host arrays: page-locked ones (cudaHostAlloc,
 * cudaHostRegister) are copied to the device directly, pageable ones through
 * the handle's pinned staging buffer. */
int cig_apply_batch(cig_handle *h, const uint32_t *del_u, const uint32_t *del_v, uint64_t nd,
                    const uint32_t *add_u, const uint32_t *add_v, uint64_t na, cig_batch_stats *stats);

/* Same with device-resident arrays. */
int cig_apply_batch_device(cig_handle *h, const uint32_t *del_u, const uint32_t *del_v, uint64_t nd,
                           const uint32_t *add_u, const uint32_t *add_v, uint64_t na,
                           cig_batch_stats *stats);

/* One update batch of device-resident arrays (for cig_apply_batches_device). */
typedef struct {
    const uint32_t *del_u;
    const uint32_t *del_v;
    uint64_t nd;
    const uint32_t *add_u;
    const uint32_t *add_v;
    uint64_t na;
} cig_update_batch;

/* The batched form of cig_apply_batch_device: `count` batches of any sizes
 * queued back to back with one host synchronisation at the end, so the
 * launches of batch i+1 overlap the execution of batch i.  Each batch is
 * applied completely (deletion phase, insertion phase, repair, cache
 * service) before the next, exactly as by `count` single calls.  stats[i]
 * (optional) gets batch i's counters and stage times; digests[i] (optional,
 * not for PR) the cig_value_digest of the values after batch i.  No
 * reference counterpart (the reference synchronises with the host every
 * round of every batch). */
int cig_apply_batches_device(cig_handle *h, const cig_update_batch *batches, uint32_t count,
                             cig_batch_stats *stats, uint64_t *digests);

/* Launch-shape autotuner: times the static solve on the loaded graph for
 * cooperative blocks per SM in {2, 4, 8} (the frontier tile of the persistent
 * closures) x hub-row split degree in {1024, 4096, 16384} (rows at least that
 * long are expanded by the whole grid in 1024-entry chunks), then single-
 * source BFS waves for push/pull divisors {off, 8, 16, 32, 64} (a wave of up
 * to 16 sources goes bottom-up while its frontier holds more than n/divisor
 * vertices), and keeps
 * the fastest for the handle.  Values are unchanged (the solve's values are
 * unique).  BFS/SSSP/CC.  No reference counterpart (the reference's
 * --lb_push/--lb_pull/--block_size hints have no effect). */
typedef struct {
    uint32_t blocks_per_sm;
    uint32_t split_degree;
    double best_ms;           /* static solve with the chosen shape */
    uint32_t candidates;
    uint32_t pull_divisor;    /* 0: BFS waves stay top-down */
} cig_tune_result;

int cig_autotune(cig_handle *h, cig_tune_result *res);

/* ---------------------------------------------------------------- serving
 * A request loop on one handle: update batches and BFS/SSSP queries are
 * submitted from any host thread and served in submission order (a query
 * sees every update submitted before it and none after).  Consecutive
 * queries of one kind are answered together as one bitmask wave (up to
 * max_wave sources: continuous batching), a wave overlaps the copy and key
 * sort of the update that follows it, and requests are admitted by their
 * device-memory footprint: an update larger than the budget allows is
 * applied as consecutive deletion chunks then insertion chunks (the same
 * rows and values as one batch).  While serving, the handle's other calls
 * return CIG_ERR_STATE; the serve calls may come from any threads and report
 * their errors through cig_last_error(NULL) of the calling thread.  Every
 * ticket's result is taken once (wait or poll) before cig_serve_stop.  No
 * reference counterpart (the reference samples replay a file of batches). */
typedef enum { CIG_REQ_UPDATE = 0, CIG_REQ_BFS = 1, CIG_REQ_SSSP = 2 } cig_request_kind;

typedef struct {
    int32_t kind;             /* cig_request_kind */
    uint32_t source;          /* queries: source vertex */
    const uint32_t *del_u;    /* updates: host arrays, copied by cig_serve_submit */
    const uint32_t *del_v;
    uint64_t nd;
    const uint32_t *add_u;
    const uint32_t *add_v;
    uint64_t na;
    uint32_t *out;            /* queries: n words of host memory for the depths/distances, or NULL */
} cig_request;

typedef struct {
    int32_t status;           /* CIG_OK or the request's error */
    uint32_t wave;            /* queries: sources answered in the same wave */
    uint64_t digest;          /* updates: cig_value_digest after the batch (not PR);
                                 queries: order-independent digest of the result row */
    double submit_ms;         /* times since cig_serve_start */
    double start_ms;
    double done_ms;
} cig_result;

typedef struct {
    uint64_t budget_bytes;    /* device bytes for per-request buffers (0: half of the free memory) */
    uint32_t max_wave;        /* sources per query wave, 1..64 (0: 64) */
    uint32_t max_pending;     /* submitted, unfinished requests before submit blocks (0: 4096) */
} cig_serve_options;

int cig_serve_start(cig_handle *h, const cig_serve_options *o);
int cig_serve_submit(cig_handle *h, const cig_request *r, uint64_t *ticket);
/* Block until request `ticket` is done and return its result (once). */
int cig_serve_wait(cig_handle *h, uint64_t ticket, cig_result *res);
/* Non-blocking: *done = 1 and the result when finished, else *done = 0. */
int cig_serve_poll(cig_handle *h, uint64_t ticket, cig_result *res, int *done);
/* Serve what is pending, then stop the loop; the handle is usable again. */
int cig_serve_stop(cig_handle *h);

/* Replaces GatherValue / GatherParent (framework.cuh:2896-2916): BFS depth,
 * SSSP distance or CC label; parents (0xFFFFFFFF for none). */
int cig_get_values(cig_handle *h, uint32_t *out);
int cig_get_parents(cig_handle *h, uint32_t *out);

/* PR ranks and signed residuals (GatherValue/GatherBuffer for hybrid_pr). */
int cig_get_pr(cig_handle *h, float *rank, float *residual);
int cig_get_pr64(cig_handle *h, double *rank, double *residual);

/* Order-independent 64-bit digest of the values computed on the device
 * (sum of a hash of (vertex, value) over reached vertices); 8 bytes cross the
 * host link.  The reference's ordered DistanceChecksum
 * (samples/hybrid_sssp/hybrid_sssp.cu:318-330) is computed by the tools on
 * the host from cig_get_values. */
int cig_value_digest(cig_handle *h, uint64_t *out);

/* The current adjacency (SourceLocalChunkStore::Descriptor/SlabData views,
 * source_local_chunk_store.h:395-410): row degrees, one row, or all rows. */
int cig_num_edges(cig_handle *h, uint64_t *m);
int cig_get_degrees(cig_handle *h, uint32_t *deg);
int cig_get_row(cig_handle *h, uint32_t v, uint32_t *out, uint32_t capacity, uint32_t *degree);
int cig_export_csr(cig_handle *h, uint64_t *xadj, uint32_t *adj);

int cig_graph_info_get(cig_handle *h, cig_graph_info *info);

/* Multi-source queries on the current graph (no reference counterpart): k BFS
 * depths or SSSP distances, k x n row-major, computed with 64-wide bitmask
 * frontiers.  Does not change the maintained state. */
int cig_query_bfs_multi(cig_handle *h, const uint32_t *sources, uint32_t k, uint32_t *out_depth);
int cig_query_sssp_multi(cig_handle *h, const uint32_t *sources, uint32_t k, uint32_t *out_dist);

typedef struct {
    double ms;                     /* device time of the whole query (all waves) */
    uint64_t edges_scanned;        /* adjacency entries read: edge-scans, the GTEPS numerator */
    uint64_t edges_scanned_cached; /* of which from HBM */
    uint64_t rows_expanded;
    uint64_t source_edges;         /* sum over expanded rows of (source bits x row length) */
    uint64_t rounds;
    uint64_t waves;
    uint64_t kernel_launches;
} cig_query_stats;

/* Device-memory form of the two calls above for callers that keep results
 * on the GPU: `algo` is CIG_BFS or CIG_SSSP, `sources` a host array of k
 * vertex ids, `out_device` a device array of k x n words.  Sources run in
 * waves of `width` (1..64): 64 is the batched bitmask form, 1 the plain
 * per-source form over the same kernels.  No reference counterpart (the
 * reference runs one source per engine run). */
int cig_query_multi_device(cig_handle *h, int algo, const uint32_t *sources, uint32_t k, uint32_t width,
                           uint32_t *out_device, cig_query_stats *stats);

/* Per-stage device time and work counters, measured with CUDA events on the
 * engine's own stream.  Replaces the reference's [ATTR] stage attribution
 * (samples/hybrid_sssp/hybrid_sssp.cu:496-512) and its NVTX marks
 * (include/utils/markers.h).  cig_profile_enable(h, 1) clears and starts the
 * accumulators; cig_profile_read copies CIG_STAGE_COUNT entries. */
enum {
    CIG_STAGE_GROUP = 0,  /* update keys, radix sort, source groups */
    CIG_STAGE_MUTATE = 1, /* forward rows: deletion/append/relocation, block allocation */
    CIG_STAGE_SEED = 2,   /* deletion and insertion seeds */
    CIG_STAGE_INVAL = 3,  /* invalidation closure */
    CIG_STAGE_PULL = 4,   /* reset + pull repair over in-rows + re-queue */
    CIG_STAGE_PUSH = 5,   /* push closure */
    CIG_STAGE_PR = 6,     /* PageRank amend + converge */
    CIG_STAGE_CACHE = 7,  /* edge-cache maintenance */
    CIG_STAGE_MUTATE_REV = 8, /* reverse (in-edge) rows */
    CIG_STAGE_ADD = 9,        /* forward rows, addition phase (MUTATE is then the deletion phase) */
    CIG_STAGE_ADD_REV = 10,   /* reverse rows, addition phase */
    CIG_STAGE_DEL_SCAN = 11,  /* deletion positions (inside MUTATE and MUTATE_REV): the flat scan
                                 and the position-index lookups; edges = row entries read,
                                 edges_cached = of which from HBM, hits = deletion keys */
    CIG_STAGE_INDEX = 12,     /* position-index rebuilds (inside ADD and ADD_REV) */
    CIG_STAGE_COUNT = 13
};

typedef struct {
    double ms;              /* summed device time */
    uint64_t launches;      /* timed regions */
    uint64_t edges;         /* adjacency entries read (traversal stages) */
    uint64_t edges_cached;  /* of which from HBM */
    uint64_t rows;          /* rows expanded */
    uint64_t hits;          /* relaxations / invalidations / residual pushes */
} cig_stage_profile;

int cig_profile_enable(cig_handle *h, int enable);
int cig_profile_read(cig_handle *h, cig_stage_profile *out, uint32_t count);

/* BFS depths over a CSR already in device memory, with no device
 * allocation.  No counterpart in the reference.  For callers that cannot
 * call cudaMalloc where they need a traversal: plugins and embedded runtimes
 * whose device memory belongs to a host framework with its own allocator
 * (raw cudaMalloc/cudaFree there bypass its accounting and can fail once the
 * pool holds the memory), and latency-bound loops that must not take the
 * device-wide synchronisation cudaFree implies.
 *   xadj[n+1] (uint64) and adj[xadj[n]] (uint32): device CSR, rows in any
 *   order; both must be non-null (an edge-free graph passes a dummy adj);
 *   depth[n] (uint32): device output, 0xFFFFFFFF for unreached vertices;
 *   stream: a cudaStream_t (NULL = the legacy default stream).  The call is
 *   blocking: it copies the device error word to the host and synchronises
 *   `stream` before it returns.
 * All scratch lives in a fixed __device__ array sized for at most
 * CIG_NOALLOC_MAX_VERTICES vertices (about 3 MiB, held by every GPU that
 * loads the library until the process exits); larger n is rejected with
 * CIG_ERR_ARG.  The first call on a device looks up that array's device
 * address (set-up), so make the first call on each device before any stream
 * capture.  Calls on one device share the array and each starts by clearing
 * what must start at zero: calls that overlap on the GPU (two host threads,
 * two streams) race and must be serialised by the caller.
 * Errors: the message is available from cig_last_error(NULL). */
#define CIG_NOALLOC_MAX_VERTICES (1u << 18)
int cig_bfs_csr_noalloc(const uint64_t *xadj, const uint32_t *adj, uint32_t n, uint32_t source, uint32_t *depth,
                        void *stream);

/* Library version string. */
const char *cig_version(void);

/* SASS architecture the engine's kernels were compiled for, as
 * cudaFuncGetAttributes reports it on the current device (100 = sm_100a),
 * and whether this is the bounds-checked build (libcig_bc.so).  No
 * reference counterpart. */
int cig_build_info(int *binary_version, int *bounds_checked);

#ifdef __cplusplus
}
#endif
#endif
