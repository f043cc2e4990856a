/*
 * oracle.h - CPU oracle for the incremental streaming-graph path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libcig, the hybrid_*
 * command-line tools) links or calls this code; only tests/, the smoke check
 * and the benchmark's CPU-baseline arm use it, as the checker.
 *
 * It restates, in plain C, the reference's semantics for:
 *   - the source-local chunk-store row mutation
 *     (include/groute/graphs/source_local_chunk_store.h:670-848,
 *      include/framework/effective_update_batch.h:33-115);
 *   - the --check algorithms of the four samples
 *     (samples/hybrid_sssp/hybrid_sssp.cu:211-330,
 *      samples/hybrid_sssp/hybrid_sssp_host.cu:34-63 with the +1 of
 *      include/framework/variants/api.cuh:26-28,
 *      samples/hybrid_cc/hybrid_cc_host.cu:8-32,
 *      samples/hybrid_pr/hybrid_pr_host.cu:9-56).
 *
 * Parity is pinned by tests/test_oracle_pin.py against the reference's own
 * SourceLocalChunkStore, CCCheck and PageRankCheck compiled from the
 * reference sources (oracle/build_ref.py -> oracle/_ref/).
 */
#ifndef CIG_ORACLE_H
#define CIG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OG_INF 0xFFFFFFFFu

enum { OG_BFS = 0, OG_SSSP = 1, OG_CC = 2, OG_SSSP_U255 = 3 };

typedef struct og_graph og_graph;

og_graph *og_create(uint32_t n, const uint64_t *xadj, const uint32_t *adj);
void og_free(og_graph *g);
uint32_t og_n(const og_graph *g);
uint64_t og_m(const og_graph *g);
uint32_t og_degree(const og_graph *g, uint32_t v);
const uint32_t *og_row(const og_graph *g, uint32_t v);
void og_export(const og_graph *g, uint64_t *xadj, uint32_t *adj);

/* Deletion phase: each request removes the first remaining occurrence. */
uint64_t og_delete(og_graph *g, const uint32_t *u, const uint32_t *v, uint64_t m);
/* Addition phase: append in input order.  Returns the invalid count. */
uint64_t og_add(og_graph *g, const uint32_t *u, const uint32_t *v, uint64_t m);

uint32_t og_weight(int mode, uint32_t u, uint32_t v);

/* From-scratch recompute; parent may be NULL. */
void og_sssp_fifo(const og_graph *g, uint32_t src, int mode, uint32_t *dist, uint32_t *parent);
void og_sssp_dial(const og_graph *g, uint32_t src, int mode, uint32_t *dist);
void og_cc(const og_graph *g, uint32_t *label);
int og_pr(const og_graph *g, double tol_per_vertex, int max_rounds, double *x);

/* out = {relaxable_edges, missing_tight_witnesses} */
void og_bellman_check(const og_graph *g, const uint32_t *dist, uint32_t src, int mode, uint64_t *out);
/* out = {invalid_vertices, missing_parent_edges, wrong_parent_distances} */
void og_parent_check(const og_graph *g, const uint32_t *dist, const uint32_t *parent, uint32_t src,
                     int mode, uint64_t *out);
uint64_t og_checksum(const uint32_t *dist, uint32_t n);
uint64_t og_row_hash(const og_graph *g, uint32_t v);

/* PageRankCheck restated: out = {ok, l1, bound, max_error, invariant_l1, max_residual}. */
void og_pr_check(const og_graph *g, const float *rank, const float *residual, double epsilon,
                 double *out);

#ifdef __cplusplus
}
#endif
#endif
