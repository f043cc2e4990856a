/*
 * cig_gen.h - seeded synthetic inputs for the incremental streaming-graph path.
 *
 * The reference ships no graphs and no update streams; its own generator
 * (include/framework/generator.h:80-111, GAP-style R-MAT with a mt19937
 * shuffle) is not compiled into any binary.  This header declares the
 * replacement used by the tests, the benchmark and the data-preparation
 * helpers:
 *
 *   - R-MAT edges with quadrant probabilities a/b/c/d, `scale` levels per
 *     edge and a counter-based RNG keyed by (seed, edge index), so that the
 *     output does not depend on the number of threads;
 *   - a seeded bijective vertex-id permutation that keeps id 0 fixed (id 0 is
 *     the R-MAT hub before permutation, so "source 0" reaches the giant
 *     component, as in an unpermuted R-MAT);
 *   - self-loops and duplicate (u,v) pairs removed, rows sorted by
 *     destination; "symmetric" adds (v,u) for every (u,v) before the dedup;
 *   - update batches: deletions drawn uniformly without replacement from the
 *     current edge set, insertions drawn uniformly from the pairs u != v that
 *     are not in the current edge set (after this batch's deletions).  In
 *     symmetric mode every update is emitted as the pair (u,v),(v,u).
 *
 * All functions return 0 on success and a negative code on failure.
 * Buffers passed in are caller-owned.
 */
#ifndef CIG_GEN_H
#define CIG_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cig_gen_graph cig_gen_graph;

/* Generate a graph.  a+b+c must be < 1; d = 1-a-b-c. */
int cig_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                 uint64_t seed, int symmetric, int permute, cig_gen_graph **out);

/* Number of vertices and (deduplicated) directed edges. */
int cig_gen_sizes(const cig_gen_graph *g, uint32_t *n, uint64_t *m);

/* Copy the CSR out: xadj[n+1], adj[m]. */
int cig_gen_copy_csr(const cig_gen_graph *g, uint64_t *xadj, uint32_t *adj);

/* Borrow the CSR arrays (valid until cig_gen_free). */
int cig_gen_borrow_csr(const cig_gen_graph *g, const uint64_t **xadj, const uint32_t **adj);

/*
 * Generate `nbatches` update batches against the evolving edge set.  Batch i
 * has del_sizes[i] deletions and add_sizes[i] insertions (directed records;
 * in symmetric mode both must be even).  Output arrays are the concatenation
 * of all batches in order and must hold sum(del_sizes) / sum(add_sizes)
 * entries.  The generator state of `g` is not modified.
 */
int cig_gen_updates(const cig_gen_graph *g, uint32_t nbatches, const uint64_t *del_sizes,
                    const uint64_t *add_sizes, uint64_t seed, int symmetric,
                    uint32_t *del_u, uint32_t *del_v, uint32_t *add_u, uint32_t *add_v);

void cig_gen_free(cig_gen_graph *g);

/* Threads used by the generator (OpenMP). */
int cig_gen_threads(void);

#ifdef __cplusplus
}
#endif
#endif
