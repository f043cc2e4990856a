/*
 * oracle.c - CPU oracle (test infrastructure only; see oracle.h).
 *
 * Plain C restatement of the reference's row-mutation semantics and of the
 * --check algorithms of its four samples.  Each function cites the reference
 * lines it follows.  Nothing here is on the product path.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

struct og_graph {
    uint32_t n;
    uint64_t m;
    uint32_t *deg;
    uint32_t *cap;
    uint32_t **rows;
};

static int reserve_row(og_graph *g, uint32_t v, uint32_t need) {
    if (need <= g->cap[v]) return 0;
    uint32_t cap = g->cap[v] ? g->cap[v] : 4;
    while (cap < need) cap *= 2;
    uint32_t *row = (uint32_t *)realloc(g->rows[v], (size_t)cap * sizeof(uint32_t));
    if (!row) return -1;
    g->rows[v] = row;
    g->cap[v] = cap;
    return 0;
}

/* Load in row order, as LoadSource does (source_local_chunk_store.h:129-147). */
og_graph *og_create(uint32_t n, const uint64_t *xadj, const uint32_t *adj) {
    og_graph *g = (og_graph *)calloc(1, sizeof(og_graph));
    if (!g) return NULL;
    g->n = n;
    g->deg = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    g->cap = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    g->rows = (uint32_t **)calloc(n ? n : 1, sizeof(uint32_t *));
    if (!g->deg || !g->cap || !g->rows) {
        og_free(g);
        return NULL;
    }
    for (uint32_t v = 0; v < n; ++v) {
        const uint64_t d = xadj[v + 1] - xadj[v];
        if (d == 0) continue;
        if (reserve_row(g, v, (uint32_t)d)) {
            og_free(g);
            return NULL;
        }
        memcpy(g->rows[v], adj + xadj[v], (size_t)d * sizeof(uint32_t));
        g->deg[v] = (uint32_t)d;
        g->m += d;
    }
    return g;
}

void og_free(og_graph *g) {
    if (!g) return;
    if (g->rows)
        for (uint32_t v = 0; v < g->n; ++v) free(g->rows[v]);
    free(g->rows);
    free(g->deg);
    free(g->cap);
    free(g);
}

uint32_t og_n(const og_graph *g) { return g->n; }
uint64_t og_m(const og_graph *g) { return g->m; }
uint32_t og_degree(const og_graph *g, uint32_t v) { return v < g->n ? g->deg[v] : 0; }
const uint32_t *og_row(const og_graph *g, uint32_t v) { return v < g->n ? g->rows[v] : NULL; }

void og_export(const og_graph *g, uint64_t *xadj, uint32_t *adj) {
    xadj[0] = 0;
    for (uint32_t v = 0; v < g->n; ++v) {
        xadj[v + 1] = xadj[v] + g->deg[v];
        if (g->deg[v]) memcpy(adj + xadj[v], g->rows[v], (size_t)g->deg[v] * sizeof(uint32_t));
    }
}

/*
 * Deletion phase.  The reference groups a batch by source (stable radix sort,
 * effective_update_batch.h:33-87), counts how often each destination is
 * requested, and removes the first min(requested, present) occurrences while
 * keeping the order of the survivors (BuildDeletionPlan / ShouldDelete /
 * CompactSourceInPlace, source_local_chunk_store.h:670-773).  Removing the
 * first remaining occurrence once per request, in any order, yields the same
 * row.  Requests whose source is out of range, or whose destination is not
 * present, are ignored and counted as missing (:258-262).
 */
uint64_t og_delete(og_graph *g, const uint32_t *u, const uint32_t *v, uint64_t m) {
    uint64_t missing = 0;
    for (uint64_t i = 0; i < m; ++i) {
        const uint32_t s = u[i];
        if (s >= g->n) {
            ++missing;
            continue;
        }
        uint32_t *row = g->rows[s];
        const uint32_t d = g->deg[s];
        uint32_t pos = 0;
        while (pos < d && row[pos] != v[i]) ++pos;
        if (pos == d) {
            ++missing;
            continue;
        }
        memmove(row + pos, row + pos + 1, (size_t)(d - pos - 1) * sizeof(uint32_t));
        g->deg[s] = d - 1;
        g->m -= 1;
    }
    return missing;
}

/*
 * Addition phase: destinations are appended in input order
 * (CompactSourceInPlace / RewriteSourceToNewBlock append `additions` after the
 * survivors, source_local_chunk_store.h:755-761, 812-818).  Out-of-range
 * sources are ignored as invalid additions (:258-262).  Out-of-range
 * destinations are also rejected here; the reference would store them and
 * later index past its vertex arrays.
 */
uint64_t og_add(og_graph *g, const uint32_t *u, const uint32_t *v, uint64_t m) {
    uint64_t invalid = 0;
    for (uint64_t i = 0; i < m; ++i) {
        const uint32_t s = u[i];
        if (s >= g->n || v[i] >= g->n) {
            ++invalid;
            continue;
        }
        if (reserve_row(g, s, g->deg[s] + 1)) {
            ++invalid;
            continue;
        }
        g->rows[s][g->deg[s]++] = v[i];
        g->m += 1;
    }
    return invalid;
}

/* Edge weights: BFS 1 (samples/hybrid_bfs/hybrid_bfs.cu:41-47), SSSP
 * (src+dst)%128+1 (include/framework/variants/api.cuh:26-28), CC 0
 * (samples/hybrid_cc/hybrid_cc.cu:51-57). */
uint32_t og_weight(int mode, uint32_t u, uint32_t v) {
    if (mode == OG_BFS) return 1;
    if (mode == OG_CC) return 0;
    if (mode == OG_SSSP_U255) {
        /* the extension's weights in [1, 255]: lowbias32 (C. Wellons) of a
         * linear mix of the ids, as the engine's weight_u255 */
        uint32_t x = u * 0x9E3779B1u + v * 0x85EBCA77u;
        x ^= x >> 16;
        x *= 0x7FEB352Du;
        x ^= x >> 15;
        x *= 0x846CA68Bu;
        x ^= x >> 16;
        return 1u + x % 255u;
    }
    return (uint32_t)(((uint64_t)u + v) % 128 + 1);
}

/*
 * FIFO label-correcting recompute, as SSSPHostNaive_p
 * (samples/hybrid_sssp/hybrid_sssp_host.cu:63-93) but with the +1 weight the
 * engine actually uses (api.cuh:26-28).  The queue may hold duplicates.
 */
void og_sssp_fifo(const og_graph *g, uint32_t src, int mode, uint32_t *dist, uint32_t *parent) {
    const uint32_t n = g->n;
    for (uint32_t v = 0; v < n; ++v) {
        dist[v] = OG_INF;
        if (parent) parent[v] = OG_INF;
    }
    if (src >= n) return;
    size_t cap = (size_t)n + 16, head = 0, tail = 0, count = 0;
    uint32_t *queue = (uint32_t *)malloc(cap * sizeof(uint32_t));
    if (!queue) return;
    dist[src] = 0;
    queue[tail++] = src;
    count = 1;
    while (count) {
        const uint32_t x = queue[head];
        head = (head + 1) % cap;
        --count;
        const uint64_t dx = dist[x];
        for (uint32_t k = 0; k < g->deg[x]; ++k) {
            const uint32_t y = g->rows[x][k];
            const uint64_t nd = dx + og_weight(mode, x, y);
            if (nd < dist[y]) {
                dist[y] = (uint32_t)nd;
                if (parent) parent[y] = x;
                if (count == cap) {
                    /* grow the ring buffer */
                    size_t ncap = cap * 2;
                    uint32_t *nq = (uint32_t *)malloc(ncap * sizeof(uint32_t));
                    if (!nq) {
                        free(queue);
                        return;
                    }
                    for (size_t i = 0; i < count; ++i) nq[i] = queue[(head + i) % cap];
                    free(queue);
                    queue = nq;
                    head = 0;
                    tail = count;
                    cap = ncap;
                }
                queue[tail] = y;
                tail = (tail + 1) % cap;
                ++count;
            }
        }
    }
    free(queue);
}

/*
 * Independent cross-check: Dial's bucket-queue Dijkstra (weights are at most
 * 255 < NB buckets), so that two unrelated algorithms agree on every distance.
 */
void og_sssp_dial(const og_graph *g, uint32_t src, int mode, uint32_t *dist) {
    const uint32_t n = g->n;
    for (uint32_t v = 0; v < n; ++v) dist[v] = OG_INF;
    if (src >= n) return;
    enum { NB = 256 };
    size_t *cnt = (size_t *)calloc(NB, sizeof(size_t));
    size_t *capb = (size_t *)calloc(NB, sizeof(size_t));
    uint32_t **bucket = (uint32_t **)calloc(NB, sizeof(uint32_t *));
    if (!cnt || !capb || !bucket) goto done;
    dist[src] = 0;
    bucket[0] = (uint32_t *)malloc(16 * sizeof(uint32_t));
    capb[0] = 16;
    bucket[0][cnt[0]++] = src;
    {
        uint64_t cur = 0;
        size_t pending = 1;
        while (pending) {
            const size_t b = (size_t)(cur % NB);
            while (cnt[b]) {
                const uint32_t x = bucket[b][--cnt[b]];
                --pending;
                if (dist[x] != cur) continue; /* stale entry */
                for (uint32_t k = 0; k < g->deg[x]; ++k) {
                    const uint32_t y = g->rows[x][k];
                    const uint64_t nd = cur + og_weight(mode, x, y);
                    if (nd < dist[y]) {
                        dist[y] = (uint32_t)nd;
                        const size_t nb = (size_t)(nd % NB);
                        if (cnt[nb] == capb[nb]) {
                            size_t nc = capb[nb] ? capb[nb] * 2 : 16;
                            uint32_t *p = (uint32_t *)realloc(bucket[nb], nc * sizeof(uint32_t));
                            if (!p) goto done;
                            bucket[nb] = p;
                            capb[nb] = nc;
                        }
                        bucket[nb][cnt[nb]++] = y;
                        ++pending;
                    }
                }
            }
            ++cur;
        }
    }
done:
    if (bucket)
        for (int i = 0; i < NB; ++i) free(bucket[i]);
    free(bucket);
    free(cnt);
    free(capb);
}

/*
 * Directed minimum-label propagation: label[v] = the smallest id from which v
 * is reachable.  Restates CCCheck (samples/hybrid_cc/hybrid_cc_host.cu:8-32):
 * seeds in ascending order, depth-first flood of unlabelled vertices.
 */
void og_cc(const og_graph *g, uint32_t *label) {
    const uint32_t n = g->n;
    for (uint32_t v = 0; v < n; ++v) label[v] = OG_INF;
    uint32_t *stack = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    if (!stack) return;
    for (uint32_t seed = 0; seed < n; ++seed) {
        if (label[seed] != OG_INF) continue;
        label[seed] = seed;
        size_t top = 0;
        stack[top++] = seed;
        while (top) {
            const uint32_t x = stack[--top];
            for (uint32_t k = 0; k < g->deg[x]; ++k) {
                const uint32_t y = g->rows[x][k];
                if (label[y] != OG_INF) continue;
                label[y] = seed;
                stack[top++] = y;
            }
        }
    }
    free(stack);
}

/*
 * Unnormalised PageRank x = 0.15 + 0.85 * sum_{u->v} x[u]/outdeg(u), parallel
 * edges counted, dangling vertices send nothing.  FP64 Jacobi from x = 0 as in
 * PageRankCheck (samples/hybrid_pr/hybrid_pr_host.cu:15-33); stops when the L1
 * change is <= tol_per_vertex * n.  Returns 1 when converged.
 */
int og_pr(const og_graph *g, double tol_per_vertex, int max_rounds, double *x) {
    const uint32_t n = g->n;
    double *next = (double *)malloc(((size_t)n + 1) * sizeof(double));
    if (!next) return 0;
    for (uint32_t v = 0; v < n; ++v) x[v] = 0.0;
    int converged = 0;
    for (int round = 0; round < max_rounds; ++round) {
        for (uint32_t v = 0; v < n; ++v) next[v] = 0.15;
        for (uint32_t s = 0; s < n; ++s) {
            if (!g->deg[s]) continue;
            const double c = 0.85 * x[s] / g->deg[s];
            for (uint32_t k = 0; k < g->deg[s]; ++k) next[g->rows[s][k]] += c;
        }
        double delta = 0;
        for (uint32_t v = 0; v < n; ++v) {
            delta += fabs(next[v] - x[v]);
            x[v] = next[v];
        }
        if (delta <= tol_per_vertex * (n ? n : 1)) {
            converged = 1;
            break;
        }
    }
    free(next);
    return converged;
}

/*
 * Bellman certificate, restating CheckBellmanRelaxed
 * (samples/hybrid_sssp/hybrid_sssp.cu:211-264): no edge may be relaxable and
 * every finite non-source vertex needs a tight in-edge.
 */
void og_bellman_check(const og_graph *g, const uint32_t *dist, uint32_t src, int mode, uint64_t *out) {
    const uint32_t n = g->n;
    uint8_t *tight = (uint8_t *)calloc(n ? n : 1, 1);
    uint64_t relaxable = 0, missing = 0;
    if (!tight) return;
    if (src < n) tight[src] = 1;
    for (uint32_t s = 0; s < n; ++s) {
        if (dist[s] == OG_INF) continue;
        for (uint32_t k = 0; k < g->deg[s]; ++k) {
            const uint32_t d = g->rows[s][k];
            if (d >= n) continue;
            const uint64_t cand = (uint64_t)dist[s] + og_weight(mode, s, d);
            if (dist[d] != OG_INF && cand == dist[d]) tight[d] = 1;
            if (cand < dist[d]) ++relaxable;
        }
    }
    for (uint32_t v = 0; v < n; ++v)
        if (dist[v] != OG_INF && !tight[v]) ++missing;
    free(tight);
    out[0] = relaxable;
    out[1] = missing;
}

/* Parent witnesses, restating CheckParentWitness (hybrid_sssp.cu:266-316). */
void og_parent_check(const og_graph *g, const uint32_t *dist, const uint32_t *parent, uint32_t src,
                     int mode, uint64_t *out) {
    uint64_t invalid = 0, missing_edge = 0, wrong = 0;
    for (uint32_t v = 0; v < g->n; ++v) {
        if (v == src || dist[v] == OG_INF) continue;
        const uint32_t p = parent[v];
        int valid = p < g->n && dist[p] != OG_INF;
        if (valid) {
            int exists = 0;
            for (uint32_t k = 0; k < g->deg[p]; ++k)
                if (g->rows[p][k] == v) {
                    exists = 1;
                    break;
                }
            const int matches = (uint64_t)dist[p] + og_weight(mode, p, v) == dist[v];
            if (!exists)
                ++missing_edge;
            else if (!matches)
                ++wrong;
            valid = exists && matches;
        }
        if (!valid) ++invalid;
    }
    out[0] = invalid;
    out[1] = missing_edge;
    out[2] = wrong;
}

/* DistanceChecksum / LabelChecksum (hybrid_sssp.cu:318-330, hybrid_cc.cu:188-200). */
uint64_t og_checksum(const uint32_t *dist, uint32_t n) {
    uint64_t h = 1469598103934665603ull;
    for (uint32_t v = 0; v < n; ++v) {
        if (dist[v] == OG_INF) continue;
        h ^= (uint64_t)v + 0x9e3779b97f4a7c15ull + ((uint64_t)dist[v] << 6) + ((uint64_t)dist[v] >> 2);
        h *= 1099511628211ull;
    }
    return h;
}

/* OrderedHash (source_local_chunk_store.h:378-392). */
uint64_t og_row_hash(const og_graph *g, uint32_t v) {
    uint64_t h = 1469598103934665603ULL;
    const uint32_t d = og_degree(g, v);
    for (uint32_t k = 0; k < d; ++k) {
        h ^= (uint64_t)g->rows[v][k];
        h *= 1099511628211ULL;
    }
    h ^= (uint64_t)d;
    h *= 1099511628211ULL;
    return h;
}

/*
 * PageRankCheck restated (samples/hybrid_pr/hybrid_pr_host.cu:9-56): FP64
 * Jacobi reference (<= 10000 rounds, tolerance 1e-12 n), L1 error bound
 * (n eps + roundoff)/0.15, residual invariant |P x + 0.15 - x - r|_1 <=
 * roundoff and max|r| <= eps.
 */
void og_pr_check(const og_graph *g, const float *rank, const float *residual, double epsilon,
                 double *out) {
    const uint32_t n = g->n;
    double *ref = (double *)malloc(((size_t)n + 1) * sizeof(double));
    double *next = (double *)malloc(((size_t)n + 1) * sizeof(double));
    if (!ref || !next) {
        free(ref);
        free(next);
        out[0] = 0;
        return;
    }
    const int converged = og_pr(g, 1e-12, 10000, ref);
    for (uint32_t v = 0; v < n; ++v) next[v] = 0.15;
    for (uint32_t s = 0; s < n; ++s) {
        if (!g->deg[s]) continue;
        const double c = 0.85 * (double)rank[s] / g->deg[s];
        for (uint32_t k = 0; k < g->deg[s]; ++k) next[g->rows[s][k]] += c;
    }
    double l1 = 0, defect = 0, max_res = 0, max_err = 0, mass = 0;
    int finite = 1;
    for (uint32_t v = 0; v < n; ++v) {
        finite &= isfinite(rank[v]) && isfinite(residual[v]) && rank[v] >= -epsilon;
        const double err = fabs((double)rank[v] - ref[v]);
        l1 += err;
        if (err > max_err) max_err = err;
        defect += fabs(next[v] - (double)rank[v] - (double)residual[v]);
        if (fabs((double)residual[v]) > max_res) max_res = fabs((double)residual[v]);
        mass += fabs(ref[v]);
    }
    const double roundoff = 64 * (double)FLT_EPSILON * (mass > 1.0 ? mass : 1.0);
    const double bound = (n * epsilon + roundoff) / 0.15;
    const int ok = finite && converged && l1 <= bound && defect <= roundoff &&
                   max_res <= (double)(float)epsilon;
    out[0] = ok;
    out[1] = l1;
    out[2] = bound;
    out[3] = max_err;
    out[4] = defect;
    out[5] = max_res;
    free(ref);
    free(next);
}
