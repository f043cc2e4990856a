// ref_shim.cpp - C entry points over the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/build.py against the
// reference headers where they lie (include/groute/graphs/
// source_local_chunk_store.h, include/framework/effective_update_batch.h)
// together with the reference's own host checkers
// (samples/hybrid_cc/hybrid_cc_host.cu, samples/hybrid_pr/hybrid_pr_host.cu),
// into oracle/_ref/libcigref.so.  Tests use it to pin the plain-C oracle
// (oracle/oracle.c) and the benchmark's CPU arm uses it as the reference's
// batch-maintenance implementation.  No reference source is copied here: this
// file only calls the reference's classes and functions.
#include <groute/graphs/source_local_chunk_store.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <vector>

#include "hybrid_cc_common.h"
#undef IDENTITY_ELEMENT
#include "hybrid_pr_common.h"

using sepgraph::topology::ChunkArenaOptions;
using sepgraph::topology::GroupedUpdateBatch;
using sepgraph::topology::IgnoreEffectiveUpdates;
using sepgraph::topology::SourceLocalChunkStore;
using sepgraph::topology::TopologyMutationBatch;
using sepgraph::topology::UpdatePhase;

struct ref_store {
    SourceLocalChunkStore *store = nullptr;
    uint32_t n = 0;
};

extern "C" {

// Capacity follows LoadGraph (include/framework/framework.cuh:886-892):
// sum of pow2 row blocks plus max(sum/8, 2^20) headroom; host (unpinned) slabs.
ref_store *ref_store_create(uint32_t n, const uint64_t *xadj, const uint32_t *adj, uint32_t workers,
                            uint64_t extra_capacity) {
    try {
        uint64_t required = 0;
        for (uint32_t v = 0; v < n; ++v)
            required += SourceLocalChunkStore::RequiredChunkCapacity(xadj[v + 1] - xadj[v]);
        ChunkArenaOptions options;
        options.capacity_edges = required + std::max<uint64_t>(required / 8, 1ULL << 20) + extra_capacity;
        options.slab_capacity_edges = 1ULL << 24;
        options.minimum_chunk_edges = 4;
        options.pinned = false;
        options.mutation_workers = workers;
        ref_store *r = new ref_store();
        r->n = n;
        r->store = new SourceLocalChunkStore(n, options);
        for (uint32_t v = 0; v < n; ++v)
            r->store->LoadSource(v, std::vector<index_t>(adj + xadj[v], adj + xadj[v + 1]));
        r->store->FinalizeLoad(xadj[n]);
        return r;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_store_create: %s\n", e.what());
        return nullptr;
    }
}

void ref_store_free(ref_store *r) {
    if (!r) return;
    delete r->store;
    delete r;
}

// One update batch as the engine applies it: reclaim retired blocks of the
// published epoch, deletion phase, addition phase, publish
// (framework.cuh:1564-1586 del_edge, :1397-1401 add_edge).
// out = {missing_deletes, invalid_additions, changed_sources_delete, changed_sources_add}
int ref_store_apply(ref_store *r, const uint32_t *du, const uint32_t *dv, uint64_t nd, const uint32_t *au,
                    const uint32_t *av, uint64_t na, uint64_t *out) {
    try {
        r->store->ReclaimThrough(r->store->PublishedEpoch());
        TopologyMutationBatch dels, adds;
        dels.deletions.reserve(nd);
        adds.additions.reserve(na);
        for (uint64_t i = 0; i < nd; ++i) dels.deletions.push_back({du[i], dv[i]});
        for (uint64_t i = 0; i < na; ++i) adds.additions.push_back({au[i], av[i]});
        IgnoreEffectiveUpdates observer;
        GroupedUpdateBatch gd(dels);
        const auto md = r->store->ApplyGroupedPhase(gd, UpdatePhase::Delete, observer);
        GroupedUpdateBatch ga(adds);
        const auto ma = r->store->ApplyGroupedPhase(ga, UpdatePhase::Add, observer);
        r->store->Publish();
        if (out) {
            out[0] = md.missing_deletes;
            out[1] = ma.invalid_additions;
            out[2] = md.changed_sources;
            out[3] = ma.changed_sources;
        }
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_store_apply: %s\n", e.what());
        return -1;
    }
}

uint64_t ref_store_edges(const ref_store *r) { return r->store->EdgeCount(); }

uint32_t ref_store_degree(const ref_store *r, uint32_t v) { return r->store->Descriptor(v).degree; }

void ref_store_export(const ref_store *r, uint64_t *xadj, uint32_t *adj) {
    xadj[0] = 0;
    for (uint32_t v = 0; v < r->n; ++v) {
        const auto &d = r->store->Descriptor(v);
        xadj[v + 1] = xadj[v] + d.degree;
        if (d.degree) {
            const index_t *row = r->store->SlabData(d.slab_id) + d.index;
            std::copy(row, row + d.degree, adj + xadj[v]);
        }
    }
}

uint64_t ref_store_row_hash(const ref_store *r, uint32_t v) { return r->store->OrderedHash(v); }

// The reference's own CC checker (samples/hybrid_cc/hybrid_cc_host.cu:8-32):
// returns the number of vertices whose label differs from its flood fill.
uint64_t ref_cc_check(const ref_store *r, const uint32_t *labels) {
    std::vector<label_t> l(labels, labels + r->n);
    return CCCheck(*r->store, l);
}

// The reference's own PR checker (samples/hybrid_pr/hybrid_pr_host.cu:9-56).
int ref_pr_check(const ref_store *r, const float *ranks, const float *residual, double epsilon) {
    std::vector<rank_t> x(ranks, ranks + r->n), res(residual, residual + r->n);
    return PageRankCheck(*r->store, x, res, epsilon, "oracle", -1) ? 1 : 0;
}

}  // extern "C"
