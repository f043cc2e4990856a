// engine.cu - libcig: host engine and C ABI (include/cig.h).
//
// One handle = one graph on one GPU.  The forward adjacency is a
// power-of-two block arena in pinned, mapped host memory; an HBM edge cache
// holds whole 64 KiB segments of it under the --cache budget, selected by a
// device segment table.  A device-only reverse arena holds in-edges for
// deletion repair.  Every phase of a batch is a chain of asynchronous
// launches on one stream (including the cooperative closure kernels); the
// host synchronises once per API call.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/cig.h"
#include "cache.cuh"
#include "common.cuh"
#include "expand.cuh"
#include "mutate.cuh"
#include "pr.cuh"
#include "query.cuh"
#include "traverse.cuh"

using namespace cig;

namespace {

struct CigError : std::runtime_error {
    int code;
    CigError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CK(expr)                                                                                          \
    do {                                                                                                  \
        const cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess)                                                                            \
            throw CigError(CIG_ERR_DEVICE, std::string(#expr) + ": " + cudaGetErrorString(e_) + " (line " + \
                                               std::to_string(__LINE__) + ")");                           \
    } while (0)

template <class T>
void dmalloc(T *&p, size_t count) {
    p = nullptr;
    if (count == 0) count = 1;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CigError(CIG_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                          " bytes failed: " + cudaGetErrorString(e));
    }
}

template <class T>
void dfree(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

inline uint32_t host_class(uint64_t deg) {
    if (deg == 0) return 0;
    if (deg <= (1u << kMinClass)) return kMinClass;
    uint32_t c = 0;
    while ((1ull << c) < deg) ++c;
    return c;
}

// Initial arena layout: one region per class (largest classes first, each
// region segment aligned), rows in vertex order inside a region.
// Rows of at most 2^kSmallRowClass entries are "small" (one warp expands
// them; larger rows take the whole block): most vertices, and most rows a
// traversal reads, each read a short dependent access.
constexpr uint32_t kSmallRowClass = 8;

struct Layout {
    std::vector<RowDesc> desc;
    unsigned long long cur_next[kNumClasses] = {};
    unsigned long long cur_end[kNumClasses] = {};
    uint64_t used_segs = 0;
    uint64_t small_segs = 0;  // the last segments, which hold the small rows
};

Layout plan_layout(uint32_t n, const uint32_t *deg) {
    Layout L;
    L.desc.assign(n, RowDesc{0, 0, 0});
    uint64_t count[kNumClasses] = {};
    for (uint32_t v = 0; v < n; ++v) count[host_class(deg[v])] += deg[v] ? 1 : 0;
    uint64_t start[kNumClasses] = {};
    uint64_t seg = 0;
    for (int c = kNumClasses - 1; c >= static_cast<int>(kMinClass); --c) {
        if (!count[c]) continue;
        start[c] = seg << kSegShift;
        uint64_t segs;
        if (static_cast<uint32_t>(c) <= kSegShift) {
            const uint64_t edges = count[c] << c;
            segs = (edges + kSegEdges - 1) >> kSegShift;
            L.cur_next[c] = start[c] + edges;
            L.cur_end[c] = (seg + segs) << kSegShift;
        } else {
            segs = count[c] << (c - kSegShift);
        }
        seg += segs;
        if (static_cast<uint32_t>(c) <= kSmallRowClass) L.small_segs += segs;
    }
    L.used_segs = seg;
    uint64_t cursor[kNumClasses];
    std::memcpy(cursor, start, sizeof(start));
    for (uint32_t v = 0; v < n; ++v) {
        if (!deg[v]) continue;
        const uint32_t c = host_class(deg[v]);
        L.desc[v] = RowDesc{cursor[c], deg[v], rd_meta(c, 0)};
        cursor[c] += 1ull << c;
    }
    return L;
}

unsigned hw_threads() {
    const unsigned t = std::thread::hardware_concurrency();
    return t ? std::min(t, 64u) : 4u;
}

template <class F>
void parallel_for(uint64_t n, F f) {
    const unsigned t = hw_threads();
    if (n < 65536 || t <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const uint64_t chunk = (n + t - 1) / t;
    for (unsigned i = 0; i < t; ++i) {
        const uint64_t b = i * chunk, e = std::min<uint64_t>(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([=] { f(b, e); });
    }
    for (auto &th : pool) th.join();
}

__global__ void count_indeg(const uint32_t *adj, uint64_t m, uint32_t *indeg) {
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < m;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        atomicAdd(indeg + adj[e], 1u);
}

// One warp per source row: append the source to every destination's in-row.
__global__ void fill_reverse(const uint64_t *xadj, const uint32_t *adj, uint32_t n, const RowDesc *rdesc,
                             uint32_t *cursor, uint32_t *rarena) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        for (uint64_t e = xadj[u] + lane_id(); e < xadj[u + 1]; e += 32) {
            const uint32_t v = adj[e];
            const uint32_t pos = atomicAdd(cursor + v, 1u);
            rarena[rdesc[v].off + pos] = u;
        }
    }
}

__global__ void set_single(uint32_t *q, uint32_t *cnt, uint32_t value) {
    q[0] = value;
    cnt[0] = 1;
    cnt[1] = 0;
    cnt[2] = 0;
}

enum SmallIdx : int {
    kFr = 0,        // 3 frontier counters
    kAff = 3,       // 3 affected-list counters
    kAffTotal = 6,
    kGcF = 7,
    kGcR = 8,
    kBigF = 9,
    kBigR = 10,
    kTouched = 11,
    kFinalRound = 12,
    kBigRows = 13,  // 3 counters of deferred hub rows
    kCompactCount = 16,
    kOrderedCount = 17,
    kIndexedCount = 20,  // deletion groups answered by the position index
    kIdxRows = 21,       // rows of an arena being indexed (load time)
    kInvalDone = 22,     // vertices expanded by the invalidation closure's local sweeps
    kGaF = 18,  // addition-phase group counts of a presorted batch
    kGaR = 19,
    kEpoch = 23,  // batch epoch of the traversal algorithms (aff_stamp marker)
    // the deletion counters of the reverse arena (its phase runs on the side stream)
    kCompactCountR = 24,
    kOrderedCountR = 25,
    kIndexedCountR = 26,
    kCoopF = 27,  // addition groups left to mutate_add_warp, per arena
    kCoopR = 28,
    kHugeF = 29,  // hub deletion groups served by the whole grid, per arena
    kHugeR = 30,
    kSmallCount = 32
};

constexpr uint32_t kBigRowCap = 65536;

struct DevArena {
    RowDesc *desc = nullptr;
    uint32_t *dev = nullptr;
    uint32_t *host = nullptr;
    uint32_t *host_dptr = nullptr;
    int32_t *seg_slot = nullptr;
    uint8_t *seg_dirty = nullptr;
    ArenaAlloc *alloc = nullptr;
    uint64_t seg_total = 0;
    uint64_t seg_used = 0;
    Status *bstatus = nullptr;  // bounds-check build: where violations are reported
    uint32_t nverts = 0;
    AdjView view() const {
        AdjView v{desc, dev, host_dptr, seg_slot, seg_dirty};
#ifdef CIG_BOUNDS_CHECK
        v.nslots = seg_total * kSegEdges;
        v.nverts = nverts;
        v.bst = bstatus;
#endif
        return v;
    }
};

// Write-back of the edge cache: copy every dirty resident segment to its
// pinned host copy (one block per segment) and clear the flag.
__global__ void flush_dirty(uint8_t *dirty, const int32_t *seg_slot, const uint32_t *cache, uint32_t *host,
                            uint64_t nsegs) {
    for (uint64_t s = blockIdx.x; s < nsegs; s += gridDim.x) {
        if (!dirty[s]) continue;
        const int32_t slot = seg_slot[s];
        if (slot >= 0)
            copy_segment(reinterpret_cast<uint4 *>(host + (s << kSegShift)),
                         reinterpret_cast<const uint4 *>(cache + (static_cast<uint64_t>(slot) << kSegShift)));
        __syncthreads();
        if (threadIdx.x == 0) dirty[s] = 0;
        __syncthreads();
    }
}

const char *kVersion = "cig 0.2.0 (sm_100a)";

// NVTX range over a host-side stage (deletion phase, insertion phase, cache
// service, query, PR batch, load): visible to nsys/ncu timelines, free when
// no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

template <class T>
struct Identity {
    using type = T;
};

}  // namespace

struct cig_handle {
    cig_options opt{};
    std::string err;
    bool dead = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    // The reverse arena's mutation runs on `side` concurrently with the
    // forward arena's (disjoint rows, counters and scratch); `cs` is the
    // stream that launch() and the mutation helpers queue on.
    cudaStream_t side = nullptr, cs = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaEvent_t ev[4] = {};
    int sms = 0;
    uint32_t n = 0;
    uint32_t source = 0;
    bool loaded = false;
    bool initialized = false;
    DevArena fwd, rev;
    uint64_t cache_slots = 0;
    uint64_t resident = 0;
    uint32_t *seg_hot = nullptr;
    // Segment table service (cache.cuh); off with CIG_FLAG_NO_CACHE_REFRESH.
    bool refresh = false;
    int32_t *slot_seg = nullptr;
    uint32_t *seg_score = nullptr, *free_slots = nullptr, *seg_victims = nullptr, *seg_admits = nullptr;
    uint32_t *seg_ctl = nullptr;
    SegTable seg_table() const {
        return SegTable{fwd.seg_slot, slot_seg, fwd.seg_dirty, seg_score, seg_hot, free_slots, seg_victims,
                        seg_admits, seg_ctl, static_cast<uint32_t>(cache_slots), static_cast<uint32_t>(fwd.seg_total),
                        admit_score, cold_score};
    }
    // Service thresholds; CIG_CACHE_ADMIT_SCORE / CIG_CACHE_COLD_SCORE
    // override them when the graph is loaded.
    uint32_t admit_score = kAdmitScore, cold_score = kColdScore;

    unsigned long long *state = nullptr;
    uint32_t *qstamp = nullptr, *aff_stamp = nullptr, *q0 = nullptr, *q1 = nullptr, *list = nullptr;
    uint32_t *small = nullptr;
    unsigned long long *small64 = nullptr;
    unsigned long long *small64x = nullptr;  // 64 more (per-class slot counts)
    TagState *tags = nullptr;
    Status *status = nullptr;
    Status *h_status = nullptr;
    uint32_t epoch = 0;

    void *pr_rank = nullptr, *pr_res = nullptr, *pr_contrib = nullptr, *pr_amend = nullptr;
    double *pr_amend64 = nullptr;  // FP32 mode: per-vertex FP64 amend accumulator (pr_amend_fold)
    uint32_t *pr_hub_bits = nullptr, *pr_hub_prefix = nullptr;  // FP32 mode: FP64 residual slots (pr.cuh)
    uint32_t pr_hubs = 0;
    double *pr_res_hub = nullptr;
    float *pr_comp = nullptr;
    uint32_t *pr_queued = nullptr;
    bool pr64 = false;

    uint64_t bcap = 0;
    uint32_t *du = nullptr, *dv = nullptr, *au = nullptr, *av = nullptr;
    unsigned long long *kf = nullptr, *kr = nullptr, *t1 = nullptr, *t2 = nullptr;
    uint32_t *gf = nullptr, *gr = nullptr, *mf = nullptr, *mr = nullptr, *bigf = nullptr, *bigr = nullptr;
    unsigned long long *pf = nullptr, *prr = nullptr;
    uint32_t *touched = nullptr;
    uint32_t *compact = nullptr;  // rows queued for tombstone compaction
    // The reverse arena's copies of the deletion scratch (its deletion phase
    // runs on the side stream while the forward one runs on the engine
    // stream), and its scan-chunk map and scan scratch.
    uint32_t *compact_r = nullptr, *chunks_r = nullptr, *chunk_end_r = nullptr, *ordered_r = nullptr;
    uint32_t *firstpos_r = nullptr, *indexed_groups_r = nullptr, *chunk_map_r = nullptr;
    uint8_t *gtype_r = nullptr;
    uint32_t *coopf = nullptr, *coopr = nullptr;  // addition groups served one warp each
    uint32_t *hugef = nullptr, *huger = nullptr;  // hub deletion groups served by the grid
    void *cub_r = nullptr;
    size_t cub_r_bytes = 0;
    // flat deletion: per-group chunk counts, their inclusive prefix sum, the
    // groups left to the ordered kernels, first match per key
    uint32_t *chunks = nullptr, *chunk_end = nullptr, *ordered = nullptr, *firstpos = nullptr;
    uint32_t *chunk_map = nullptr;  // group of every 512-entry scan chunk
    uint8_t *gtype = nullptr;             // kind of every deletion group
    uint32_t *indexed_groups = nullptr;   // deletion groups of indexed rows

    // Position index of hub rows, per arena (posindex.cuh); off with
    // CIG_POS_INDEX=0 or when the tables would not fit their share of memory.
    struct IndexBuf {
        unsigned long long *keys = nullptr;
        uint2 *val = nullptr;
        uint32_t *rowbit = nullptr;
        uint64_t cap = 0;
        uint64_t rows = 0, entries = 0;  // at the last build
        uint64_t inserted = 0;           // addition requests since (a bound on new keys)
        uint32_t cls = 0;                // smallest class indexed
        uint64_t builds = 0;
    } ixb[2];  // [0] forward, [1] reverse
    bool use_index = true;
    uint32_t index_cls = kIdxCls;             // smallest block class to index
    uint64_t index_headroom = 1ull << 20;    // least insert room of a table
    double index_spare = 1.0;                // insert room per entry
    PosIndex pos_index(bool forward) const {
        const IndexBuf &b = ixb[forward ? 0 : 1];
        return PosIndex{b.keys, b.val, b.cap ? b.cap - 1 : 0, b.rowbit};
    }

    // (Re)build the index of arena A.  A table for e entries has room for
    // max(index_headroom, index_spare * e) inserts at a load factor of one
    // half (2 * (e + room) slots, to the next power of two), so that at
    // steady state a rebuild comes at most once per e inserted keys and its
    // cost stays a small share of the batches between.  Rows of class >=
    // index_cls are indexed when their table fits a quarter of the free
    // device memory; otherwise the threshold rises until it does, and the
    // arena goes unindexed when no class fits.  Synchronises.
    uint64_t index_cap(uint64_t e) const {
        const uint64_t room = std::max<uint64_t>(index_headroom, static_cast<uint64_t>(index_spare * e));
        uint64_t cap = 1;
        while (cap < 2 * (e + room)) cap <<= 1;
        return cap;
    }
    // The initially resident segments: the small rows first (the last
    // `small_segs` segments of the arena), then the largest classes (the
    // first segments) while the `filled` slots last, the middle classes in
    // host memory.  A small row costs a traversal one dependent host access
    // per read and most reads are of small rows, while a large row crosses
    // the link in long requests but carries the most bytes; the rows between
    // gain the least from HBM -- as long as the position index covers them.
    // An unindexed row is scanned whole by every deletion in it, so when the
    // index leaves rows above the small classes out (a small --index_budget,
    // or no index) the largest classes come first alone.
    // CIG_CACHE_SMALL_PCT=p gives the last segments p % of the slots instead
    // (0: the first segments only).
    void place_resident(uint64_t filled, uint64_t small_segs) {
        uint64_t small = 0;
        if (refresh) {
            if (cache_small_pct >= 0.0) {
                small = std::min<uint64_t>(filled, static_cast<uint64_t>(filled * cache_small_pct / 100.0));
            } else {
                const bool middle_indexed = ixb[0].cap && ixb[0].cls <= kSmallRowClass + 1;
                small = middle_indexed ? std::min<uint64_t>(filled, small_segs) : 0;
            }
        }
        const uint64_t big = filled - small;
        auto seg_of_slot = [&](uint64_t i) { return i < big ? i : fwd.seg_used - small + (i - big); };
        const size_t seg_bytes = kSegEdges * sizeof(uint32_t);
        if (big) CK(cudaMemcpy(fwd.dev, fwd.host, big * seg_bytes, cudaMemcpyHostToDevice));
        if (small)
            CK(cudaMemcpy(fwd.dev + big * kSegEdges, fwd.host + (fwd.seg_used - small) * kSegEdges, small * seg_bytes,
                          cudaMemcpyHostToDevice));
        std::vector<int32_t> slot(fwd.seg_total, -1);
        for (uint64_t i = 0; i < resident; ++i) slot[seg_of_slot(i)] = static_cast<int32_t>(i);
        CK(cudaMemcpy(fwd.seg_slot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        if (!refresh) return;
        std::vector<int32_t> owner(cache_slots, -1);
        for (uint64_t i = 0; i < filled; ++i) owner[i] = static_cast<int32_t>(seg_of_slot(i));
        std::vector<uint32_t> stack;
        for (uint64_t k = cache_slots; k-- > filled;) stack.push_back(static_cast<uint32_t>(k));
        CK(cudaMemcpy(slot_seg, owner.data(), cache_slots * sizeof(int32_t), cudaMemcpyHostToDevice));
        if (!stack.empty())
            CK(cudaMemcpy(free_slots, stack.data(), stack.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        const uint32_t ctl[kCtlCount] = {static_cast<uint32_t>(stack.size()), static_cast<uint32_t>(fwd.seg_used)};
        CK(cudaMemcpy(seg_ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice));
    }

    void build_index(DevArena &A, bool forward) {
        IndexBuf &b = ixb[forward ? 0 : 1];
        if (!use_index) return;
        CK(cudaMemsetAsync(small64x, 0, 64 * sizeof(unsigned long long), stream));
        launch(idx_class_slots, sms * 2, 256, A.desc, n, small64x);
        unsigned long long hist[64];
        CK(cudaMemcpyAsync(hist, small64x, sizeof(hist), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        // Each table may take half of --index_budget, or else a quarter of
        // the free device memory (counting the table it replaces).
        const uint64_t share = opt.index_budget_gib > 0
                                   ? static_cast<uint64_t>(opt.index_budget_gib * 1073741824.0 / 2.0)
                                   : (fr + b.cap * (sizeof(unsigned long long) + sizeof(uint2))) / 4;
        uint64_t entries = 0, cap = 0;
        uint32_t cls = 64;
        for (uint32_t c = 63; c + 1 > index_cls; --c) {
            const uint64_t e = entries + hist[c];
            const uint64_t cp = index_cap(e);
            if (cp * (sizeof(unsigned long long) + sizeof(uint2)) > share) break;
            entries = e;
            cap = cp;
            cls = c;
            if (c == 0) break;
        }
        if (entries == 0) {
            dfree(b.keys);
            dfree(b.val);
            dfree(b.rowbit);
            b = IndexBuf{};
            return;
        }
        if (cap > b.cap) {
            dfree(b.keys);
            dfree(b.val);
            dmalloc(b.keys, cap);
            dmalloc(b.val, cap);
            b.cap = cap;
        }
        b.cls = cls;
        const uint32_t words = (n + 31) / 32;
        if (!b.rowbit) dmalloc(b.rowbit, words);
        b.entries = entries;
        b.inserted = 0;
        b.builds += 1;
        const PosIndex ix = pos_index(forward);
        launch(idx_init, sms * 8, 256, ix);
        CK(cudaMemsetAsync(small + kIdxRows, 0, sizeof(uint32_t), stream));
        launch(idx_pick_rows, persistent_grid(), 256, A.desc, n, b.cls, b.rowbit, tmp_u32, small + kIdxRows, n,
               status);
        launch(idx_build, sms * 4, 256, A.view(), A.desc, tmp_u32, small + kIdxRows, ix, status);
        check_launch();
        uint32_t rows = 0;
        CK(cudaMemcpyAsync(&rows, small + kIdxRows, sizeof(rows), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        b.rows = rows;
    }
    uint64_t chunk_map_cap = 0;
    int del_scan_per_sm = 0;
    int del_scan_blocks_per_sm() {
        if (!del_scan_per_sm) {
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&del_scan_per_sm, del_scan, kMutWarps * 32, 0));
            del_scan_per_sm = std::max(1, del_scan_per_sm);
        }
        return del_scan_per_sm;
    }
    // group building: head flags, their exclusive scan, group ends per direction
    uint32_t *gflags = nullptr, *gpos = nullptr, *gendf = nullptr, *gendr = nullptr;
    // whole-batch sort (apply_batch): packed keys, and the addition phase's
    // groups, kept apart from the deletion phase's
    unsigned long long *kc = nullptr, *tc = nullptr;
    uint32_t *gaf = nullptr, *gar = nullptr, *gaendf = nullptr, *gaendr = nullptr;
    bool presorted = false;
    void *cub = nullptr;
    size_t cub_bytes = 0;
    uint32_t *stage = nullptr;  // pinned staging for host update arrays (4 * bcap)

    uint32_t *tmp_u32 = nullptr;  // n entries (exports)
    uint64_t last_nd = 0, last_na = 0;

    // Stage profiler (CUDA events on `stream`, resolved in finish()).
    struct ProfRec {
        int stage;
        cudaEvent_t a, b;
    };
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<ProfRec> prof_pending;
    cig_stage_profile prof[CIG_STAGE_COUNT] = {};

    cudaEvent_t take_event() {
        if (capturing) {
            // A captured graph records its own events on every replay.
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            capture_events.push_back(e);
            return e;
        }
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }
    // Record an event on the engine stream; under stream capture it becomes
    // an event-record node of the graph (recorded at every replay).
    void rec(cudaEvent_t e) {
        if (capturing)
            CK(cudaEventRecordWithFlags(e, cs, cudaEventRecordExternal));
        else
            CK(cudaEventRecord(e, cs));
    }
    int prof_begin(int stage) {
        if (!prof_on) return -1;
        cudaEvent_t a = take_event();
        rec(a);
        prof_pending.push_back({stage, a, nullptr});
        return static_cast<int>(prof_pending.size()) - 1;
    }
    void prof_end(int idx) {
        if (idx < 0) return;
        cudaEvent_t b = take_event();
        rec(b);
        prof_pending[idx].b = b;
    }
    void prof_resolve() {
        for (const auto &p : prof_pending) {
            float ms = 0;
            if (p.b && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                prof[p.stage].ms += ms;
                prof[p.stage].launches += 1;
            }
        }
        prof_pending.clear();
        ev_used = 0;
        if (!prof_on) return;
        const unsigned long long *c = h_status->counters;
        const std::pair<int, int> groups[] = {{CIG_STAGE_PUSH, kCntPush}, {CIG_STAGE_INVAL, kCntInval},
                                              {CIG_STAGE_PULL, kCntPull}, {CIG_STAGE_PR, kCntPr}};
        for (const auto &g : groups) {
            prof[g.first].edges += c[g.second + 0];
            prof[g.first].edges_cached += c[g.second + 1];
            prof[g.first].rows += c[g.second + 2];
            prof[g.first].hits += c[g.second + 3];
        }
        prof[CIG_STAGE_DEL_SCAN].edges += c[kCntDelScanned];
        prof[CIG_STAGE_DEL_SCAN].edges_cached += c[kCntDelScannedCached];
        prof[CIG_STAGE_ADD].rows += c[kCntRelocated];
        prof[CIG_STAGE_ADD].edges += c[kCntMovedEntries];
        prof[CIG_STAGE_CACHE].rows += c[kCntSegLoaded] + c[kCntSegEvicted];
    }

    // ------------------------------------------------------------ helpers
    int grid_for(uint64_t items, int tpb = 256) const {
        const uint64_t g = (items + tpb - 1) / tpb;
        return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(g, 1u << 30)));
    }
    int persistent_grid() const { return sms * 8; }

    Frontier frontier() const { return Frontier{q0, q1, small + kFr, n + 1}; }

    BigRow *big_rows = nullptr;
    // Deferred hub rows; the counters are cleared before every launch that uses them.
    BigList big_list() {
        CK(cudaMemsetAsync(small + kBigRows, 0, 3 * sizeof(uint32_t), stream));
        return BigList{big_rows, small + kBigRows, kBigRowCap, tune.split};
    }

    template <class K>
    int coop_blocks(K kernel, int tpb) const {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, tpb, 0));
        per_sm = std::min(per_sm, static_cast<int>(in_batch && tune.inc_per_sm ? tune.inc_per_sm : tune.per_sm));
        if (per_sm < 1) throw CigError(CIG_ERR_DEVICE, "cooperative kernel does not fit on an SM");
        return per_sm * sms;
    }
    // Set while the closures of an update batch are queued: they may use
    // their own launch shape (tune.inc_per_sm), the static solve uses per_sm.
    bool in_batch = false;

    uint64_t n_launch = 0;  // kernels this engine launched (CUB sort kernels not included)

    // Launch-shape parameters of the persistent closures, chosen by
    // cig_autotune (or CIG_COOP_BLOCKS_PER_SM / CIG_SPLIT_DEG at create).
    struct Tune {
        uint32_t per_sm = 4;        // cooperative blocks per SM (frontier tile = per_sm x 148 blocks)
        // The same for the closures of update batches (0: per_sm).  Their
        // rounds carry a few items per block, and half the blocks meet at
        // each grid barrier sooner (s24 SSSP stream: 2 per SM ~1 % faster
        // than 4).
        uint32_t inc_per_sm = 2;
        uint32_t split = kSplitDeg; // rows of at least this many entries are expanded by the whole grid
        uint32_t pull_on = 32;      // BFS waves go bottom-up above n/pull_on frontier vertices (0: never)
        uint32_t pull_off = 64;     // ... and stay while at least n/pull_off
        uint32_t pull_width = 16;   // waves of more sources stay top-down
    } tune;

    template <class... P>
    void launch(void (*kernel)(P...), int grid, int block, typename Identity<P>::type... args) {
        kernel<<<grid, block, 0, cs>>>(args...);
        ++n_launch;
    }

    // Arguments are converted to the kernel's exact parameter types, as the
    // void* argument array of a cooperative launch requires.
    template <class... P>
    void launch_coop(void (*kernel)(P...), int tpb, typename Identity<P>::type... args) {
        void *argv[] = {static_cast<void *>(&args)...};
        const int blocks = coop_blocks(kernel, tpb);
        if (capturing) {
            // Captured as a kernel node with the cooperative attribute: the
            // graph launch keeps the co-residency guarantee of the grid.
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(blocks);
            cfg.blockDim = dim3(tpb);
            cfg.dynamicSmemBytes = 0;
            cfg.stream = stream;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            CK(cudaLaunchKernelExC(&cfg, reinterpret_cast<const void *>(kernel), argv));
        } else {
            CK(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kernel), dim3(blocks), dim3(tpb), argv, 0,
                                           stream));
        }
        ++n_launch;
    }

    template <class... P>
    void launch_coop_on(cudaStream_t st, void (*kernel)(P...), int tpb, typename Identity<P>::type... args) {
        void *argv[] = {static_cast<void *>(&args)...};
        const int blocks = coop_blocks(kernel, tpb);
        CK(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kernel), dim3(blocks), dim3(tpb), argv, 0, st));
        ++n_launch;
    }

    void check_launch() { CK(cudaGetLastError()); }

    // ------------------------------------------------------------ CUDA graphs of the batch path
    // A batch (or one phase) of the traversal algorithms is a fixed chain of
    // ~60 launches and memsets on the engine stream whose arguments depend
    // only on the batch shape (deletions, insertions) and on device buffers
    // that stay put between reallocations; everything that changes per batch
    // (epoch, tags, counts) lives on the device.  So the chain is captured
    // once per shape into a CUDA graph and replayed with one launch.  A shape
    // is captured the second time it is seen (uneven streams of one-off
    // sizes stay on direct launches).  Anything that reallocates a captured
    // buffer or changes a launch shape bumps `graph_gen`, which retires every
    // graph.  Host decisions that used to sit inside the chain run before
    // the replay: position-index upkeep (index_upkeep) and the scan-chunk map
    // size (reserve_chunk_map).  CIG_GRAPHS=0 turns graphs off.
    struct BatchGraph {
        int kind = 0;  // 0 whole batch, 1 deletion phase, 2 insertion phase
        uint64_t nd = 0, na = 0, gen = 0, last_use = 0;
        bool prof = false;
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
        std::vector<ProfRec> prof_recs;
        std::vector<cudaEvent_t> events;
    };
    std::vector<BatchGraph> graphs;
    std::vector<std::pair<int, std::pair<uint64_t, uint64_t>>> shapes_seen;
    std::vector<cudaEvent_t> capture_events;
    bool use_graphs = true;
    bool capturing = false;
    uint64_t graph_gen = 1, graph_clock = 0;
    uint64_t graph_replays = 0, graph_captures = 0;
    static constexpr size_t kMaxGraphs = 8;

    static void release_graph(BatchGraph &g) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto e : g.events) cudaEventDestroy(e);
        g.exec = nullptr;
        g.events.clear();
    }
    void drop_graphs() {
        for (auto &g : graphs) release_graph(g);
        graphs.clear();
        shapes_seen.clear();
    }
    void retire_graphs() { ++graph_gen; }

    // Run `body` (the launches of one batch or phase of shape kind/nd/na on
    // the engine stream) through the graph cache.
    template <class F>
    void run_graphed(int kind, uint64_t nd, uint64_t na, F body) {
        if (!use_graphs) {
            body();
            return;
        }
        for (auto &g : graphs) {
            if (g.kind == kind && g.nd == nd && g.na == na && g.gen == graph_gen && g.prof == prof_on) {
                CK(cudaGraphLaunch(g.exec, stream));
                n_launch += g.launches;
                g.last_use = ++graph_clock;
                ++graph_replays;
                if (prof_on) prof_pending.insert(prof_pending.end(), g.prof_recs.begin(), g.prof_recs.end());
                return;
            }
        }
        const std::pair<int, std::pair<uint64_t, uint64_t>> shape{kind, {nd, na}};
        if (std::find(shapes_seen.begin(), shapes_seen.end(), shape) == shapes_seen.end()) {
            if (shapes_seen.size() >= 64) shapes_seen.erase(shapes_seen.begin());
            shapes_seen.push_back(shape);
            body();
            return;
        }
        // Second sighting of this shape: capture it, then replay it.
        for (auto it = graphs.begin(); it != graphs.end();) {
            if (it->gen != graph_gen) {
                release_graph(*it);
                it = graphs.erase(it);
            } else {
                ++it;
            }
        }
        if (graphs.size() >= kMaxGraphs) {
            auto lru = std::min_element(graphs.begin(), graphs.end(),
                                        [](const BatchGraph &a, const BatchGraph &b) { return a.last_use < b.last_use; });
            release_graph(*lru);
            graphs.erase(lru);
        }
        BatchGraph g;
        g.kind = kind;
        g.nd = nd;
        g.na = na;
        g.gen = graph_gen;
        g.prof = prof_on;
        const uint64_t l0 = n_launch;
        const size_t p0 = prof_pending.size();
        const bool presorted0 = presorted;
        capture_events.clear();
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        cudaGraph_t graph = nullptr;
        try {
            body();
        } catch (...) {
            capturing = false;
            cudaStreamEndCapture(stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            for (auto e : capture_events) cudaEventDestroy(e);
            capture_events.clear();
            prof_pending.resize(p0);
            n_launch = l0;
            throw;
        }
        capturing = false;
        const cudaError_t ec = cudaStreamEndCapture(stream, &graph);
        cudaError_t ei = cudaErrorUnknown;
        if (ec == cudaSuccess) ei = cudaGraphInstantiateWithFlags(&g.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        g.events.swap(capture_events);
        if (ec != cudaSuccess || ei != cudaSuccess) {
            release_graph(g);
            cudaGetLastError();
            throw CigError(CIG_ERR_DEVICE, std::string("batch graph capture failed: ") +
                                               cudaGetErrorString(ec != cudaSuccess ? ec : ei));
        }
        g.launches = n_launch - l0;
        n_launch = l0;
        g.prof_recs.assign(prof_pending.begin() + p0, prof_pending.end());
        prof_pending.resize(p0);
        presorted = presorted0;
        ++graph_captures;
        graphs.push_back(std::move(g));
        BatchGraph &r = graphs.back();
        CK(cudaGraphLaunch(r.exec, stream));
        n_launch += r.launches;
        ++graph_replays;
        r.last_use = ++graph_clock;
        if (prof_on) prof_pending.insert(prof_pending.end(), r.prof_recs.begin(), r.prof_recs.end());
    }

    uint64_t launch_mark = 0;

    uint64_t replay_mark = 0;
    void reset_counters() {
        presorted = false;
        CK(cudaMemsetAsync(status->counters, 0, sizeof(status->counters), stream));
        launch_mark = n_launch;
        replay_mark = graph_replays;
    }

    void require_alive() const {
        if (dead) throw CigError(CIG_ERR_STATE, "handle unusable after an earlier device error: " + err);
    }

    // Synchronise, read the device status, raise on device-reported errors.
    void finish() {
        CK(cudaStreamSynchronize(stream));
        CK(cudaGetLastError());
        CK(cudaMemcpy(h_status, status, sizeof(Status), cudaMemcpyDeviceToHost));
        prof_resolve();
        const uint32_t e = h_status->err;
        if (e) {
            dead = true;
            std::string what;
            int code = CIG_ERR_LIMIT;
            if (e & kErrArena) {
                what += "adjacency arena exhausted; ";
                code = CIG_ERR_ARENA;
            }
            if (e & kErrRounds) what += "round bound exceeded; ";
            if (e & kErrBarrier) what += "grid barrier wait limit exceeded; ";
            if (e & kErrQueue) what += "work queue overflow; ";
            if (e & kErrNonFinite) what += "non-finite PageRank value; ";
            if (e & kErrInternal) what += "internal consistency error; ";
            if (e & kErrBounds) what += "device index out of bounds (bounds-check build); ";
            throw CigError(code, "device reported: " + what + "info=" + std::to_string(h_status->err_info));
        }
    }

    template <class F>
    void dispatch(F f) {
        switch (opt.algo) {
        case CIG_BFS: f(std::integral_constant<int, kBfs>{}); break;
        case CIG_SSSP:
            if (opt.flags & CIG_FLAG_WEIGHT_U255)
                f(std::integral_constant<int, kSsspU>{});
            else
                f(std::integral_constant<int, kSssp>{});
            break;
        case CIG_CC: f(std::integral_constant<int, kCc>{}); break;
        default: throw CigError(CIG_ERR_ARG, "algorithm has no traversal state");
        }
    }

    // ------------------------------------------------------------ lifecycle
    void create(const cig_options &o) {
        opt = o;
        if (opt.algo < CIG_BFS || opt.algo > CIG_PR) throw CigError(CIG_ERR_ARG, "unknown algorithm");
        device = opt.device;
        CK(cudaSetDevice(device));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        int coop = 0;
        CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        if (!coop) throw CigError(CIG_ERR_DEVICE, "device does not support cooperative launch");
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
        cs = stream;
        for (auto &e : ev) CK(cudaEventCreate(&e));
        dmalloc(status, 1);
        CK(cudaMemset(status, 0, sizeof(Status)));
        CK(cudaHostAlloc(reinterpret_cast<void **>(&h_status), sizeof(Status), cudaHostAllocDefault));
        dmalloc(small, kSmallCount);
        CK(cudaMemset(small, 0, kSmallCount * sizeof(uint32_t)));
        dmalloc(small64, 4);
        dmalloc(small64x, 64);
        dmalloc(big_rows, kBigRowCap);
        dmalloc(tags, 1);
        CK(cudaMemset(tags, 0, sizeof(TagState)));
        pr64 = (opt.flags & CIG_FLAG_PR_FP64) != 0;
        if (const char *e = std::getenv("CIG_COOP_BLOCKS_PER_SM")) tune.per_sm = std::max(1, std::atoi(e));
        if (const char *e = std::getenv("CIG_SPLIT_DEG")) tune.split = std::max(32, std::atoi(e));
        if (const char *e = std::getenv("CIG_INC_BLOCKS_PER_SM")) tune.inc_per_sm = std::max(0, std::atoi(e));
        if (const char *e = std::getenv("CIG_LOCAL_SWEEPS")) local_sweeps = static_cast<uint32_t>(std::max(0, std::atoi(e)));
        if (const char *e = std::getenv("CIG_CACHE_SMALL_PCT")) cache_small_pct = std::min(100.0, std::max(0.0, std::atof(e)));
        if (opt.flags & CIG_FLAG_NO_GRAPHS) use_graphs = false;
        if (const char *e = std::getenv("CIG_GRAPHS")) use_graphs = std::atoi(e) != 0;
        if (const char *e = std::getenv("CIG_MERGE_PUSH")) merge_push = std::atoi(e) != 0;
        if (const char *e = std::getenv("CIG_POS_INDEX")) use_index = std::atoi(e) != 0;
        if (const char *e = std::getenv("CIG_POS_INDEX_CLS")) index_cls = static_cast<uint32_t>(std::atoi(e));
        if (const char *e = std::getenv("CIG_POS_INDEX_HEADROOM"))
            index_headroom = std::max<uint64_t>(64, std::strtoull(e, nullptr, 10));
        if (const char *e = std::getenv("CIG_POS_INDEX_SPARE")) index_spare = std::max(0.0, std::atof(e));
        if (const char *e = std::getenv("CIG_PULL_ON")) tune.pull_on = static_cast<uint32_t>(std::max(0, std::atoi(e)));
        if (const char *e = std::getenv("CIG_PULL_OFF")) tune.pull_off = static_cast<uint32_t>(std::max(1, std::atoi(e)));
    }

    void destroy() {
        stager_stop();
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : ev_pool) cudaEventDestroy(e);
        ev_pool.clear();
        dfree(fwd.desc);
        dfree(fwd.dev);
        dfree(fwd.seg_slot);
        dfree(fwd.seg_dirty);
        dfree(fwd.alloc);
        if (fwd.host) cudaFreeHost(fwd.host);
        dfree(rev.desc);
        dfree(rev.dev);
        dfree(rev.alloc);
        dfree(seg_hot);
        dfree(slot_seg);
        dfree(seg_score);
        dfree(free_slots);
        dfree(seg_victims);
        dfree(seg_admits);
        dfree(seg_ctl);
        dfree(state);
        dfree(qstamp);
        dfree(aff_stamp);
        dfree(q0);
        dfree(q1);
        dfree(list);
        dfree(small);
        dfree(small64);
        dfree(small64x);
        dfree(big_rows);
        dfree(tags);
        dfree(status);
        if (h_status) cudaFreeHost(h_status);
        dfree(pr_rank);
        dfree(pr_res);
        dfree(pr_contrib);
        dfree(pr_amend);
        dfree(pr_amend64);
        dfree(pr_hub_bits);
        dfree(pr_hub_prefix);
        dfree(pr_res_hub);
        dfree(pr_comp);
        dfree(pr_queued);
        free_batch();
        dfree(tmp_u32);
        dfree(inval_done);
        dfree(chunk_map);
        dfree(chunk_map_r);
        for (auto &b : ixb) {
            dfree(b.keys);
            dfree(b.val);
            dfree(b.rowbit);
            b = IndexBuf{};
        }
        dfree(bsnap);
        dfree(bdig);
        for (auto &e : bev) cudaEventDestroy(e);
        bev.clear();
        free_queries();
        if (side) cudaStreamSynchronize(side);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }

    void free_batch() {
        dfree(du);
        dfree(dv);
        dfree(au);
        dfree(av);
        dfree(kf);
        dfree(kr);
        dfree(t1);
        dfree(t2);
        dfree(gf);
        dfree(gr);
        dfree(mf);
        dfree(mr);
        dfree(bigf);
        dfree(bigr);
        dfree(gtype);
        dfree(indexed_groups);
        dfree(kc);
        dfree(tc);
        dfree(gaf);
        dfree(gar);
        dfree(gaendf);
        dfree(gaendr);
        dfree(pf);
        dfree(prr);
        dfree(touched);
        dfree(compact);
        dfree(chunks);
        dfree(chunk_end);
        dfree(ordered);
        dfree(firstpos);
        dfree(compact_r);
        dfree(chunks_r);
        dfree(chunk_end_r);
        dfree(ordered_r);
        dfree(firstpos_r);
        dfree(indexed_groups_r);
        dfree(gtype_r);
        dfree(coopf);
        dfree(coopr);
        dfree(hugef);
        dfree(huger);
        if (cub_r) cudaFree(cub_r);
        cub_r = nullptr;
        dfree(gflags);
        dfree(gpos);
        dfree(gendf);
        dfree(gendr);
        dfree(cub);
        if (stage) cudaFreeHost(stage);
        stage = nullptr;
        bcap = 0;
    }

    void ensure_batch(uint64_t need) {
        if (need <= bcap) return;
        if (need > 0x7FFFFFFFull) throw CigError(CIG_ERR_ARG, "update phase larger than 2^31 records");
        CK(cudaStreamSynchronize(stream));
        free_batch();
        uint64_t cap = std::max<uint64_t>(need, std::max<uint64_t>(opt.max_batch, 1024));
        dmalloc(du, cap);
        dmalloc(dv, cap);
        dmalloc(au, cap);
        dmalloc(av, cap);
        dmalloc(kf, cap);
        dmalloc(kr, cap);
        dmalloc(t1, cap);
        dmalloc(t2, cap);
        dmalloc(gf, cap);
        dmalloc(gr, cap);
        dmalloc(mf, cap);
        dmalloc(mr, cap);
        dmalloc(bigf, cap);
        dmalloc(bigr, cap);
        dmalloc(pf, cap);
        dmalloc(prr, cap);
        dmalloc(touched, 2 * cap);
        dmalloc(compact, cap);
        dmalloc(chunks, cap);
        dmalloc(chunk_end, cap);
        dmalloc(ordered, cap);
        dmalloc(gtype, cap);
        dmalloc(indexed_groups, cap);
        dmalloc(firstpos, cap);
        dmalloc(compact_r, cap);
        dmalloc(chunks_r, cap);
        dmalloc(chunk_end_r, cap);
        dmalloc(ordered_r, cap);
        dmalloc(gtype_r, cap);
        dmalloc(indexed_groups_r, cap);
        dmalloc(firstpos_r, cap);
        dmalloc(coopf, cap);
        dmalloc(coopr, cap);
        dmalloc(hugef, cap);
        dmalloc(huger, cap);
        dmalloc(gflags, 4 * cap);
        dmalloc(gpos, 4 * cap);
        dmalloc(gendf, cap);
        dmalloc(gendr, cap);
        dmalloc(kc, 4 * cap);
        dmalloc(tc, 4 * cap);
        dmalloc(gaf, cap);
        dmalloc(gar, cap);
        dmalloc(gaendf, cap);
        dmalloc(gaendr, cap);
        if (opt.algo == CIG_PR) {
            dfree(pr_amend);
            CK(cudaMalloc(&pr_amend, 2 * cap * sizeof(double)));
        }
        cub::DoubleBuffer<unsigned long long> db(kc, tc);
        size_t bytes = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, static_cast<int>(4 * cap), 0, 64, stream));
        size_t scan_bytes = 0;
        CK(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, chunks, chunk_end, static_cast<int>(cap), stream));
        bytes = std::max(bytes, scan_bytes);
        CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, gflags, gpos, static_cast<int>(4 * cap), stream));
        bytes = std::max(bytes, scan_bytes);
        cub_bytes = bytes;
        CK(cudaMalloc(&cub, std::max<size_t>(bytes, 16)));
        CK(cub::DeviceScan::InclusiveSum(nullptr, cub_r_bytes, chunks_r, chunk_end_r, static_cast<int>(cap), stream));
        CK(cudaMalloc(&cub_r, std::max<size_t>(cub_r_bytes, 16)));
        CK(cudaHostAlloc(reinterpret_cast<void **>(&stage), 4 * cap * sizeof(uint32_t), cudaHostAllocDefault));
        bcap = cap;
        retire_graphs();
        // Size the scan-chunk maps for the whole capacity now: a map that
        // grew between the batches of a batched call synchronised in the
        // middle of its queue.
        if (fwd.seg_total) reserve_chunk_map(cap);
    }

    int key_end_bit() const {
        int hb = 0;
        while (hb < 32 && (1ull << hb) <= n) ++hb;
        return 32 + hb;
    }

    // Sort keys in place through the double buffer; returns the sorted array.
    unsigned long long *sort_keys(unsigned long long *keys, unsigned long long *tmp, uint64_t count) {
        if (count == 0) return keys;
        cub::DoubleBuffer<unsigned long long> db(keys, tmp);
        size_t bytes = cub_bytes;
        CK(cub::DeviceRadixSort::SortKeys(cub, bytes, db, static_cast<int>(count), 0, key_end_bit(), stream));
        return db.Current();
    }

    // ------------------------------------------------------------ load
    void load_csr(uint32_t nv, const uint64_t *xadj, const uint32_t *adj) {
        const NvtxRange range("cig.load");
        if (loaded) throw CigError(CIG_ERR_ARG, "graph already loaded");
        if (nv == 0) throw CigError(CIG_ERR_ARG, "graph must have at least one vertex");
        if (!xadj || (xadj[nv] && !adj)) throw CigError(CIG_ERR_ARG, "null CSR arrays");
        if (xadj[0] != 0) throw CigError(CIG_ERR_ARG, "xadj[0] must be 0");
        std::vector<uint32_t> deg(nv);
        for (uint32_t v = 0; v < nv; ++v) {
            if (xadj[v + 1] < xadj[v]) throw CigError(CIG_ERR_ARG, "xadj must be non-decreasing");
            const uint64_t d = xadj[v + 1] - xadj[v];
            if (d > 0xFFFFFFFFull) throw CigError(CIG_ERR_ARG, "row degree exceeds 2^32-1");
            deg[v] = static_cast<uint32_t>(d);
        }
        const uint64_t m = xadj[nv];
        std::atomic<bool> bad{false};
        parallel_for(m, [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i)
                if (adj[i] >= nv) bad = true;
        });
        if (bad) throw CigError(CIG_ERR_ARG, "edge destination out of range");
        n = nv;
        source = std::min<uint32_t>(opt.source, n - 1);
        if (opt.algo == CIG_CC) {
            // Depth bits below the label (labels are vertex ids < n).
            uint32_t label_bits = 1;
            while (label_bits < 32 && (1ull << label_bits) < n) ++label_bits;
            cc_shift = 32 - label_bits;
            // CIG_CC_DEPTH_BITS caps the depth field (0 keeps the equal-label
            // rule everywhere; small values make saturation common).
            if (const char *e = std::getenv("CIG_CC_DEPTH_BITS"))
                cc_shift = std::min<uint32_t>(cc_shift, static_cast<uint32_t>(std::max(0, std::atoi(e))));
            CK(cudaMemcpy(&status->cc_shift, &cc_shift, sizeof(cc_shift), cudaMemcpyHostToDevice));
        }
        CK(cudaSetDevice(device));

        // Forward arena in pinned mapped host memory.
        Layout L = plan_layout(n, deg.data());
        const double pct = opt.arena_headroom_pct ? opt.arena_headroom_pct : 12.5;
        const uint64_t head = std::max<uint64_t>(static_cast<uint64_t>(L.used_segs * pct / 100.0) + 1,
                                                 (1ull << 20) >> kSegShift);
        fwd.seg_used = L.used_segs;
        fwd.seg_total = L.used_segs + head;
        fwd.nverts = n;
        fwd.bstatus = status;
        const size_t host_bytes = fwd.seg_total * kSegEdges * sizeof(uint32_t);
        {
            const cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&fwd.host), host_bytes,
                                                cudaHostAllocMapped | cudaHostAllocPortable);
            if (e != cudaSuccess) {
                cudaGetLastError();
                fwd.host = nullptr;
                throw CigError(CIG_ERR_NOMEM, "pinned host arena of " + std::to_string(host_bytes) + " bytes failed");
            }
        }
        CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&fwd.host_dptr), fwd.host, 0));
        const RowDesc *desc_h = L.desc.data();
        uint32_t *arena = fwd.host;
        parallel_for(n, [&](uint64_t b, uint64_t e) {
            for (uint64_t v = b; v < e; ++v)
                if (deg[v]) std::memcpy(arena + desc_h[v].off, adj + xadj[v], deg[v] * sizeof(uint32_t));
        });
        dmalloc(fwd.desc, n);
        CK(cudaMemcpy(fwd.desc, L.desc.data(), n * sizeof(RowDesc), cudaMemcpyHostToDevice));
        upload_alloc(fwd, L);

        // HBM edge cache: whole segments (which ones start resident: place_resident).
        uint64_t budget_slots;
        if (opt.cache_compat) {
            const long long c = static_cast<long long>(opt.cache_gib);
            static const uint64_t table[] = {0ull, 268435455ull, 536870921ull, 805306365ull, 1073741824ull};
            budget_slots = (c >= 0 && c <= 4) ? table[c] : 1073741824ull;
        } else {
            budget_slots = opt.cache_gib > 0 ? static_cast<uint64_t>(opt.cache_gib * 1073741824.0 / 4.0) : 0;
        }
        // Slots beyond the used segments serve the segments that the block
        // allocator hands out later: with the segment-table service they sit
        // on its free stack, without it they are bound to the headroom
        // segments in order.  Either way relocated rows land in HBM while the
        // budget lasts.
        cache_slots = std::min<uint64_t>(budget_slots >> kSegShift, fwd.seg_total);
        refresh = cache_slots > 0 && !(opt.flags & CIG_FLAG_NO_CACHE_REFRESH);
        const uint64_t filled = std::min<uint64_t>(cache_slots, fwd.seg_used);
        resident = refresh ? filled : cache_slots;
        if (cache_slots) dmalloc(fwd.dev, cache_slots * kSegEdges);
        // Which segments start resident is chosen once the position index
        // is built (place_resident); until then every segment is read from
        // host memory (the index build reads the rows through the table).
        {
            std::vector<int32_t> slot(fwd.seg_total, -1);
            dmalloc(fwd.seg_slot, fwd.seg_total);
            CK(cudaMemcpy(fwd.seg_slot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
            dmalloc(fwd.seg_dirty, fwd.seg_total);
            CK(cudaMemset(fwd.seg_dirty, 0, fwd.seg_total));
        }
        dmalloc(seg_hot, fwd.seg_total);
        CK(cudaMemset(seg_hot, 0, fwd.seg_total * sizeof(uint32_t)));
        if (refresh) {
            if (const char *e = std::getenv("CIG_CACHE_ADMIT_SCORE")) admit_score = static_cast<uint32_t>(std::atol(e));
            if (const char *e = std::getenv("CIG_CACHE_COLD_SCORE")) cold_score = static_cast<uint32_t>(std::atol(e));
            dmalloc(slot_seg, cache_slots);
            dmalloc(free_slots, cache_slots);
            dmalloc(seg_score, fwd.seg_total);
            CK(cudaMemset(seg_score, 0, fwd.seg_total * sizeof(uint32_t)));
            dmalloc(seg_victims, kMaxEvict);
            dmalloc(seg_admits, kMaxAdmit);
            dmalloc(seg_ctl, kCtlCount);
        }

        // Reverse arena (device only) for deletion repair.
        if (opt.algo != CIG_PR) build_reverse(xadj, adj, m);

        // Vertex state.
        dmalloc(q0, n + 1);
        dmalloc(q1, n + 1);
        dmalloc(tmp_u32, n);
        if (local_sweeps && opt.algo != CIG_PR) dmalloc(inval_done, n + 1);
        build_index(fwd, true);
        place_resident(filled, L.small_segs);
        if (opt.algo != CIG_PR) build_index(rev, false);
        if (opt.algo == CIG_PR) {
            const size_t es = pr64 ? sizeof(double) : sizeof(float);
            CK(cudaMalloc(&pr_rank, n * es));
            CK(cudaMalloc(&pr_res, n * es));
            CK(cudaMalloc(&pr_contrib, (n + 1) * es));
            if (!pr64) {
                dmalloc(pr_comp, n);
                dmalloc(pr_amend64, n);
                CK(cudaMemset(pr_amend64, 0, n * sizeof(double)));
                // FP64 residual slots for vertices of in-degree >= kPrHubInDeg.
                std::vector<std::atomic<uint32_t>> indeg(n);
                parallel_for(m, [&](uint64_t b, uint64_t e) {
                    for (uint64_t i = b; i < e; ++i) indeg[adj[i]].fetch_add(1, std::memory_order_relaxed);
                });
                uint64_t hub_deg = kPrHubInDeg;
                if (const char *e = std::getenv("CIG_PR_HUB_INDEG")) hub_deg = std::strtoull(e, nullptr, 10);
                const uint32_t words = (n + 31) / 32;
                std::vector<uint32_t> bits(words, 0), prefix(words, 0);
                uint32_t nh = 0;
                for (uint32_t w = 0; w < words; ++w) {
                    prefix[w] = nh;
                    for (uint32_t k = 0; k < 32 && 32 * w + k < n; ++k)
                        if (indeg[32 * w + k].load(std::memory_order_relaxed) >= hub_deg) {
                            bits[w] |= 1u << k;
                            ++nh;
                        }
                }
                dmalloc(pr_hub_bits, words);
                dmalloc(pr_hub_prefix, words);
                CK(cudaMemcpy(pr_hub_bits, bits.data(), words * sizeof(uint32_t), cudaMemcpyHostToDevice));
                CK(cudaMemcpy(pr_hub_prefix, prefix.data(), words * sizeof(uint32_t), cudaMemcpyHostToDevice));
                dmalloc(pr_res_hub, std::max<uint32_t>(nh, 1));
                CK(cudaMemset(pr_res_hub, 0, std::max<uint32_t>(nh, 1) * sizeof(double)));
                pr_hubs = nh;
            }
            dmalloc(pr_queued, n);
            dmalloc(aff_stamp, n);
            CK(cudaMemset(aff_stamp, 0, n * sizeof(uint32_t)));
        } else {
            dmalloc(state, n);
            dmalloc(qstamp, n);
            dmalloc(aff_stamp, n);
            dmalloc(list, n + 1);
            CK(cudaMemset(qstamp, 0, n * sizeof(uint32_t)));
            CK(cudaMemset(aff_stamp, 0, n * sizeof(uint32_t)));
        }
        ensure_batch(std::max<uint64_t>(opt.max_batch, 1024));
        CK(cudaDeviceSynchronize());
        loaded = true;
    }

    void upload_alloc(DevArena &a, const Layout &L) {
        ArenaAlloc h{};
        h.seg_bump = a.seg_used;
        h.seg_total = a.seg_total;
        std::memcpy(h.cur_next, L.cur_next, sizeof(h.cur_next));
        std::memcpy(h.cur_end, L.cur_end, sizeof(h.cur_end));
        dmalloc(a.alloc, 1);
        CK(cudaMemcpy(a.alloc, &h, sizeof(h), cudaMemcpyHostToDevice));
    }

    void build_reverse(const uint64_t *xadj, const uint32_t *adj, uint64_t m) {
        uint32_t *d_adj = nullptr, *d_cnt = nullptr;
        uint64_t *d_xadj = nullptr;
        dmalloc(d_adj, m);
        dmalloc(d_xadj, n + 1);
        dmalloc(d_cnt, n);
        CK(cudaMemcpy(d_adj, adj, m * sizeof(uint32_t), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_xadj, xadj, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice));
        CK(cudaMemset(d_cnt, 0, n * sizeof(uint32_t)));
        if (m) count_indeg<<<sms * 16, 256>>>(d_adj, m, d_cnt);
        check_launch();
        std::vector<uint32_t> indeg(n);
        CK(cudaMemcpy(indeg.data(), d_cnt, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        Layout L = plan_layout(n, indeg.data());
        const double pct = opt.arena_headroom_pct ? opt.arena_headroom_pct : 12.5;
        const uint64_t head = std::max<uint64_t>(static_cast<uint64_t>(L.used_segs * pct / 100.0) + 1,
                                                 (1ull << 20) >> kSegShift);
        rev.seg_used = L.used_segs;
        rev.seg_total = L.used_segs + head;
        rev.nverts = n;
        rev.bstatus = status;
        dmalloc(rev.dev, rev.seg_total * kSegEdges);
        dmalloc(rev.desc, n);
        CK(cudaMemcpy(rev.desc, L.desc.data(), n * sizeof(RowDesc), cudaMemcpyHostToDevice));
        CK(cudaMemset(d_cnt, 0, n * sizeof(uint32_t)));
        if (m) fill_reverse<<<sms * 16, 256>>>(d_xadj, d_adj, n, rev.desc, d_cnt, rev.dev);
        check_launch();
        CK(cudaDeviceSynchronize());
        upload_alloc(rev, L);
        dfree(d_adj);
        dfree(d_xadj);
        dfree(d_cnt);
    }

    // ------------------------------------------------------------ solve
    void init() {
        if (!loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        require_alive();
        reset_counters();
        if (opt.algo == CIG_PR) {
            if (pr64)
                pr_init_run<double>();
            else
                pr_init_run<float>();
        } else {
            dispatch([&](auto tag) { static_solve<decltype(tag)::value>(); });
        }
        finish();
        initialized = true;
    }

    // The static solve from scratch (Start, framework.cuh:1151-1182).
    template <int A>
    void static_solve() {
        launch(init_state<A>, persistent_grid(), 256, state, n, source, cc_shift);
        CK(cudaMemsetAsync(small + kFr, 0, 3 * sizeof(uint32_t), stream));
        if (A == kCc)
            launch(enqueue_all_nonempty, persistent_grid(), 256, fwd.desc, n, frontier(), status);
        else
            launch(set_single, 1, 1, q0, small + kFr, source);
        check_launch();
        run_push<A>();
    }

    // Push closure from the queued seeds (persistent, cooperative, bounded
    // grid barriers), for the static solve and for incremental batches.
    template <int A>
    void run_push() {
        const int p = prof_begin(CIG_STAGE_PUSH);
        launch_coop(push_closure<A>, kTpb, fwd.view(), state, qstamp, tags, frontier(), big_list(), n + 2,
                    local_sweeps, seg_hot, status);
        prof_end(p);
    }
    uint32_t local_sweeps = 8;  // block-local hops per closure round (CIG_LOCAL_SWEEPS; 0 = off)
    // Share of the initially resident slots given to the last segments of the
    // arena (the smallest row classes), in percent (CIG_CACHE_SMALL_PCT); a
    // negative value: the segments of the small row classes.
    double cache_small_pct = -1.0;
    // Whole batches run one push closure (after the insertions) instead of
    // one per phase (CIG_MERGE_PUSH=0: one per phase, as the per-phase calls).
    bool merge_push = true;
    uint32_t cc_shift = 0;      // CC: depth bits below the label in a value (also in Status)
    uint32_t *inval_done = nullptr;  // n + 1: vertices the invalidation sweeps expanded

    // ------------------------------------------------------------ PR
    template <class T>
    PrArrays<T> pr_arrays() {
        return PrArrays<T>{static_cast<T *>(pr_rank), static_cast<T *>(pr_res), pr_hub_bits, pr_hub_prefix, pr_res_hub,
                           pr_comp, pr_queued, q0, q1, small + kFr, static_cast<T *>(pr_contrib), small + kFinalRound,
                           n + 1};
    }

    template <class T>
    void pr_init_run() {
        auto a = pr_arrays<T>();
        launch(pr_init<T>, persistent_grid(), 256, a, n);
        const uint32_t counts[3] = {n, 0, 0};
        CK(cudaMemcpyAsync(small + kFr, counts, sizeof(counts), cudaMemcpyHostToDevice, stream));
        check_launch();
        pr_run_converge<T>();
    }

    template <class T>
    void pr_run_converge() {
        auto a = pr_arrays<T>();
        const T eps = static_cast<T>(opt.pr_epsilon);
        const int p = prof_begin(CIG_STAGE_PR);
        launch_coop(pr_converge<T>, kTpbPr, fwd.view(), a, eps, static_cast<uint32_t>(opt.pr_max_rounds), seg_hot,
                    status);
        prof_end(p);
        launch(pr_normalize_frontier<T>, persistent_grid(), 256, a);
        launch(pr_set_counts<T>, 1, 1, a);
        CK(cudaMemsetAsync(small64, 0, sizeof(double), stream));
        launch(pr_residual_l1<T>, persistent_grid(), 256, pr_arrays<T>(), n,
                                                                  reinterpret_cast<double *>(small64));
        check_launch();
    }

    template <class T>
    void pr_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                  const uint32_t *d_av, uint64_t na) {
        const NvtxRange range("cig.pr_batch");
        reserve_chunk_map(nd);
        index_upkeep(na);
        auto a = pr_arrays<T>();
        const T eps = static_cast<T>(opt.pr_epsilon);
        ++epoch;
        CK(cudaMemsetAsync(small + kTouched, 0, sizeof(uint32_t), stream));
        if (nd + na)
            launch(collect_touched, grid_for(nd + na), 256, d_du, static_cast<uint32_t>(nd), d_au,
                                                                  static_cast<uint32_t>(na), n, aff_stamp, epoch,
                                                                  touched, small + kTouched,
                                                                  static_cast<uint32_t>(2 * bcap), status);
        // r' = r + alpha (P_new^T - P_old^T) x over the touched sources.
        auto amend_pass = [&](double sign) {
            const int p = prof_begin(CIG_STAGE_PR);
            if (sizeof(T) == 4) {
                double *c64 = static_cast<double *>(pr_amend);
                launch(pr_amend_contrib64<T>, persistent_grid(), 256, fwd.desc, a, touched, small + kTouched, sign,
                       c64);
                launch(pr_amend_scatter64<T>, persistent_grid(), kTpbPr, fwd.view(), touched, small + kTouched, c64,
                       pr_amend64, status);
            } else {
                T *amend = static_cast<T *>(pr_amend);
                launch(pr_amend_contrib<T>, persistent_grid(), 256, fwd.desc, a, touched, small + kTouched,
                       static_cast<T>(sign), amend);
                launch(pr_amend_scatter<T>, persistent_grid(), kTpbPr, fwd.view(), a, touched, small + kTouched,
                       amend, eps, status);
            }
            prof_end(p);
            check_launch();
        };
        amend_pass(-1.0);
        mutate_forward_delete(d_du, d_dv, nd, true);
        mutate_forward_add(d_au, d_av, na, true);
        amend_pass(1.0);
        if (sizeof(T) == 4) launch(pr_amend_fold<T>, persistent_grid(), 256, a, pr_amend64, n, eps, status);
        pr_run_converge<T>();
    }

    // ------------------------------------------------------------ topology
    void mutate_forward_delete(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, bool with_stats) {
        mutate_delete_arena(fwd, d_du, d_dv, nd, true, with_stats);
    }
    void mutate_forward_add(const uint32_t *d_au, const uint32_t *d_av, uint64_t na, bool with_stats) {
        mutate_add_arena(fwd, d_au, d_av, na, true, with_stats);
    }

    // Source groups of a sorted key array, in key order (flags, exclusive
    // scan, scatter): group g spans keys [start[g], end[g]).
    Groups build_groups(const unsigned long long *sorted, uint64_t count, uint32_t *start, uint32_t *end,
                        uint32_t *gcount) {
        const uint32_t m = static_cast<uint32_t>(count);
        CK(cudaMemsetAsync(gcount, 0, sizeof(uint32_t), stream));
        launch(group_flags, grid_for(count), 256, sorted, m, gflags);
        size_t bytes = cub_bytes;
        CK(cub::DeviceScan::ExclusiveSum(cub, bytes, gflags, gpos, static_cast<int>(count), stream));
        launch(group_scatter, grid_for(count), 256, sorted, m, gflags, gpos, start, end, gcount);
        return Groups{start, end, gcount};
    }

    // Time the static solve (the heaviest closure, from scratch) for every
    // candidate launch shape and keep the fastest.  The solve's values are
    // unique, so re-running it leaves the maintained values unchanged; the
    // last run uses the chosen shape.
    void autotune(cig_tune_result *res) {
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "autotune covers the BFS/SSSP/CC closures");
        const uint32_t per_sm_c[] = {2, 4, 8};
        const uint32_t split_c[] = {1024, 4096, 16384};
        Tune best = tune;
        float best_ms = 1e30f;
        uint32_t tried = 0;
        for (uint32_t ps : per_sm_c) {
            for (uint32_t sp : split_c) {
                tune.per_sm = ps;
                tune.split = sp;
                float ms = 0;
                for (int rep = 0; rep < 2; ++rep) {  // first run warms caches and occupancy queries
                    CK(cudaEventRecord(ev[0], stream));
                    dispatch([&](auto tag) { static_solve<decltype(tag)::value>(); });
                    CK(cudaEventRecord(ev[1], stream));
                    finish();
                    CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
                }
                ++tried;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = tune;
                }
            }
        }
        tune = best;
        dispatch([&](auto tag) { static_solve<decltype(tag)::value>(); });
        finish();
        // Push/pull threshold of the BFS query waves: time single-source waves
        // (the first 8 vertices with out-edges) for each divisor.
        uint32_t pull_best = tune.pull_on;
        if (rev.desc) {
            std::vector<RowDesc> d = host_desc();
            std::vector<uint32_t> src;
            for (uint32_t v = 0; v < n && src.size() < 8; ++v)
                if (d[v].len) src.push_back(v);
            if (!src.empty()) {
                uint32_t *out = nullptr;
                dmalloc(out, static_cast<size_t>(src.size()) * n);
                float best_q = 1e30f;
                const uint32_t pull_c[] = {0, 8, 16, 32, 64};
                try {
                    for (uint32_t pc : pull_c) {
                        tune.pull_on = pc;
                        tune.pull_off = pc * 2;
                        cig_query_stats qs{};
                        for (int rep = 0; rep < 2; ++rep)
                            query_multi(CIG_BFS, src.data(), static_cast<uint32_t>(src.size()), 1, out, &qs);
                        ++tried;
                        if (qs.ms < best_q) {
                            best_q = static_cast<float>(qs.ms);
                            pull_best = pc;
                        }
                    }
                } catch (...) {
                    dfree(out);
                    throw;
                }
                dfree(out);
            }
        }
        tune.pull_on = pull_best;
        tune.pull_off = pull_best * 2;
        retire_graphs();  // launch shapes changed
        if (res) {
            std::memset(res, 0, sizeof(*res));
            res->blocks_per_sm = best.per_sm;
            res->split_degree = best.split;
            res->best_ms = best_ms;
            res->candidates = tried;
            res->pull_divisor = pull_best;
        }
    }

    void run_cache_service() {
        const NvtxRange range("cig.cache_service");
        const int p = prof_begin(CIG_STAGE_CACHE);
        cache_service();
        prof_end(p);
    }

    // Per-batch residency decisions of the segment table (cache.cuh), on the
    // engine stream after the insertion phase.
    void cache_service() {
        if (!refresh) return;
        const SegTable t = seg_table();
        CK(cudaMemsetAsync(seg_ctl + kCtlVictims, 0, 2 * sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(seg_ctl + kCtlHist, 0, kScoreBuckets * sizeof(uint32_t), stream));
        launch(seg_rescore, grid_for(fwd.seg_total), 256, t, static_cast<uint32_t>(fwd.seg_total));
        launch(seg_plan, 1, 32, t);
        launch(seg_pick, grid_for(fwd.seg_total), 256, t, static_cast<uint32_t>(fwd.seg_total));
        launch(seg_evict, static_cast<int>(std::min<uint64_t>(kMaxEvict, sms * 4)), 256, t, fwd.dev, fwd.host_dptr,
               status);
        launch(seg_admit, static_cast<int>(kMaxAdmit), 256, t, fwd.dev, fwd.host_dptr, status);
        check_launch();
    }

    // Sort the keys of a whole batch at once (PackedSets): fills kf/kr (forward
    // and reverse deletion keys), t1/t2 (addition keys) and their groups, and
    // sets `presorted` for the two phases that follow.  Returns false (and
    // leaves the per-phase sorts to the phases) when the fields do not fit.
    uint32_t presort_field_bits(uint64_t nd, uint64_t na) const {
        const uint64_t mx = std::max<uint64_t>(n, std::max(nd, na));
        uint32_t f = 0;
        while (f < 32 && (1ull << f) <= mx) ++f;
        return f;
    }
    bool presort_fits(uint64_t nd, uint64_t na) const { return 2 + 2 * presort_field_bits(nd, na) <= 64; }

    bool presort_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                       const uint32_t *d_av, uint64_t na) {
        const uint32_t f = presort_field_bits(nd, na);
        if (!presort_fits(nd, na)) return false;
        PackedSets ps{};
        ps.off[0] = 0;
        ps.off[1] = static_cast<uint32_t>(nd);
        ps.off[2] = static_cast<uint32_t>(2 * nd);
        ps.off[3] = static_cast<uint32_t>(2 * nd + na);
        ps.off[4] = static_cast<uint32_t>(2 * nd + 2 * na);
        ps.f = f;
        const uint64_t total = ps.off[4];
        const int p = prof_begin(CIG_STAGE_GROUP);
        CK(cudaMemsetAsync(small + kGcF, 0, 2 * sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(small + kGaF, 0, 2 * sizeof(uint32_t), stream));
        if (total) {
            launch(make_keys_batch, grid_for(total), 256, d_du, d_dv, static_cast<uint32_t>(nd), d_au, d_av,
                   static_cast<uint32_t>(na), n, ps, kc, status);
            const unsigned long long *sorted;
            size_t bytes = cub_bytes;
            // ~0 pads the small sort's tail: keys of 2 + 2F < 64 bits sort below it.
            if (total <= kSmallSortKeys) {
                launch(sort_small, 1, kSmallSortThreads, kc, static_cast<uint32_t>(total), 2 + 2 * static_cast<int>(f),
                       tc);
                sorted = tc;
            } else {
                cub::DoubleBuffer<unsigned long long> db(kc, tc);
                CK(cub::DeviceRadixSort::SortKeys(cub, bytes, db, static_cast<int>(total), 0,
                                                  2 + 2 * static_cast<int>(f), stream));
                sorted = db.Current();
            }
            launch(unpack_keys_batch, grid_for(total), 256, sorted, ps, kf, kr, t1, t2, gflags);
            bytes = cub_bytes;
            CK(cub::DeviceScan::ExclusiveSum(cub, bytes, gflags, gpos, static_cast<int>(total), stream));
            SetGroups sg{};
            sg.start[0] = gf;
            sg.end[0] = gendf;
            sg.count[0] = small + kGcF;
            sg.start[1] = gr;
            sg.end[1] = gendr;
            sg.count[1] = small + kGcR;
            sg.start[2] = gaf;
            sg.end[2] = gaendf;
            sg.count[2] = small + kGaF;
            sg.start[3] = gar;
            sg.end[3] = gaendr;
            sg.count[3] = small + kGaR;
            launch(group_scatter_batch, grid_for(total), 256, sorted, ps, gflags, gpos, sg);
        }
        prof_end(p);
        check_launch();
        presorted = true;
        return true;
    }

    // Scan-chunk map of a deletion phase: at most one chunk per 512 arena
    // slots plus one per group.  Sized before the phase's launches are
    // queued (or captured).
    void reserve_chunk_map(uint64_t nd) {
        const uint64_t need = std::max(fwd.seg_total, rev.seg_total) * (kSegEdges / kDelChunk) + nd + 1;
        if (need <= chunk_map_cap) return;
        if (capturing) throw CigError(CIG_ERR_DEVICE, "internal: scan-chunk map grows under capture");
        CK(cudaStreamSynchronize(stream));
        CK(cudaStreamSynchronize(side));
        dfree(chunk_map);
        dfree(chunk_map_r);
        dmalloc(chunk_map, need);
        dmalloc(chunk_map_r, need);
        chunk_map_cap = need;
        retire_graphs();
    }

    // Position-index upkeep before an insertion phase of `na` additions: a
    // table is rebuilt once its load factor could pass one half (every
    // addition may add a key).  Runs before the phase's launches are queued
    // or replayed; a rebuild synchronises and retires the captured graphs.
    void index_upkeep(uint64_t na) {
        if (!na) return;
        for (int a = 0; a < 2; ++a) {
            IndexBuf &b = ixb[a];
            if (!b.cap) continue;
            b.inserted += na;
            if (2 * (b.entries + b.inserted) > b.cap) {
                const int pi = prof_begin(CIG_STAGE_INDEX);
                build_index(a == 0 ? fwd : rev, a == 0);
                prof_end(pi);
                retire_graphs();
            }
        }
    }

    // Host-side accounting of the phases for the stage profiler (kept out of
    // captured code): requests per stage, sorted keys.
    void note_delete_phase(uint64_t nd) {
        if (!prof_on || !nd) return;
        prof[CIG_STAGE_DEL_SCAN].hits += 2 * nd;
        prof[CIG_STAGE_MUTATE].hits += nd;
        prof[CIG_STAGE_MUTATE_REV].hits += nd;
        prof[CIG_STAGE_GROUP].hits += 2 * nd;
    }
    void note_insert_phase(uint64_t na) {
        if (!prof_on || !na) return;
        prof[CIG_STAGE_ADD].hits += na;
        prof[CIG_STAGE_ADD_REV].hits += na;
        prof[CIG_STAGE_GROUP].hits += 2 * na;
    }

    // `zeroed`: the phase's counters were cleared by phase_begin.
    void mutate_delete_arena(DevArena &A, const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, bool forward,
                             bool with_stats, bool zeroed = false) {
        if (nd == 0) return;
        reserve_chunk_map(nd);  // before the map's address is taken below
        const uint32_t m = static_cast<uint32_t>(nd);
        unsigned long long *keys = forward ? kf : kr;
        unsigned long long *tmp = forward ? t1 : t2;
        uint32_t *groups = forward ? gf : gr;
        uint32_t *matched = forward ? mf : mr;
        uint32_t *big = forward ? bigf : bigr;
        uint32_t *gcount = small + (forward ? kGcF : kGcR);
        uint32_t *bcount = small + (forward ? kBigF : kBigR);
        uint32_t *chunks = forward ? this->chunks : chunks_r;
        uint32_t *chunk_end = forward ? this->chunk_end : chunk_end_r;
        uint32_t *ordered = forward ? this->ordered : ordered_r;
        uint32_t *firstpos = forward ? this->firstpos : firstpos_r;
        uint32_t *indexed_groups = forward ? this->indexed_groups : indexed_groups_r;
        uint32_t *compact = forward ? this->compact : compact_r;
        uint32_t *chunk_map = forward ? this->chunk_map : chunk_map_r;
        uint8_t *gtype = forward ? this->gtype : gtype_r;
        void *scan_tmp = forward ? cub : cub_r;
        size_t scan_tmp_bytes = forward ? cub_bytes : cub_r_bytes;
        int p = prof_begin(CIG_STAGE_GROUP);
        unsigned long long *sorted = keys;
        Groups grp{groups, forward ? gendf : gendr, gcount};
        if (!presorted) {
            // make_keys_del fills both kf and kr; only build them once per phase.
            if (forward || opt.algo == CIG_PR) {
                launch(make_keys_del, grid_for(nd), 256, d_du, d_dv, m, n, kf, kr, status);
                check_launch();
            }
            sorted = sort_keys(keys, tmp, nd);
            grp = build_groups(sorted, nd, groups, forward ? gendf : gendr, gcount);
        }
        if (!zeroed) CK(cudaMemsetAsync(bcount, 0, sizeof(uint32_t), cs));
        prof_end(p);
        p = prof_begin(forward ? CIG_STAGE_MUTATE : CIG_STAGE_MUTATE_REV);
        unsigned long long *stats = with_stats ? status->counters : nullptr;
        uint32_t *ccount = small + (forward ? kCompactCount : kCompactCountR);
        uint32_t *ocount = small + (forward ? kOrderedCount : kOrderedCountR);
        // Flat path: rows whose deletion requests are all distinct.
        uint32_t *icount = small + (forward ? kIndexedCount : kIndexedCountR);
        if (!zeroed) {
            CK(cudaMemsetAsync(ccount, 0, sizeof(uint32_t), cs));
            CK(cudaMemsetAsync(ocount, 0, sizeof(uint32_t), cs));
            CK(cudaMemsetAsync(icount, 0, sizeof(uint32_t), cs));
        }
        const PosIndex ix = pos_index(forward);
        launch(del_classify, persistent_grid(), 256, A.desc, sorted, grp, chunks, gtype, ordered, ocount, ix,
               indexed_groups, icount, m, firstpos, matched);
        CK(cub::DeviceScan::InclusiveSum(scan_tmp, scan_tmp_bytes, chunks, chunk_end, static_cast<int>(nd), cs));
        launch(del_chunk_map, persistent_grid(), 256, grp, chunk_end, chunk_map);
        const int ps = prof_begin(CIG_STAGE_DEL_SCAN);
        launch(del_scan, sms * del_scan_blocks_per_sm(), kMutWarps * 32, A.view(), A.desc, sorted, grp, chunk_end,
               chunk_map, m, firstpos, status->counters, forward ? seg_hot : nullptr);
        if (ix.keys) {
            // groups of more than kLaneKeys keys: one warp each, hub groups the
            // whole grid (del_index_wide); the warp list is the arena's
            // addition warp-group list, free during deletions
            uint32_t *wide = forward ? coopf : coopr;
            uint32_t *huge = forward ? hugef : huger;
            uint32_t *wcount = small + (forward ? kCoopF : kCoopR);
            uint32_t *hcount = small + (forward ? kHugeF : kHugeR);
            if (!zeroed) {
                CK(cudaMemsetAsync(wcount, 0, sizeof(uint32_t), cs));
                CK(cudaMemsetAsync(hcount, 0, sizeof(uint32_t), cs));
            }
            launch(del_index, persistent_grid(), 256, A.view(), A.desc, sorted, grp, indexed_groups, icount, firstpos,
                   ix, wide, wcount, huge, hcount, stats, status);
            launch(del_index_wide, persistent_grid(), 256, A.view(), A.desc, sorted, grp, wide, wcount, huge, hcount,
                   firstpos, ix, stats, status);
        }
        prof_end(ps);
        launch(del_apply, grid_for(nd), 256, A.view(), A.desc, sorted, m, firstpos, stats);
        launch(del_finish, persistent_grid(), 256, A.desc, sorted, grp, gtype, firstpos, compact, ccount, stats);
        // Ordered path: rows with repeated requests for a destination.
        launch(mutate_delete, persistent_grid(), kMutWarps * 32, A.view(), A.desc, sorted, grp, ordered, ocount,
               matched, big, bcount, compact, ccount, stats, status);
        launch(mutate_delete_big, sms * 4, kTpbMut, A.view(), A.desc, sorted, grp, big, bcount, matched, compact,
               ccount, stats, status);
        if (ix.keys) launch(idx_fix_ordered, persistent_grid(), 256, A.view(), A.desc, sorted, grp, ordered, ocount, ix,
                            status);
        launch(compact_rows, sms * 4, kTpbMut, A.view(), A.desc, compact, ccount, ix, status);
        prof_end(p);
        check_launch();
    }

    void mutate_add_arena(DevArena &A, const uint32_t *d_au, const uint32_t *d_av, uint64_t na, bool forward,
                          bool with_stats) {
        if (na == 0) return;
        const uint32_t m = static_cast<uint32_t>(na);
        unsigned long long *keys = forward ? kf : kr;
        unsigned long long *tmp = forward ? t1 : t2;
        uint32_t *groups = forward ? gf : gr;
        uint32_t *big = forward ? bigf : bigr;
        unsigned long long *plan = forward ? pf : prr;
        uint32_t *gcount = small + (forward ? kGcF : kGcR);
        uint32_t *bcount = small + (forward ? kBigF : kBigR);
        int p = prof_begin(CIG_STAGE_GROUP);
        unsigned long long *sorted;
        Groups grp;
        if (presorted) {
            sorted = forward ? t1 : t2;
            grp = Groups{forward ? gaf : gar, forward ? gaendf : gaendr, small + (forward ? kGaF : kGaR)};
        } else {
            if (forward || opt.algo == CIG_PR) {
                launch(make_keys_add, grid_for(na), 256, d_au, d_av, m, n, kf, kr, status);
                check_launch();
            }
            sorted = sort_keys(keys, tmp, na);
            grp = build_groups(sorted, na, groups, forward ? gendf : gendr, gcount);
        }
        CK(cudaMemsetAsync(bcount, 0, sizeof(uint32_t), cs));
        prof_end(p);
        p = prof_begin(forward ? CIG_STAGE_ADD : CIG_STAGE_ADD_REV);
        launch(plan_add, persistent_grid(), 256, A.desc, sorted, grp, plan, A.alloc);
        launch(alloc_classes, 1, 64, A.alloc, status);
        if (forward && refresh) launch(seg_assign_new, 1, 32, seg_table(), &A.alloc->seg_bump, status);
        unsigned long long *stats = with_stats ? status->counters : nullptr;
        const uint32_t *vals = forward ? d_av : d_au;
        const PosIndex ix = pos_index(forward);
        uint32_t *coop = forward ? coopf : coopr;
        uint32_t *ccount = small + (forward ? kCoopF : kCoopR);
        CK(cudaMemsetAsync(ccount, 0, sizeof(uint32_t), cs));
        launch(mutate_add, persistent_grid(), 256, A.view(), A.desc, sorted, grp, plan, A.alloc, vals, coop, ccount,
               stats, ix, status);
        launch(mutate_add_warp, persistent_grid(), 256, A.view(), A.desc, sorted, grp, plan, A.alloc, vals, coop,
               ccount, big, bcount, stats, ix, status);
        launch(mutate_add_big, sms * 2, kTpbMut, A.view(), A.desc, sorted, grp, plan, A.alloc, vals, big, bcount,
               stats, ix, status);
        prof_end(p);
        check_launch();
    }

    // ------------------------------------------------------------ batches
    // The forward and reverse rows of a presorted batch are mutated
    // concurrently: the reverse arena's kernels go to the side stream, forked
    // from and joined back into the engine stream (a fork/join of the
    // captured graph under capture).  The two touch disjoint rows, scratch
    // and counters; unsorted per-phase calls stay on one stream (their key
    // building is shared).
    template <class F, class G>
    void fork_arenas(F fwd_part, G rev_part) {
        if (!presorted) {
            fwd_part();
            rev_part();
            return;
        }
        CK(cudaEventRecord(fork_ev, stream));
        CK(cudaStreamWaitEvent(side, fork_ev, 0));
        cs = side;
        try {
            rev_part();
        } catch (...) {
            cs = stream;
            throw;
        }
        cs = stream;
        fwd_part();
        CK(cudaEventRecord(join_ev, side));
        CK(cudaStreamWaitEvent(stream, join_ev, 0));
    }

    struct InBatch {
        bool &flag;
        explicit InBatch(bool &f) : flag(f) { flag = true; }
        ~InBatch() { flag = false; }
    };

    // `push` false: leave the re-propagation from the repaired vertices to
    // the insertion phase's push closure (whole batches, merge_push): their
    // frontier stays queued and the insertion seeds join it, so one closure
    // converges to the final graph's values.  The values after a whole batch
    // are the unique fixpoint of the final graph either way; only the
    // intermediate deletion-phase values, which a whole batch does not
    // expose, are skipped.
    template <int A>
    void delete_phase_dev(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, bool push = true) {
        const InBatch ib(in_batch);
        const uint32_t *ep = small + kEpoch;
        // frontier, affected and deletion-path counters of both arenas
        static_assert(kSmallCount == 32 && kEpoch == 23, "phase_begin clears one 32-word counter block");
        const uint32_t mask = (0x3Fu << kFr) | (1u << kBigF) | (1u << kBigR) | (1u << kCompactCount) |
                              (1u << kOrderedCount) | (1u << kIndexedCount) | (1u << kInvalDone) |
                              (1u << kCompactCountR) | (1u << kOrderedCountR) | (1u << kIndexedCountR) |
                              (1u << kCoopF) | (1u << kCoopR) | (1u << kHugeF) | (1u << kHugeR);
        launch(phase_begin, 1, 32, small + kEpoch, small, mask);
        int p = prof_begin(CIG_STAGE_SEED);
        if (nd)
            launch(seed_deletions<A>, grid_for(nd), 256, d_du, d_dv, static_cast<uint32_t>(nd), n, state,
                                                                aff_stamp, ep, list, small + kAff, n + 1, status);
        prof_end(p);
        check_launch();
        fork_arenas([&] { mutate_delete_arena(fwd, d_du, d_dv, nd, true, true, true); },
                    [&] { mutate_delete_arena(rev, d_du, d_dv, nd, false, false, true); });
        p = prof_begin(CIG_STAGE_INVAL);
        launch_coop(inval_closure<A>, kTpb, fwd.view(), state, aff_stamp, ep, list, small + kAff, n + 1,
                    big_list(), n + 2, local_sweeps, inval_done, small + kInvalDone, small + kAffTotal, seg_hot,
                    status);
        prof_end(p);
        p = prof_begin(CIG_STAGE_PULL);
        launch(reset_affected<A>, persistent_grid(), 256, list, small + kAffTotal, state, cc_shift);
        const BigList pull_big = big_list();
        // One resident wave (__launch_bounds__(kTpb, 4)): a second wave of
        // blocks would start its few rows only after the first wave ends.
        launch(pull_repair<A>, sms * 4, kTpb, rev.view(), state, aff_stamp, ep, list, small + kAffTotal, pull_big,
               status);
        launch(pull_deferred<A>, persistent_grid(), kTpb, rev.view(), state, aff_stamp, ep, pull_big, status);
        launch(enqueue_affected<A>, persistent_grid(), 256, list, small + kAffTotal, state, frontier(), status);
        prof_end(p);
        check_launch();
        if (push) run_push<A>();
    }

    // `fresh` false: keep the frontier the deletion phase left queued.
    template <int A>
    void insert_phase_dev(const uint32_t *d_au, const uint32_t *d_av, uint64_t na, bool fresh = true) {
        const InBatch ib(in_batch);
        if (fresh) CK(cudaMemsetAsync(small + kFr, 0, 3 * sizeof(uint32_t), stream));
        fork_arenas([&] { mutate_add_arena(fwd, d_au, d_av, na, true, true); },
                    [&] { mutate_add_arena(rev, d_au, d_av, na, false, false); });
        int p = prof_begin(CIG_STAGE_SEED);
        if (na)
            launch(seed_insertions<A>, grid_for(na), 256, d_au, d_av, static_cast<uint32_t>(na), n, state,
                                                                 qstamp, tags, frontier(), status);
        prof_end(p);
        check_launch();
        run_push<A>();
    }

    // Copy host update arrays into the device batch buffers (pinned staging).
    // Host update arrays go through the pinned staging buffer.  Reading the
    // caller's arrays (cold in host DRAM) is what costs: one thread moves
    // ~6 GB/s, so the calling thread and stage_workers persistent workers
    // each copy one part of every array.  The workers spin for kStageSpin
    // after a job before they sleep on a condition variable, so in a stream
    // of batches a call finds them awake (a wake-up from sleep costs about
    // what the split saves).  Then the host-to-device copies are queued on
    // the engine stream.  The previous call's copies have completed (every
    // call ends with a synchronisation), so the buffer is free.
    // Up to 7 workers, leaving one host thread free.
    const int stage_workers = std::max(1, std::min(7, static_cast<int>(hw_threads()) - 1));
    static constexpr auto kStageSpin = std::chrono::milliseconds(3);
    struct Stager {
        std::vector<std::thread> threads;
        std::mutex m;
        std::condition_variable go;
        std::atomic<uint64_t> gen{0};
        std::atomic<int> pending{0};
        std::atomic<bool> stop{false};
        std::function<void(int)> job;
    } stager;

    void stager_run(const std::function<void(int)> &job) {
        Stager &S = stager;
        if (S.threads.empty())
            for (int w = 0; w < stage_workers; ++w)
                S.threads.emplace_back([&S, w] {
                    uint64_t seen = 0;
                    for (;;) {
                        const auto t0 = std::chrono::steady_clock::now();
                        while (S.gen.load(std::memory_order_acquire) == seen && !S.stop.load(std::memory_order_relaxed) &&
                               std::chrono::steady_clock::now() - t0 < kStageSpin)
                            std::this_thread::yield();
                        if (S.gen.load(std::memory_order_acquire) == seen) {
                            std::unique_lock<std::mutex> lk(S.m);
                            S.go.wait(lk, [&] { return S.stop.load() || S.gen.load() != seen; });
                        }
                        if (S.stop.load()) return;
                        seen = S.gen.load(std::memory_order_acquire);
                        S.job(w + 1);  // unchanged until every worker reported
                        S.pending.fetch_sub(1, std::memory_order_release);
                    }
                });
        S.job = job;
        S.pending.store(stage_workers, std::memory_order_relaxed);
        {
            std::lock_guard<std::mutex> lk(S.m);
            S.gen.fetch_add(1, std::memory_order_release);
        }
        S.go.notify_all();
        job(0);
        while (S.pending.load(std::memory_order_acquire) != 0) std::this_thread::yield();
    }

    void stager_stop() {
        {
            std::lock_guard<std::mutex> lk(stager.m);
            stager.stop.store(true);
        }
        stager.go.notify_all();
        for (auto &t : stager.threads) t.join();
        stager.threads.clear();
    }

    void stage_batch(const uint32_t *hdu, const uint32_t *hdv, uint64_t nd, const uint32_t *hau, const uint32_t *hav,
                     uint64_t na) {
        const NvtxRange range("cig.stage_host_arrays");
        if ((nd && (!hdu || !hdv)) || (na && (!hau || !hav))) throw CigError(CIG_ERR_ARG, "null update array");
        const uint32_t *src[4] = {hdu, hdv, hau, hav};
        const uint64_t cnt[4] = {nd, nd, na, na};
        uint32_t *dev[4] = {du, dv, au, av};
        // Caller arrays in page-locked host memory (cudaHostAlloc,
        // cudaHostRegister, a pinned torch tensor) are copied by DMA
        // straight from where they are; the call ends synchronised, so they
        // may change again once it returns.
        bool all_pinned = true;
        for (int a = 0; a < 4 && all_pinned; ++a) {
            if (!cnt[a]) continue;
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, src[a]) != cudaSuccess) {
                cudaGetLastError();
                all_pinned = false;
            } else {
                all_pinned = at.type == cudaMemoryTypeHost;
            }
        }
        if (all_pinned) {
            for (int a = 0; a < 4; ++a)
                if (cnt[a])
                    CK(cudaMemcpyAsync(dev[a], src[a], cnt[a] * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
            return;
        }
        uint32_t *dst[4] = {stage, stage + bcap, stage + 2 * bcap, stage + 3 * bcap};
        auto copy = [&](int part, int parts) {
            for (int a = 0; a < 4; ++a) {
                const uint64_t q = (cnt[a] + parts - 1) / parts;
                const uint64_t b = std::min<uint64_t>(cnt[a], static_cast<uint64_t>(part) * q);
                const uint64_t e = std::min<uint64_t>(cnt[a], b + q);
                if (e > b) std::memcpy(dst[a] + b, src[a] + b, (e - b) * sizeof(uint32_t));
            }
        };
        if (nd + na >= (1u << 16))
            stager_run([&](int part) { copy(part, stage_workers + 1); });
        else
            copy(0, 1);
        for (int a = 0; a < 4; ++a)
            if (cnt[a])
                CK(cudaMemcpyAsync(dev[a], dst[a], cnt[a] * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    }

    void require_ready() {
        require_alive();
        if (!initialized) throw CigError(CIG_ERR_ARG, "call cig_init first");
    }

    void delete_phase_host(const uint32_t *hu, const uint32_t *hv, uint64_t nd, cig_batch_stats *s) {
        const NvtxRange range("cig.delete_phase");
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank applies whole batches (cig_apply_batch)");
        ensure_batch(nd);
        reset_counters();
        CK(cudaEventRecord(ev[0], stream));
        stage_batch(hu, hv, nd, nullptr, nullptr, 0);
        note_delete_phase(nd);
        reserve_chunk_map(nd);
        dispatch([&](auto tag) {
            run_graphed(1, nd, 0, [&] { delete_phase_dev<decltype(tag)::value>(du, dv, nd); });
        });
        CK(cudaEventRecord(ev[1], stream));
        finish();
        fill_stats(s, nd, 0, true, false);
    }

    void insert_phase_host(const uint32_t *hu, const uint32_t *hv, uint64_t na, cig_batch_stats *s) {
        const NvtxRange range("cig.insert_phase");
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank applies whole batches (cig_apply_batch)");
        ensure_batch(na);
        reset_counters();
        CK(cudaEventRecord(ev[1], stream));
        stage_batch(nullptr, nullptr, 0, hu, hv, na);
        note_insert_phase(na);
        index_upkeep(na);
        dispatch([&](auto tag) {
            run_graphed(2, 0, na, [&] { insert_phase_dev<decltype(tag)::value>(au, av, na); });
        });
        CK(cudaEventRecord(ev[2], stream));
        cache_service_graphed();
        CK(cudaEventRecord(ev[3], stream));
        finish();
        fill_stats(s, 0, na, false, true);
    }

    // The launches of one traversal batch on the engine stream: whole-batch
    // key sort and deletion phase, then insertion phase (on the presorted
    // keys), then the segment-table service.  The three parts are queued
    // directly or each replayed from a graph (run_graphed), with the phase
    // events e1, e2 recorded between them on the stream, so per-phase device
    // times stay exact for every batch.  Caller arrays are first copied into
    // the engine's batch buffers, whose addresses the graphs hold.
    // `mutation_after` (a query wave's event) keeps the batch on direct
    // launches.
    void traversal_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                         const uint32_t *d_av, uint64_t na, cudaEvent_t mutation_after, cudaEvent_t e1,
                         cudaEvent_t e2) {
        const NvtxRange range("cig.batch");
        note_delete_phase(nd);
        note_insert_phase(na);
        index_upkeep(na);
        reserve_chunk_map(nd);
        if (mutation_after || !use_graphs) {
            dispatch([&](auto tag) {
                constexpr int A = decltype(tag)::value;
                presort_batch(d_du, d_dv, nd, d_au, d_av, na);
                if (mutation_after) CK(cudaStreamWaitEvent(stream, mutation_after, 0));
                delete_phase_dev<A>(d_du, d_dv, nd, !merge_push);
                CK(cudaEventRecord(e1, stream));
                insert_phase_dev<A>(d_au, d_av, na, !merge_push);
                CK(cudaEventRecord(e2, stream));
                presorted = false;
            });
            run_cache_service();
            return;
        }
        const uint32_t *src[4] = {d_du, d_dv, d_au, d_av};
        uint32_t *dst[4] = {du, dv, au, av};
        const uint64_t cnt[4] = {nd, nd, na, na};
        for (int a = 0; a < 4; ++a)
            if (cnt[a] && src[a] != dst[a])
                CK(cudaMemcpyAsync(dst[a], src[a], cnt[a] * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream));
        dispatch([&](auto tag) {
            constexpr int A = decltype(tag)::value;
            bool sorted = false;
            run_graphed(3, nd, na, [&] {
                sorted = presort_batch(du, dv, nd, au, av, na);
                delete_phase_dev<A>(du, dv, nd, !merge_push);
            });
            // A replay runs no host code: the whole-batch sort's outcome is
            // a function of the shape.
            presorted = sorted || presort_fits(nd, na);
            CK(cudaEventRecord(e1, stream));
            run_graphed(4, nd, na, [&] { insert_phase_dev<A>(au, av, na, !merge_push); });
            presorted = false;
            CK(cudaEventRecord(e2, stream));
        });
        cache_service_graphed();
    }

    void cache_service_graphed() {
        if (refresh)
            run_graphed(5, 0, 0, [&] { run_cache_service(); });
        else
            run_cache_service();
    }

    // `mutation_after` (optional): an event the topology changes must wait
    // for (a query wave still reading the rows); the key sort runs before it.
    void apply_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                     const uint32_t *d_av, uint64_t na, cig_batch_stats *s, cudaEvent_t mutation_after = nullptr) {
        if (opt.algo == CIG_PR) {
            if (mutation_after) CK(cudaStreamWaitEvent(stream, mutation_after, 0));
            if (pr64)
                pr_batch<double>(d_du, d_dv, nd, d_au, d_av, na);
            else
                pr_batch<float>(d_du, d_dv, nd, d_au, d_av, na);
            CK(cudaEventRecord(ev[1], stream));
            CK(cudaEventRecord(ev[2], stream));
            run_cache_service();
        } else {
            traversal_batch(d_du, d_dv, nd, d_au, d_av, na, mutation_after, ev[1], ev[2]);
        }
        CK(cudaEventRecord(ev[3], stream));
        finish();
        fill_stats(s, nd, na, true, true);
    }

    void apply_batch_host(const uint32_t *hdu, const uint32_t *hdv, uint64_t nd, const uint32_t *hau,
                          const uint32_t *hav, uint64_t na, cig_batch_stats *s, cudaEvent_t mutation_after = nullptr) {
        require_ready();
        ensure_batch(std::max(nd, na));
        reset_counters();
        CK(cudaEventRecord(ev[0], stream));
        stage_batch(hdu, hdv, nd, hau, hav, na);
        apply_batch(du, dv, nd, au, av, na, s, mutation_after);
    }

    void apply_batch_device(const uint32_t *ddu, const uint32_t *ddv, uint64_t nd, const uint32_t *dau,
                            const uint32_t *dav, uint64_t na, cig_batch_stats *s) {
        require_ready();
        if ((nd && (!ddu || !ddv)) || (na && (!dau || !dav))) throw CigError(CIG_ERR_ARG, "null update array");
        ensure_batch(std::max(nd, na));
        reset_counters();
        CK(cudaEventRecord(ev[0], stream));
        apply_batch(ddu, ddv, nd, dau, dav, na, s);
    }

    // The batched form: `count` batches (device arrays) queued back to back
    // with one host synchronisation at the end.  Per batch the counters are
    // snapshotted on the device and, if asked, the value digest is computed
    // into a device slot, so every batch's result stays checkable.
    std::vector<cudaEvent_t> bev;
    unsigned long long *bsnap = nullptr, *bdig = nullptr;
    uint32_t bsnap_cap = 0;

    void apply_batches_device(const cig_update_batch *b, uint32_t count, cig_batch_stats *stats,
                              uint64_t *digests) {
        require_ready();
        if (!b && count) throw CigError(CIG_ERR_ARG, "null batch list");
        if (digests && opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank has no integer digest");
        uint64_t mx = 0;
        for (uint32_t i = 0; i < count; ++i) {
            if ((b[i].nd && (!b[i].del_u || !b[i].del_v)) || (b[i].na && (!b[i].add_u || !b[i].add_v)))
                throw CigError(CIG_ERR_ARG, "null update array");
            mx = std::max(mx, std::max(b[i].nd, b[i].na));
        }
        if (!count) return;
        ensure_batch(mx);
        if (count > bsnap_cap) {
            CK(cudaStreamSynchronize(stream));
            dfree(bsnap);
            dfree(bdig);
            dmalloc(bsnap, static_cast<size_t>(count) * 40);
            dmalloc(bdig, count);
            bsnap_cap = count;
        }
        while (bev.size() < 4ull * count) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            bev.push_back(e);
        }
        // The stage profiler resolves once per call: keep a profiled batched
        // call on direct launches (a graph replayed twice in one call would
        // leave only its last replay's event times).
        const bool graphs_saved = use_graphs;
        if (prof_on) use_graphs = false;
        struct Restore {
            bool &flag;
            bool value;
            ~Restore() { flag = value; }
        } restore{use_graphs, graphs_saved};
        std::vector<uint64_t> launches(count), replays(count);
        for (uint32_t i = 0; i < count; ++i) {
            const uint64_t l0 = n_launch, r0 = graph_replays;
            reset_counters();
            cudaEvent_t *e = bev.data() + 4ull * i;
            CK(cudaEventRecord(e[0], stream));
            if (opt.algo == CIG_PR) {
                if (pr64)
                    pr_batch<double>(b[i].del_u, b[i].del_v, b[i].nd, b[i].add_u, b[i].add_v, b[i].na);
                else
                    pr_batch<float>(b[i].del_u, b[i].del_v, b[i].nd, b[i].add_u, b[i].add_v, b[i].na);
                CK(cudaEventRecord(e[1], stream));
                CK(cudaEventRecord(e[2], stream));
                run_cache_service();
            } else {
                traversal_batch(b[i].del_u, b[i].del_v, b[i].nd, b[i].add_u, b[i].add_v, b[i].na, nullptr, e[1],
                                e[2]);
            }
            CK(cudaEventRecord(e[3], stream));
            if (digests) {
                CK(cudaMemsetAsync(bdig + i, 0, sizeof(unsigned long long), stream));
                launch(value_digest, persistent_grid(), 256, state, n, bdig + i, cc_shift);
            }
            CK(cudaMemcpyAsync(bsnap + 40ull * i, status->counters, 40 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToDevice, stream));
            check_launch();
            launches[i] = n_launch - l0;
            replays[i] = graph_replays - r0;
        }
        finish();
        std::vector<unsigned long long> snap(40ull * count);
        CK(cudaMemcpy(snap.data(), bsnap, snap.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        if (digests) {
            static_assert(sizeof(unsigned long long) == sizeof(uint64_t), "digest width");
            CK(cudaMemcpy(digests, bdig, count * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        }
        for (uint32_t i = 0; i < count; ++i)
            if (stats) {
                fill_stats_from(stats + i, snap.data() + 40ull * i, bev.data() + 4ull * i, launches[i], b[i].nd,
                                b[i].na, true, true);
                stats[i].graph_replays = replays[i];
            }
    }

    void fill_stats(cig_batch_stats *s, uint64_t nd, uint64_t na, bool del, bool ins) {
        fill_stats_from(s, h_status->counters, ev, n_launch - launch_mark, nd, na, del, ins);
        if (s) s->graph_replays = graph_replays - replay_mark;
    }

    void fill_stats_from(cig_batch_stats *s, const unsigned long long *c, const cudaEvent_t *evs, uint64_t launches,
                         uint64_t nd, uint64_t na, bool del, bool ins) {
        if (!s) return;
        std::memset(s, 0, sizeof(*s));
        s->requested_deletes = nd;
        s->missing_deletes = nd >= c[kCntRemoved] ? nd - c[kCntRemoved] : 0;
        s->requested_additions = na;
        s->invalid_additions = ins ? c[kCntInvalid] : 0;
        s->changed_sources = c[kCntChanged];
        s->relocated_rows = c[kCntRelocated];
        s->affected = c[kCntAffected];
        s->seeds = c[kCntSeeds];
        s->rounds = c[kCntRounds];
        s->edges_scanned = c[kCntEdges];
        s->edges_scanned_cached = c[kCntEdgesCached];
        s->vertices_expanded = c[kCntExpanded];
        s->cache_segments_loaded = c[kCntSegLoaded];
        s->cache_segments_evicted = c[kCntSegEvicted];
        s->pr_rounds = c[kCntPrRounds];
        s->kernel_launches = launches;
        auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
                cudaGetLastError();  // leave no error behind for the next call
                return -1.0;
            }
            return static_cast<double>(ms);
        };
        if (del) s->ms_delete = elapsed(evs[0], evs[1]);
        if (ins) {
            s->ms_insert = elapsed(evs[1], evs[2]);
            s->ms_cache = elapsed(evs[2], evs[3]);
        }
        if (opt.algo == CIG_PR) {
            double l1 = 0;
            cudaMemcpy(&l1, small64, sizeof(double), cudaMemcpyDeviceToHost);
            s->pr_residual_l1 = l1;
        }
        last_nd = nd;
        last_na = na;
    }

    // ------------------------------------------------------------ reads
    void get_values(uint32_t *out_values, uint32_t *out_parents) {
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank has no integer values (cig_get_pr)");
        launch(unpack_values, persistent_grid(), 256, state, n, out_values ? tmp_u32 : nullptr,
               out_parents ? tmp_u32 : nullptr, cc_shift);
        check_launch();
        CK(cudaMemcpyAsync(out_values ? out_values : out_parents, tmp_u32, n * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void get_pr(float *rank, float *res, double *rank64, double *res64) {
        require_ready();
        if (opt.algo != CIG_PR) throw CigError(CIG_ERR_ARG, "not a PageRank handle");
        float *dr = nullptr, *ds = nullptr;
        double *dr64 = nullptr, *ds64 = nullptr;
        if (rank) dmalloc(dr, n);
        if (res) dmalloc(ds, n);
        if (rank64) dmalloc(dr64, n);
        if (res64) dmalloc(ds64, n);
        if (pr64)
            launch(pr_export<double>, persistent_grid(), 256, pr_arrays<double>(), n, dr, ds, dr64, ds64);
        else
            launch(pr_export<float>, persistent_grid(), 256, pr_arrays<float>(), n, dr, ds, dr64, ds64);
        check_launch();
        if (rank) CK(cudaMemcpyAsync(rank, dr, n * sizeof(float), cudaMemcpyDeviceToHost, stream));
        if (res) CK(cudaMemcpyAsync(res, ds, n * sizeof(float), cudaMemcpyDeviceToHost, stream));
        if (rank64) CK(cudaMemcpyAsync(rank64, dr64, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
        if (res64) CK(cudaMemcpyAsync(res64, ds64, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        dfree(dr);
        dfree(ds);
        dfree(dr64);
        dfree(ds64);
    }

    uint64_t digest() {
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank has no integer values");
        CK(cudaMemsetAsync(small64 + 1, 0, sizeof(unsigned long long), stream));
        launch(value_digest, persistent_grid(), 256, state, n, small64 + 1, cc_shift);
        check_launch();
        unsigned long long h = 0;
        CK(cudaMemcpyAsync(&h, small64 + 1, sizeof(h), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        return h;
    }

    // ------------------------------------------------------------ multi-source queries
    // Queries run on their own stream with their own status word and buffers,
    // ordered after the updates already issued on the engine stream.  They
    // read the forward rows (cache or zero-copy) and change no engine state.
    cudaStream_t qstream = nullptr;
    Status *qstatus = nullptr;
    Status *h_qstatus = nullptr;
    cudaEvent_t q_ev[3] = {};
    uint32_t *ms_dist = nullptr;
    unsigned long long *ms_visit = nullptr, *ms_mask0 = nullptr, *ms_mask1 = nullptr;
    uint32_t *ms_q0 = nullptr, *ms_q1 = nullptr, *ms_small = nullptr, *ms_src = nullptr, *ms_out = nullptr;
    uint64_t ms_out_cap = 0;
    BigRow *ms_big = nullptr;

    // Bottom-up switch of a BFS wave of kw sources: frontier above n/pull_on
    // vertices (then at least n/pull_off); needs the device in-edge arena.
    // Only narrow waves pull: the thread-per-vertex bottom-up scan cut a
    // 64-source wave's edge-scans 2.4x on RMAT s24 yet ran 14 % slower, while
    // single-source waves ran 3.4x faster.
    MsPull ms_pull(uint32_t kw) const {
        MsPull p{};
        if (opt.algo == CIG_PR || !rev.desc || !tune.pull_on || kw > tune.pull_width) return p;
        p.rev = rev.view();
        p.n = n;
        p.full = kw >= 64 ? ~0ull : ((1ull << kw) - 1);
        p.on = std::max<uint32_t>(1, n / tune.pull_on);
        p.off = std::max<uint32_t>(1, n / tune.pull_off);
        return p;
    }

    void alloc_queries() {
        if (qstream) return;
        CK(cudaStreamCreateWithFlags(&qstream, cudaStreamNonBlocking));
        for (auto &e : q_ev) CK(cudaEventCreate(&e));
        dmalloc(qstatus, 1);
        CK(cudaHostAlloc(reinterpret_cast<void **>(&h_qstatus), sizeof(Status), cudaHostAllocDefault));
        dmalloc(ms_dist, static_cast<size_t>(n) * kMsWidth);
        dmalloc(ms_visit, n);
        dmalloc(ms_mask0, n);
        dmalloc(ms_mask1, n);
        dmalloc(ms_q0, n + 1);
        dmalloc(ms_q1, n + 1);
        dmalloc(ms_small, 8);
        dmalloc(ms_src, kMsWidth);
        dmalloc(ms_big, kBigRowCap);
    }

    void free_queries() {
        if (qstream) cudaStreamSynchronize(qstream);
        for (auto &e : q_ev)
            if (e) cudaEventDestroy(e);
        dfree(qstatus);
        if (h_qstatus) cudaFreeHost(h_qstatus);
        h_qstatus = nullptr;
        dfree(ms_dist);
        dfree(ms_visit);
        dfree(ms_mask0);
        dfree(ms_mask1);
        dfree(ms_q0);
        dfree(ms_q1);
        dfree(ms_small);
        dfree(ms_src);
        dfree(ms_big);
        dfree(ms_out);
        if (qstream) cudaStreamDestroy(qstream);
        qstream = nullptr;
    }

    // k sources in waves of `width` (1..64) sources; results k x n source-major
    // in device memory `out`.  width 64 is the batched form, width 1 the plain
    // per-source form over the same kernels.
    void query_multi(int algo, const uint32_t *sources, uint32_t k, uint32_t width, uint32_t *out,
                     cig_query_stats *qs) {
        const uint64_t launches0 = n_launch;
        const uint32_t waves = query_launch(algo, sources, k, width, out);
        query_finish(qs, waves, n_launch - launches0);
    }

    // Queue the waves of a query on qstream (after the updates already queued
    // on the engine stream); q_ev[2] marks their end.  Returns the wave count.
    // The forward view as the query kernels see it (a bounds-check build
    // reports into the query status word).
    AdjView query_view() const {
        AdjView v = fwd.view();
#ifdef CIG_BOUNDS_CHECK
        v.bst = qstatus;
#endif
        return v;
    }

    uint32_t query_launch(int algo, const uint32_t *sources, uint32_t k, uint32_t width, uint32_t *out) {
        const NvtxRange range("cig.query");
        if (!loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        require_alive();
        if (algo != CIG_BFS && algo != CIG_SSSP) throw CigError(CIG_ERR_ARG, "queries are BFS or SSSP");
        if (!sources || !out) throw CigError(CIG_ERR_ARG, "null sources or output");
        if (width == 0 || width > kMsWidth) throw CigError(CIG_ERR_ARG, "wave width must be 1..64");
        for (uint32_t j = 0; j < k; ++j)
            if (sources[j] >= n) throw CigError(CIG_ERR_ARG, "query source out of range");
        alloc_queries();
        CK(cudaMemsetAsync(qstatus, 0, sizeof(Status), qstream));
        CK(cudaEventRecord(q_ev[0], stream));
        CK(cudaStreamWaitEvent(qstream, q_ev[0], 0));
        CK(cudaEventRecord(q_ev[1], qstream));
        uint32_t waves = 0;
        for (uint32_t j0 = 0; j0 < k; j0 += width, ++waves) {
            const uint32_t kw = std::min(width, k - j0);
            CK(cudaMemsetAsync(ms_dist, 0xFF, static_cast<size_t>(n) * width * sizeof(uint32_t), qstream));
            CK(cudaMemsetAsync(ms_mask0, 0, n * sizeof(unsigned long long), qstream));
            CK(cudaMemsetAsync(ms_mask1, 0, n * sizeof(unsigned long long), qstream));
            if (algo == CIG_BFS)
                CK(cudaMemsetAsync(ms_visit, 0, n * sizeof(unsigned long long), qstream));
            CK(cudaMemsetAsync(ms_small, 0, 8 * sizeof(uint32_t), qstream));
            CK(cudaMemcpyAsync(ms_src, sources + j0, kw * sizeof(uint32_t), cudaMemcpyHostToDevice, qstream));
            const MsFrontier fr{ms_q0, ms_q1, ms_small, ms_mask0, ms_mask1, n + 1};
            const BigList bl{ms_big, ms_small + 3, kBigRowCap, tune.split};
            ms_seed<<<1, kMsWidth, 0, qstream>>>(ms_src, kw, ms_dist, width, algo == CIG_BFS ? ms_visit : nullptr,
                                                 fr, qstatus);
            ++n_launch;
            if (algo == CIG_BFS)
                launch_coop_on(qstream, ms_closure<kBfs>, kTpbMs, query_view(), ms_dist, width, ms_visit, fr, bl, n + 2,
                               ms_pull(kw), qstatus);
            else if (opt.flags & CIG_FLAG_WEIGHT_U255)
                launch_coop_on(qstream, ms_closure<kSsspU>, kTpbMs, query_view(), ms_dist, width,
                               static_cast<unsigned long long *>(nullptr), fr, bl, n + 2, MsPull{}, qstatus);
            else
                launch_coop_on(qstream, ms_closure<kSssp>, kTpbMs, query_view(), ms_dist, width,
                               static_cast<unsigned long long *>(nullptr), fr, bl, n + 2, MsPull{}, qstatus);
            ms_transpose<<<(n + kMsTile - 1) / kMsTile, 256, 0, qstream>>>(ms_dist, n, width, kw,
                                                                         out + static_cast<uint64_t>(j0) * n);
            ++n_launch;
            check_launch();
        }
        CK(cudaEventRecord(q_ev[2], qstream));
        return waves;
    }

    // Wait for the queued query, check its status, fill its stats.
    void query_finish(cig_query_stats *qs, uint32_t waves, uint64_t launches) {
        CK(cudaStreamSynchronize(qstream));
        CK(cudaMemcpy(h_qstatus, qstatus, sizeof(Status), cudaMemcpyDeviceToHost));
        if (h_qstatus->err) {
            std::string what;
            if (h_qstatus->err & kErrRounds) what += "round bound exceeded; ";
            if (h_qstatus->err & kErrBarrier) what += "grid barrier wait limit exceeded; ";
            if (h_qstatus->err & kErrQueue) what += "work queue overflow; ";
            if (h_qstatus->err & kErrBounds) what += "device index out of bounds (bounds-check build); ";
            throw CigError(CIG_ERR_LIMIT, "query: device reported: " + what + "info=" +
                                              std::to_string(h_qstatus->err_info));
        }
        if (qs) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, q_ev[1], q_ev[2]));
            std::memset(qs, 0, sizeof(*qs));
            qs->ms = ms;
            qs->edges_scanned = h_qstatus->counters[kCntPush + 0];
            qs->edges_scanned_cached = h_qstatus->counters[kCntPush + 1];
            qs->rows_expanded = h_qstatus->counters[kCntPush + 2];
            qs->source_edges = h_qstatus->counters[kCntSrcEdges];
            qs->rounds = h_qstatus->counters[kCntRounds];
            qs->waves = waves;
            qs->kernel_launches = launches;
        }
    }

    // Host-output form: k x n values copied to host memory `out`.
    void query_multi_host(int algo, const uint32_t *sources, uint32_t k, uint32_t *out) {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        if (!loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        const uint64_t need = static_cast<uint64_t>(std::min<uint32_t>(k, kMsWidth)) * n;
        if (need > ms_out_cap) {
            dfree(ms_out);
            dmalloc(ms_out, need);
            ms_out_cap = need;
        }
        for (uint32_t j0 = 0; j0 < k; j0 += kMsWidth) {
            const uint32_t kw = std::min(kMsWidth, k - j0);
            query_multi(algo, sources + j0, kw, kMsWidth, ms_out, nullptr);
            CK(cudaMemcpy(out + static_cast<uint64_t>(j0) * n, ms_out, static_cast<uint64_t>(kw) * n * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost));
        }
    }


    // ------------------------------------------------------------ serving
    struct ServeItem {
        uint64_t ticket = 0;
        cig_request r{};
        std::vector<uint32_t> upd;  // du | dv | au | av of an update
        double t_submit = 0;
    };
    struct Serve {
        std::mutex mu;
        std::condition_variable cv_work, cv_done, cv_space;
        std::deque<ServeItem> queue;
        std::unordered_map<uint64_t, cig_result> results;
        std::unordered_set<uint64_t> open;  // submitted, result not yet taken
        uint64_t next_ticket = 1;
        uint64_t pending = 0;
        bool stop = false;
        std::thread worker;
        cig_serve_options opt{};
        std::chrono::steady_clock::time_point t0;
        uint64_t chunk_cap = 0;  // largest update phase chunk the budget admits
        uint32_t wave_cap = 64;  // sources per wave the budget admits
        unsigned long long *digests = nullptr;  // device, one per wave slot
        uint32_t *rows = nullptr;               // device wave_cap x n
    };
    std::unique_ptr<Serve> srv;
    std::atomic<bool> serving{false};
    // Device bytes per slot of the per-batch buffers that ensure_batch sizes.
    static constexpr uint64_t kBytesPerBatchSlot = 384;

    double serve_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - srv->t0).count();
    }

    void serve_start(const cig_serve_options *o) {
        require_ready();
        if (serving) throw CigError(CIG_ERR_STATE, "already serving");
        auto sv = std::make_unique<Serve>();
        if (o) sv->opt = *o;
        if (sv->opt.max_wave == 0 || sv->opt.max_wave > kMsWidth) sv->opt.max_wave = kMsWidth;
        if (sv->opt.max_pending == 0) sv->opt.max_pending = 4096;
        uint64_t budget = sv->opt.budget_bytes;
        if (!budget) {
            size_t fr = 0, tot = 0;
            CK(cudaMemGetInfo(&fr, &tot));
            budget = fr / 2;
        }
        // Half of the budget for update buffers, half for wave results.
        sv->chunk_cap = std::max<uint64_t>(1024, std::min<uint64_t>(0x40000000ull, budget / 2 / kBytesPerBatchSlot));
        const uint64_t rows = budget / 2 / (static_cast<uint64_t>(n) * sizeof(uint32_t));
        sv->wave_cap = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(sv->opt.max_wave, rows)));
        alloc_queries();
        dmalloc(sv->digests, kMsWidth);
        dmalloc(sv->rows, static_cast<size_t>(sv->wave_cap) * n);
        sv->t0 = std::chrono::steady_clock::now();
        srv = std::move(sv);
        serving = true;
        srv->worker = std::thread([this] { serve_loop(); });
    }

    void serve_stop() {
        if (!srv) return;
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->stop = true;
        }
        srv->cv_work.notify_all();
        if (srv->worker.joinable()) srv->worker.join();
        dfree(srv->digests);
        dfree(srv->rows);
        srv.reset();
        serving = false;
    }

    uint64_t serve_submit(const cig_request *r) {
        if (!srv) throw CigError(CIG_ERR_STATE, "not serving");
        if (!r) throw CigError(CIG_ERR_ARG, "null request");
        ServeItem it;
        it.r = *r;
        if (r->kind == CIG_REQ_UPDATE) {
            if ((r->nd && (!r->del_u || !r->del_v)) || (r->na && (!r->add_u || !r->add_v)))
                throw CigError(CIG_ERR_ARG, "null update array");
            it.upd.resize(2 * (r->nd + r->na));
            if (r->nd) {
                std::memcpy(it.upd.data(), r->del_u, r->nd * sizeof(uint32_t));
                std::memcpy(it.upd.data() + r->nd, r->del_v, r->nd * sizeof(uint32_t));
            }
            if (r->na) {
                std::memcpy(it.upd.data() + 2 * r->nd, r->add_u, r->na * sizeof(uint32_t));
                std::memcpy(it.upd.data() + 2 * r->nd + r->na, r->add_v, r->na * sizeof(uint32_t));
            }
        } else if (r->kind == CIG_REQ_BFS || r->kind == CIG_REQ_SSSP) {
            if (r->source >= n) throw CigError(CIG_ERR_ARG, "query source out of range");
        } else {
            throw CigError(CIG_ERR_ARG, "unknown request kind");
        }
        std::unique_lock<std::mutex> lk(srv->mu);
        srv->cv_space.wait(lk, [&] { return srv->pending < srv->opt.max_pending || srv->stop; });
        if (srv->stop) throw CigError(CIG_ERR_STATE, "serving is stopping");
        it.ticket = srv->next_ticket++;
        it.t_submit = serve_ms();
        const uint64_t t = it.ticket;
        srv->open.insert(t);
        srv->queue.push_back(std::move(it));
        ++srv->pending;
        lk.unlock();
        srv->cv_work.notify_one();
        return t;
    }

    bool serve_take(uint64_t ticket, cig_result *res, bool block) {
        if (!srv) throw CigError(CIG_ERR_STATE, "not serving");
        std::unique_lock<std::mutex> lk(srv->mu);
        if (!srv->open.count(ticket)) throw CigError(CIG_ERR_ARG, "unknown ticket or result already taken");
        auto ready = [&] { return srv->results.count(ticket) != 0; };
        if (block)
            srv->cv_done.wait(lk, ready);
        else if (!ready())
            return false;
        if (res) *res = srv->results[ticket];
        srv->results.erase(ticket);
        srv->open.erase(ticket);
        return true;
    }

    void serve_publish(const ServeItem &it, const cig_result &r) {
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->results[it.ticket] = r;
            --srv->pending;
        }
        srv->cv_done.notify_all();
        srv->cv_space.notify_all();
    }

    static int32_t error_code(const std::exception &e) {
        if (const auto *c = dynamic_cast<const CigError *>(&e)) return c->code;
        return CIG_ERR_DEVICE;
    }

    // One update request: whole, or (over the admitted size) as deletion
    // chunks followed by insertion chunks, which leave the same rows and
    // values.  `after`: event of a wave the mutation must wait for.
    void serve_update(const ServeItem &it, cig_result &res, cudaEvent_t after) {
        const uint64_t nd = it.r.nd, na = it.r.na, cap = srv->chunk_cap;
        const uint32_t *d_u = it.upd.data(), *d_v = d_u + nd, *a_u = d_u + 2 * nd, *a_v = a_u + na;
        if (nd <= cap && na <= cap) {
            apply_batch_host(d_u, d_v, nd, a_u, a_v, na, nullptr, after);
        } else {
            for (uint64_t o = 0; o < nd; o += cap, after = nullptr)
                apply_batch_host(d_u + o, d_v + o, std::min(cap, nd - o), nullptr, nullptr, 0, nullptr, after);
            for (uint64_t o = 0; o < na; o += cap, after = nullptr)
                apply_batch_host(nullptr, nullptr, 0, a_u + o, a_v + o, std::min(cap, na - o), nullptr, after);
        }
        res.digest = opt.algo == CIG_PR ? 0 : digest();
    }

    void serve_loop() {
        cudaSetDevice(device);
        for (;;) {
            std::vector<ServeItem> wave;
            ServeItem upd;
            bool have_upd = false;
            {
                std::unique_lock<std::mutex> lk(srv->mu);
                srv->cv_work.wait(lk, [&] { return srv->stop || !srv->queue.empty(); });
                if (srv->queue.empty()) return;
                if (srv->queue.front().r.kind == CIG_REQ_UPDATE) {
                    upd = std::move(srv->queue.front());
                    srv->queue.pop_front();
                    have_upd = true;
                } else {
                    // Queries do not change the graph, so the wave takes every
                    // query of the front one's kind up to the next update.
                    const int32_t kind = srv->queue.front().r.kind;
                    for (auto it = srv->queue.begin(); it != srv->queue.end() && wave.size() < srv->wave_cap;) {
                        if (it->r.kind == CIG_REQ_UPDATE) break;
                        if (it->r.kind == kind) {
                            wave.push_back(std::move(*it));
                            it = srv->queue.erase(it);
                        } else {
                            ++it;
                        }
                    }
                    // The update right behind a wave starts beside it.
                    if (!srv->queue.empty() && srv->queue.front().r.kind == CIG_REQ_UPDATE) {
                        upd = std::move(srv->queue.front());
                        srv->queue.pop_front();
                        have_upd = true;
                    }
                }
            }
            if (!wave.empty()) serve_wave(wave, have_upd ? &upd : nullptr);
            else if (have_upd) {
                cig_result res{};
                res.submit_ms = upd.t_submit;
                res.start_ms = serve_ms();
                try {
                    serve_update(upd, res, nullptr);
                    res.status = CIG_OK;
                } catch (const std::exception &e) {
                    res.status = error_code(e);
                }
                res.done_ms = serve_ms();
                serve_publish(upd, res);
            }
        }
    }

    // A wave of queries of one kind (one bitmask wave), and optionally the
    // update queued right behind it: its copy and key sort overlap the wave,
    // its topology changes wait for the wave.
    void serve_wave(std::vector<ServeItem> &wave, ServeItem *upd) {
        const uint32_t k = static_cast<uint32_t>(wave.size());
        const int algo = wave[0].r.kind == CIG_REQ_BFS ? CIG_BFS : CIG_SSSP;
        std::vector<uint32_t> src(k);
        for (uint32_t j = 0; j < k; ++j) src[j] = wave[j].r.source;
        const double t_start = serve_ms();
        int32_t status = CIG_OK;
        std::vector<unsigned long long> dig(k, 0);
        bool launched = false;
        try {
            query_launch(algo, src.data(), k, k, srv->rows);
            CK(cudaMemsetAsync(srv->digests, 0, k * sizeof(unsigned long long), qstream));
            ms_row_digest<<<dim3(static_cast<unsigned>(std::min<uint64_t>(sms * 2, (n + 255) / 256)), k), 256, 0,
                            qstream>>>(srv->rows, n, srv->digests);
            ++n_launch;
            check_launch();
            CK(cudaEventRecord(q_ev[2], qstream));
            launched = true;
        } catch (const std::exception &e) {
            status = error_code(e);
        }
        cig_result ures{};
        if (upd) {
            ures.submit_ms = upd->t_submit;
            ures.start_ms = serve_ms();
            try {
                serve_update(*upd, ures, launched ? q_ev[2] : nullptr);
                ures.status = CIG_OK;
            } catch (const std::exception &e) {
                ures.status = error_code(e);
            }
        }
        if (launched) {
            try {
                query_finish(nullptr, 1, 0);
                CK(cudaMemcpy(dig.data(), srv->digests, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
                for (uint32_t j = 0; j < k; ++j)
                    if (wave[j].r.out)
                        CK(cudaMemcpy(wave[j].r.out, srv->rows + static_cast<uint64_t>(j) * n, n * sizeof(uint32_t),
                                      cudaMemcpyDeviceToHost));
            } catch (const std::exception &e) {
                status = error_code(e);
            }
        }
        const double t_done = serve_ms();
        for (uint32_t j = 0; j < k; ++j) {
            cig_result r{};
            r.status = status;
            r.wave = k;
            r.digest = dig[j];
            r.submit_ms = wave[j].t_submit;
            r.start_ms = t_start;
            r.done_ms = t_done;
            serve_publish(wave[j], r);
        }
        if (upd) {
            ures.done_ms = serve_ms();
            serve_publish(*upd, ures);
        }
    }

    // Device bytes held, by part (cig_memory_info_get), from the sizes the
    // allocations were made with.
    void memory_info(cig_memory_info *m) const {
        std::memset(m, 0, sizeof(*m));
        const uint64_t nn = n, segs = fwd.seg_total, w = (nn + 31) / 32;
        m->edge_cache = fwd.dev ? cache_slots * kSegEdges * sizeof(uint32_t) : 0;
        m->segment_table = segs * (sizeof(int32_t) + 1 + sizeof(uint32_t)) +
                           (refresh ? cache_slots * 2 * sizeof(uint32_t) + segs * sizeof(uint32_t) +
                                          (kMaxEvict + kMaxAdmit + kCtlCount) * sizeof(uint32_t)
                                    : 0);
        m->descriptors = fwd.desc ? nn * sizeof(RowDesc) + sizeof(ArenaAlloc) : 0;
        m->reverse_arena = rev.dev ? rev.seg_total * kSegEdges * sizeof(uint32_t) + nn * sizeof(RowDesc) +
                                         sizeof(ArenaAlloc)
                                   : 0;
        for (const auto &b : ixb)
            if (b.cap) m->position_index += b.cap * (sizeof(unsigned long long) + sizeof(uint2)) + w * sizeof(uint32_t);
        uint64_t vs = 0;
        if (loaded) {
            vs += 2 * (nn + 1) * sizeof(uint32_t) + nn * sizeof(uint32_t);  // q0, q1, tmp_u32
            if (inval_done) vs += (nn + 1) * sizeof(uint32_t);
            if (opt.algo == CIG_PR) {
                const uint64_t es = pr64 ? sizeof(double) : sizeof(float);
                vs += 2 * nn * es + (nn + 1) * es + 2 * nn * sizeof(uint32_t);
                if (!pr64) vs += nn * sizeof(float) + nn * sizeof(double) + 2 * w * sizeof(uint32_t) +
                                 std::max<uint32_t>(pr_hubs, 1) * sizeof(double);
            } else {
                vs += nn * sizeof(unsigned long long) + 2 * nn * sizeof(uint32_t) + (nn + 1) * sizeof(uint32_t);
            }
        }
        vs += sizeof(Status) + kSmallCount * sizeof(uint32_t) + 68 * sizeof(unsigned long long) +
              kBigRowCap * sizeof(BigRow) + sizeof(TagState);
        m->vertex_state = vs;
        // Per slot of ensure_batch: 4 update arrays (4 B), 6 key/plan arrays
        // (8 B), 12 group/match/chunk arrays (4 B), `touched` (2 x 4 B), the
        // group type (1 B), flags + positions (2 x 4 x 4 B), group ends (2 x
        // 4 B), packed whole-batch keys (2 x 4 x 8 B), addition groups (4 x 4 B),
        // warp-served addition and hub deletion groups (4 x 4 B), the reverse arena's deletion
        // scratch (6 x 4 B + 1 B).
        const uint64_t per_slot = 16 + 48 + 48 + 8 + 1 + 32 + 8 + 64 + 16 + 16 + 6 * 4 + 1;
        m->batch_buffers = bcap * per_slot + cub_bytes + cub_r_bytes + 2 * chunk_map_cap * sizeof(uint32_t) +
                           (opt.algo == CIG_PR ? 2 * bcap * sizeof(double) : 0) +
                           static_cast<uint64_t>(bsnap_cap) * 41 * sizeof(unsigned long long);
        if (qstream)
            m->query_buffers = nn * kMsWidth * sizeof(uint32_t) + 3 * nn * sizeof(unsigned long long) +
                               2 * (nn + 1) * sizeof(uint32_t) + sizeof(Status) + (8 + kMsWidth) * sizeof(uint32_t) +
                               kBigRowCap * sizeof(BigRow);
        m->total = m->edge_cache + m->segment_table + m->descriptors + m->reverse_arena + m->position_index +
                   m->vertex_state + m->batch_buffers + m->query_buffers;
        m->pinned_host = segs * kSegEdges * sizeof(uint32_t) + 4 * bcap * sizeof(uint32_t);
    }

    // Make the pinned host arena current (write back dirty cache segments).
    void flush_host() {
        if (!loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        require_alive();
        if (cache_slots) {
            launch(flush_dirty, sms * 4, 256, fwd.seg_dirty, fwd.seg_slot, fwd.dev, fwd.host_dptr, fwd.seg_total);
            check_launch();
        }
        CK(cudaStreamSynchronize(stream));
    }

    std::vector<RowDesc> host_desc() {
        if (!loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        std::vector<RowDesc> d(n);
        CK(cudaStreamSynchronize(stream));
        CK(cudaMemcpy(d.data(), fwd.desc, n * sizeof(RowDesc), cudaMemcpyDeviceToHost));
        return d;
    }
};

// ---------------------------------------------------------------- C ABI

namespace {
thread_local std::string g_create_error;
}  // namespace

// Error message of a failed call that has no handle (read by cig_last_error(NULL)).
void cig_set_unbound_error(const std::string &message) { g_create_error = message; }

namespace {

template <class F>
int guarded(cig_handle *h, F f, bool while_serving = false) {
    if (!h) return CIG_ERR_ARG;
    if (h->serving && !while_serving) {
        h->err = "the handle is serving requests (cig_serve_stop first)";
        return CIG_ERR_STATE;
    }
    try {
        CK(cudaSetDevice(h->device));
        f();
        return CIG_OK;
    } catch (const CigError &e) {
        // Serving calls may come from several threads: their errors go to
        // the calling thread's cig_last_error(NULL) text.
        (while_serving ? g_create_error : h->err) = e.what();
        if (e.code == CIG_ERR_DEVICE) h->dead = true;
        return e.code;
    } catch (const std::bad_alloc &) {
        (while_serving ? g_create_error : h->err) = "host allocation failed";
        return CIG_ERR_NOMEM;
    } catch (const std::exception &e) {
        (while_serving ? g_create_error : h->err) = e.what();
        return CIG_ERR_DEVICE;
    }
}
}  // namespace

extern "C" {

int cig_options_default(cig_options *o) {
    if (!o) return CIG_ERR_ARG;
    std::memset(o, 0, sizeof(*o));
    o->algo = CIG_SSSP;
    o->device = 0;
    o->source = 0;
    o->cache_compat = 0;
    o->cache_gib = 4.0;         // --cache default (app_skeleton.h:89)
    o->pr_epsilon = 1e-6;       // --error default (samples/hybrid_pr/hybrid_pr.cu:23)
    o->pr_max_rounds = 100;     // --pr_max_rounds default (hybrid_pr.cu:22)
    o->max_batch = 0;
    o->arena_headroom_pct = 0;
    o->flags = 0;
    o->index_budget_gib = 0.0;
    return CIG_OK;
}

int cig_create(const cig_options *o, cig_handle **out) {
    if (!out) return CIG_ERR_ARG;
    *out = nullptr;
    cig_options def;
    cig_options_default(&def);
    cig_handle *h = new (std::nothrow) cig_handle();
    if (!h) return CIG_ERR_NOMEM;
    try {
        h->create(o ? *o : def);
    } catch (const CigError &e) {
        g_create_error = e.what();
        const int code = e.code;
        h->destroy();
        delete h;
        return code;
    }
    *out = h;
    return CIG_OK;
}

int cig_destroy(cig_handle *h) {
    if (!h) return CIG_ERR_ARG;
    h->serve_stop();
    h->destroy();
    delete h;
    return CIG_OK;
}

const char *cig_last_error(const cig_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int cig_load_csr(cig_handle *h, uint32_t n, const uint64_t *xadj, const uint32_t *adj) {
    return guarded(h, [&] { h->load_csr(n, xadj, adj); });
}

int cig_load_edges(cig_handle *h, uint32_t n, const uint32_t *src, const uint32_t *dst, uint64_t m) {
    return guarded(h, [&] {
        if (m && (!src || !dst)) throw CigError(CIG_ERR_ARG, "null edge arrays");
        std::vector<uint64_t> xadj(static_cast<size_t>(n) + 1, 0);
        for (uint64_t e = 0; e < m; ++e) {
            if (src[e] >= n || dst[e] >= n) throw CigError(CIG_ERR_ARG, "edge endpoint out of range");
            ++xadj[src[e] + 1];
        }
        for (uint32_t v = 0; v < n; ++v) xadj[v + 1] += xadj[v];
        std::vector<uint64_t> cur(xadj.begin(), xadj.end() - 1);
        std::vector<uint32_t> adj(m);
        for (uint64_t e = 0; e < m; ++e) adj[cur[src[e]]++] = dst[e];  // file order within a row
        h->load_csr(n, xadj.data(), adj.data());
    });
}

int cig_init(cig_handle *h) {
    return guarded(h, [&] { h->init(); });
}

int cig_delete_phase(cig_handle *h, const uint32_t *u, const uint32_t *v, uint64_t count, cig_batch_stats *s) {
    return guarded(h, [&] { h->delete_phase_host(u, v, count, s); });
}

int cig_insert_phase(cig_handle *h, const uint32_t *u, const uint32_t *v, uint64_t count, cig_batch_stats *s) {
    return guarded(h, [&] { h->insert_phase_host(u, v, count, s); });
}

int cig_apply_batch(cig_handle *h, const uint32_t *du, const uint32_t *dv, uint64_t nd, const uint32_t *au,
                    const uint32_t *av, uint64_t na, cig_batch_stats *s) {
    return guarded(h, [&] { h->apply_batch_host(du, dv, nd, au, av, na, s); });
}

int cig_apply_batch_device(cig_handle *h, const uint32_t *du, const uint32_t *dv, uint64_t nd, const uint32_t *au,
                           const uint32_t *av, uint64_t na, cig_batch_stats *s) {
    return guarded(h, [&] { h->apply_batch_device(du, dv, nd, au, av, na, s); });
}

int cig_get_values(cig_handle *h, uint32_t *out) {
    return guarded(h, [&] {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        h->get_values(out, nullptr);
    });
}

int cig_get_parents(cig_handle *h, uint32_t *out) {
    return guarded(h, [&] {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        h->get_values(nullptr, out);
    });
}

int cig_get_pr(cig_handle *h, float *rank, float *residual) {
    return guarded(h, [&] { h->get_pr(rank, residual, nullptr, nullptr); });
}

int cig_get_pr64(cig_handle *h, double *rank, double *residual) {
    return guarded(h, [&] { h->get_pr(nullptr, nullptr, rank, residual); });
}

int cig_value_digest(cig_handle *h, uint64_t *out) {
    return guarded(h, [&] {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        *out = h->digest();
    });
}

int cig_num_edges(cig_handle *h, uint64_t *m) {
    return guarded(h, [&] {
        if (!m) throw CigError(CIG_ERR_ARG, "null output");
        const auto d = h->host_desc();
        uint64_t s = 0;
        for (const auto &r : d) s += rd_live(r);
        *m = s;
    });
}

int cig_get_degrees(cig_handle *h, uint32_t *deg) {
    return guarded(h, [&] {
        if (!deg) throw CigError(CIG_ERR_ARG, "null output");
        const auto d = h->host_desc();
        for (uint32_t v = 0; v < h->n; ++v) deg[v] = rd_live(d[v]);
    });
}

// Copy the live entries of a row (tombstones dropped, order kept).
static uint32_t copy_live(const uint32_t *row, uint32_t len, uint32_t *out, uint32_t capacity) {
    uint32_t w = 0;
    for (uint32_t k = 0; k < len; ++k) {
        if (row[k] == kTomb) continue;
        if (out && w < capacity) out[w] = row[k];
        ++w;
    }
    return w;
}

int cig_get_row(cig_handle *h, uint32_t v, uint32_t *out, uint32_t capacity, uint32_t *degree) {
    return guarded(h, [&] {
        if (!h->loaded) throw CigError(CIG_ERR_ARG, "load a graph first");
        if (v >= h->n) throw CigError(CIG_ERR_ARG, "vertex out of range");
        RowDesc d;
        h->flush_host();
        CK(cudaMemcpy(&d, h->fwd.desc + v, sizeof(d), cudaMemcpyDeviceToHost));
        if (degree) *degree = rd_live(d);
        if (out) copy_live(h->fwd.host + d.off, d.len, out, capacity);
    });
}

int cig_export_csr(cig_handle *h, uint64_t *xadj, uint32_t *adj) {
    return guarded(h, [&] {
        if (!xadj) throw CigError(CIG_ERR_ARG, "null output");
        const auto d = h->host_desc();
        xadj[0] = 0;
        for (uint32_t v = 0; v < h->n; ++v) xadj[v + 1] = xadj[v] + rd_live(d[v]);
        if (!adj) return;
        h->flush_host();
        const uint32_t *arena = h->fwd.host;
        parallel_for(h->n, [&](uint64_t b, uint64_t e) {
            for (uint64_t v = b; v < e; ++v)
                if (d[v].len) copy_live(arena + d[v].off, d[v].len, adj + xadj[v], rd_live(d[v]));
        });
    });
}

int cig_graph_info_get(cig_handle *h, cig_graph_info *info) {
    return guarded(h, [&] {
        if (!info) throw CigError(CIG_ERR_ARG, "null output");
        std::memset(info, 0, sizeof(*info));
        info->n = h->n;
        if (!h->loaded) return;
        const auto d = h->host_desc();
        uint64_t m = 0;
        for (const auto &r : d) m += rd_live(r);
        info->m = m;
        ArenaAlloc al;
        CK(cudaMemcpy(&al, h->fwd.alloc, sizeof(al), cudaMemcpyDeviceToHost));
        info->arena_capacity_edges = h->fwd.seg_total * kSegEdges;
        info->arena_used_edges = std::min<uint64_t>(al.seg_bump, h->fwd.seg_total) * kSegEdges;
        info->segment_edges = kSegEdges;
        info->segments_total = h->fwd.seg_total;
        {
            std::vector<int32_t> slot(h->fwd.seg_total);
            CK(cudaMemcpy(slot.data(), h->fwd.seg_slot, slot.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
            const uint64_t used = std::min<uint64_t>(al.seg_bump, h->fwd.seg_total);
            uint64_t r = 0;
            for (uint64_t s = 0; s < used; ++s) r += slot[s] >= 0;
            info->segments_resident = r;
        }
        info->cache_capacity_segments = h->cache_slots;
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        info->device_bytes = total_b - free_b;
        info->pinned_bytes = h->fwd.seg_total * kSegEdges * sizeof(uint32_t);
    });
}

int cig_memory_info_get(cig_handle *h, cig_memory_info *out) {
    return guarded(h, [&] {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        h->memory_info(out);
    });
}

int cig_profile_enable(cig_handle *h, int enable) {
    return guarded(h, [&] {
        CK(cudaStreamSynchronize(h->stream));
        h->prof_pending.clear();
        h->ev_used = 0;
        std::memset(h->prof, 0, sizeof(h->prof));
        h->prof_on = enable != 0;
    });
}

int cig_profile_read(cig_handle *h, cig_stage_profile *out, uint32_t count) {
    return guarded(h, [&] {
        if (!out) throw CigError(CIG_ERR_ARG, "null output");
        std::memcpy(out, h->prof, std::min<uint32_t>(count, CIG_STAGE_COUNT) * sizeof(cig_stage_profile));
    });
}

int cig_autotune(cig_handle *h, cig_tune_result *res) {
    return guarded(h, [&] { h->autotune(res); });
}

int cig_serve_start(cig_handle *h, const cig_serve_options *o) {
    return guarded(h, [&] { h->serve_start(o); });
}

int cig_serve_submit(cig_handle *h, const cig_request *r, uint64_t *ticket) {
    return guarded(
        h, [&] {
            if (!ticket) throw CigError(CIG_ERR_ARG, "null ticket");
            *ticket = h->serve_submit(r);
        },
        true);
}

int cig_serve_wait(cig_handle *h, uint64_t ticket, cig_result *res) {
    return guarded(h, [&] { h->serve_take(ticket, res, true); }, true);
}

int cig_serve_poll(cig_handle *h, uint64_t ticket, cig_result *res, int *done) {
    return guarded(
        h, [&] {
            if (!done) throw CigError(CIG_ERR_ARG, "null done flag");
            *done = h->serve_take(ticket, res, false) ? 1 : 0;
        },
        true);
}

int cig_serve_stop(cig_handle *h) {
    return guarded(h, [&] { h->serve_stop(); }, true);
}

int cig_apply_batches_device(cig_handle *h, const cig_update_batch *batches, uint32_t count, cig_batch_stats *stats,
                             uint64_t *digests) {
    return guarded(h, [&] { h->apply_batches_device(batches, count, stats, digests); });
}

int cig_query_bfs_multi(cig_handle *h, const uint32_t *sources, uint32_t k, uint32_t *out_depth) {
    return guarded(h, [&] { h->query_multi_host(CIG_BFS, sources, k, out_depth); });
}

int cig_query_sssp_multi(cig_handle *h, const uint32_t *sources, uint32_t k, uint32_t *out_dist) {
    return guarded(h, [&] { h->query_multi_host(CIG_SSSP, sources, k, out_dist); });
}

int cig_query_multi_device(cig_handle *h, int algo, const uint32_t *sources, uint32_t k, uint32_t width,
                           uint32_t *out_device, cig_query_stats *stats) {
    return guarded(h, [&] { h->query_multi(algo, sources, k, width, out_device, stats); });
}

const char *cig_version(void) { return kVersion; }

int cig_build_info(int *binary_version, int *bounds_checked) {
    if (bounds_checked) {
#ifdef CIG_BOUNDS_CHECK
        *bounds_checked = 1;
#else
        *bounds_checked = 0;
#endif
    }
    if (!binary_version) return CIG_OK;
    cudaFuncAttributes a{};
    const cudaError_t e = cudaFuncGetAttributes(&a, reinterpret_cast<const void *>(value_digest));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cig_set_unbound_error(std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e));
        return CIG_ERR_DEVICE;
    }
    *binary_version = a.binaryVersion;
    return CIG_OK;
}

}  // extern "C"
