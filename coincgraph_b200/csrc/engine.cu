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
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/cig.h"
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
struct Layout {
    std::vector<RowDesc> desc;
    unsigned long long cur_next[kNumClasses] = {};
    unsigned long long cur_end[kNumClasses] = {};
    uint64_t used_segs = 0;
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
    kSmallCount = 20
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
    AdjView view() const { return AdjView{desc, dev, host_dptr, seg_slot, seg_dirty}; }
};

// Write-back of the edge cache: copy every dirty resident segment to its
// pinned host copy (one block per segment, 16-byte stores) and clear the flag.
__global__ void flush_dirty(uint8_t *dirty, const int32_t *seg_slot, const uint32_t *cache, uint32_t *host,
                            uint64_t nsegs) {
    for (uint64_t s = blockIdx.x; s < nsegs; s += gridDim.x) {
        if (!dirty[s]) continue;
        const int32_t slot = seg_slot[s];
        if (slot >= 0) {
            const uint4 *src = reinterpret_cast<const uint4 *>(cache + (static_cast<uint64_t>(slot) << kSegShift));
            uint4 *dst = reinterpret_cast<uint4 *>(host + (s << kSegShift));
            for (uint32_t i = threadIdx.x; i < kSegEdges / 4; i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) dirty[s] = 0;
        __syncthreads();
    }
}

const char *kVersion = "cig 0.1.0 (sm_100a)";

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

    unsigned long long *state = nullptr;
    uint32_t *qstamp = nullptr, *aff_stamp = nullptr, *q0 = nullptr, *q1 = nullptr, *list = nullptr;
    uint32_t *small = nullptr;
    unsigned long long *small64 = nullptr;
    TagState *tags = nullptr;
    Status *status = nullptr;
    Status *h_status = nullptr;
    uint32_t epoch = 0;

    void *pr_rank = nullptr, *pr_res = nullptr, *pr_contrib = nullptr, *pr_amend = nullptr;
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
    // flat deletion: per-group chunk counts, their inclusive prefix sum, the
    // groups left to the ordered kernels, first match per key
    uint32_t *chunks = nullptr, *chunk_end = nullptr, *ordered = nullptr, *firstpos = nullptr;
    // group building: head flags, their exclusive scan, group ends per direction
    uint32_t *gflags = nullptr, *gpos = nullptr, *gendf = nullptr, *gendr = nullptr;
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
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }
    int prof_begin(int stage) {
        if (!prof_on) return -1;
        cudaEvent_t a = take_event();
        CK(cudaEventRecord(a, stream));
        prof_pending.push_back({stage, a, nullptr});
        return static_cast<int>(prof_pending.size()) - 1;
    }
    void prof_end(int idx) {
        if (idx < 0) return;
        cudaEvent_t b = take_event();
        CK(cudaEventRecord(b, stream));
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
        return BigList{big_rows, small + kBigRows, kBigRowCap};
    }

    template <class K>
    int coop_blocks(K kernel, int tpb) const {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, tpb, 0));
        int want = 4;
        if (const char *e = std::getenv("CIG_COOP_BLOCKS_PER_SM")) want = std::max(1, std::atoi(e));
        per_sm = std::min(per_sm, want);
        if (per_sm < 1) throw CigError(CIG_ERR_DEVICE, "cooperative kernel does not fit on an SM");
        return per_sm * sms;
    }

    uint64_t n_launch = 0;  // kernels this engine launched (CUB sort kernels not included)

    template <class... P>
    void launch(void (*kernel)(P...), int grid, int block, typename Identity<P>::type... args) {
        kernel<<<grid, block, 0, stream>>>(args...);
        ++n_launch;
    }

    // Arguments are converted to the kernel's exact parameter types, as the
    // void* argument array of a cooperative launch requires.
    template <class... P>
    void launch_coop(void (*kernel)(P...), int tpb, typename Identity<P>::type... args) {
        void *argv[] = {static_cast<void *>(&args)...};
        const int blocks = coop_blocks(kernel, tpb);
        CK(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kernel), dim3(blocks), dim3(tpb), argv, 0,
                                       stream));
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

    uint64_t launch_mark = 0;

    void reset_counters() {
        CK(cudaMemsetAsync(status->counters, 0, sizeof(status->counters), stream));
        launch_mark = n_launch;
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
            throw CigError(code, "device reported: " + what + "info=" + std::to_string(h_status->err_info));
        }
    }

    template <class F>
    void dispatch(F f) {
        switch (opt.algo) {
        case CIG_BFS: f(std::integral_constant<int, kBfs>{}); break;
        case CIG_SSSP: f(std::integral_constant<int, kSssp>{}); break;
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
        for (auto &e : ev) CK(cudaEventCreate(&e));
        dmalloc(status, 1);
        CK(cudaMemset(status, 0, sizeof(Status)));
        CK(cudaHostAlloc(reinterpret_cast<void **>(&h_status), sizeof(Status), cudaHostAllocDefault));
        dmalloc(small, kSmallCount);
        CK(cudaMemset(small, 0, kSmallCount * sizeof(uint32_t)));
        dmalloc(small64, 4);
        dmalloc(big_rows, kBigRowCap);
        dmalloc(tags, 1);
        CK(cudaMemset(tags, 0, sizeof(TagState)));
        pr64 = (opt.flags & CIG_FLAG_PR_FP64) != 0;
    }

    void destroy() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
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
        dfree(state);
        dfree(qstamp);
        dfree(aff_stamp);
        dfree(q0);
        dfree(q1);
        dfree(list);
        dfree(small);
        dfree(small64);
        dfree(big_rows);
        dfree(tags);
        dfree(status);
        if (h_status) cudaFreeHost(h_status);
        dfree(pr_rank);
        dfree(pr_res);
        dfree(pr_contrib);
        dfree(pr_amend);
        dfree(pr_comp);
        dfree(pr_queued);
        free_batch();
        dfree(tmp_u32);
        free_queries();
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
        dfree(pf);
        dfree(prr);
        dfree(touched);
        dfree(compact);
        dfree(chunks);
        dfree(chunk_end);
        dfree(ordered);
        dfree(firstpos);
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
        dmalloc(firstpos, cap);
        dmalloc(gflags, cap);
        dmalloc(gpos, cap);
        dmalloc(gendf, cap);
        dmalloc(gendr, cap);
        if (opt.algo == CIG_PR) {
            dfree(pr_amend);
            CK(cudaMalloc(&pr_amend, 2 * cap * (pr64 ? sizeof(double) : sizeof(float))));
        }
        cub::DoubleBuffer<unsigned long long> db(kf, t1);
        size_t bytes = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, static_cast<int>(cap), 0, 64, stream));
        size_t scan_bytes = 0;
        CK(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, chunks, chunk_end, static_cast<int>(cap), stream));
        bytes = std::max(bytes, scan_bytes);
        CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, gflags, gpos, static_cast<int>(cap), stream));
        bytes = std::max(bytes, scan_bytes);
        cub_bytes = bytes;
        CK(cudaMalloc(&cub, std::max<size_t>(bytes, 16)));
        CK(cudaHostAlloc(reinterpret_cast<void **>(&stage), 4 * cap * sizeof(uint32_t), cudaHostAllocDefault));
        bcap = cap;
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
        CK(cudaSetDevice(device));

        // Forward arena in pinned mapped host memory.
        Layout L = plan_layout(n, deg.data());
        const double pct = opt.arena_headroom_pct ? opt.arena_headroom_pct : 12.5;
        const uint64_t head = std::max<uint64_t>(static_cast<uint64_t>(L.used_segs * pct / 100.0) + 1,
                                                 (1ull << 20) >> kSegShift);
        fwd.seg_used = L.used_segs;
        fwd.seg_total = L.used_segs + head;
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

        // HBM edge cache: whole segments, initially the first ones in arena order
        // (largest row classes first).
        uint64_t budget_slots;
        if (opt.cache_compat) {
            const long long c = static_cast<long long>(opt.cache_gib);
            static const uint64_t table[] = {0ull, 268435455ull, 536870921ull, 805306365ull, 1073741824ull};
            budget_slots = (c >= 0 && c <= 4) ? table[c] : 1073741824ull;
        } else {
            budget_slots = opt.cache_gib > 0 ? static_cast<uint64_t>(opt.cache_gib * 1073741824.0 / 4.0) : 0;
        }
        // Slots left over after the used segments go to the headroom segments
        // that the block allocator hands out later, so relocated rows land in
        // HBM while the budget lasts.
        cache_slots = std::min<uint64_t>(budget_slots >> kSegShift, fwd.seg_total);
        resident = cache_slots;
        if (cache_slots) {
            dmalloc(fwd.dev, cache_slots * kSegEdges);
            const uint64_t filled = std::min<uint64_t>(cache_slots, fwd.seg_used);
            if (filled)
                CK(cudaMemcpy(fwd.dev, fwd.host, filled * kSegEdges * sizeof(uint32_t), cudaMemcpyHostToDevice));
        }
        {
            std::vector<int32_t> slot(fwd.seg_total, -1);
            for (uint64_t s = 0; s < resident; ++s) slot[s] = static_cast<int32_t>(s);
            dmalloc(fwd.seg_slot, fwd.seg_total);
            CK(cudaMemcpy(fwd.seg_slot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
            dmalloc(fwd.seg_dirty, fwd.seg_total);
            CK(cudaMemset(fwd.seg_dirty, 0, fwd.seg_total));
        }
        dmalloc(seg_hot, fwd.seg_total);
        CK(cudaMemset(seg_hot, 0, fwd.seg_total * sizeof(uint32_t)));

        // Reverse arena (device only) for deletion repair.
        if (opt.algo != CIG_PR) build_reverse(xadj, adj, m);

        // Vertex state.
        dmalloc(q0, n + 1);
        dmalloc(q1, n + 1);
        dmalloc(tmp_u32, n);
        if (opt.algo == CIG_PR) {
            const size_t es = pr64 ? sizeof(double) : sizeof(float);
            CK(cudaMalloc(&pr_rank, n * es));
            CK(cudaMalloc(&pr_res, n * es));
            CK(cudaMalloc(&pr_contrib, (n + 1) * es));
            if (!pr64) dmalloc(pr_comp, n);
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
            dispatch([&](auto tag) {
                constexpr int A = decltype(tag)::value;
                launch(init_state<A>, persistent_grid(), 256, state, n, source);
                CK(cudaMemsetAsync(small + kFr, 0, 3 * sizeof(uint32_t), stream));
                if (A == kCc)
                    launch(enqueue_all_nonempty, persistent_grid(), 256, fwd.desc, n, frontier(), status);
                else
                    launch(set_single, 1, 1, q0, small + kFr, source);
                check_launch();
                run_push<A>();
            });
        }
        finish();
        initialized = true;
    }

    template <int A>
    void run_push() {
        const int p = prof_begin(CIG_STAGE_PUSH);
        launch_coop(push_closure<A>, kTpb, fwd.view(), state, qstamp, tags, frontier(), big_list(), n + 2, seg_hot,
                    status);
        prof_end(p);
    }

    // ------------------------------------------------------------ PR
    template <class T>
    PrArrays<T> pr_arrays() {
        return PrArrays<T>{static_cast<T *>(pr_rank), static_cast<T *>(pr_res), pr_comp, pr_queued, q0, q1,
                           small + kFr, static_cast<T *>(pr_contrib), small + kFinalRound, n + 1};
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
        launch(pr_residual_l1<T>, persistent_grid(), 256, static_cast<const T *>(pr_res), n,
                                                                  reinterpret_cast<double *>(small64));
        check_launch();
    }

    template <class T>
    void pr_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                  const uint32_t *d_av, uint64_t na) {
        auto a = pr_arrays<T>();
        const T eps = static_cast<T>(opt.pr_epsilon);
        ++epoch;
        CK(cudaMemsetAsync(small + kTouched, 0, sizeof(uint32_t), stream));
        if (nd + na)
            launch(collect_touched, grid_for(nd + na), 256, d_du, static_cast<uint32_t>(nd), d_au,
                                                                  static_cast<uint32_t>(na), n, aff_stamp, epoch,
                                                                  touched, small + kTouched,
                                                                  static_cast<uint32_t>(2 * bcap), status);
        T *amend = static_cast<T *>(pr_amend);
        // r' = r + alpha (P_new^T - P_old^T) x over the touched sources.
        int p = prof_begin(CIG_STAGE_PR);
        launch(pr_amend_contrib<T>, persistent_grid(), 256, fwd.desc, a, touched, small + kTouched, T(-1),
                                                                   amend);
        launch(pr_amend_scatter<T>, persistent_grid(), kTpbPr, fwd.view(), a, touched, small + kTouched,
                                                                      amend, eps, status);
        prof_end(p);
        check_launch();
        mutate_forward_delete(d_du, d_dv, nd, true);
        mutate_forward_add(d_au, d_av, na, true);
        p = prof_begin(CIG_STAGE_PR);
        launch(pr_amend_contrib<T>, persistent_grid(), 256, fwd.desc, a, touched, small + kTouched, T(1),
                                                                   amend);
        launch(pr_amend_scatter<T>, persistent_grid(), kTpbPr, fwd.view(), a, touched, small + kTouched,
                                                                      amend, eps, status);
        prof_end(p);
        check_launch();
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

    void mutate_delete_arena(DevArena &A, const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, bool forward,
                             bool with_stats) {
        if (nd == 0) return;
        const uint32_t m = static_cast<uint32_t>(nd);
        unsigned long long *keys = forward ? kf : kr;
        unsigned long long *tmp = forward ? t1 : t2;
        uint32_t *groups = forward ? gf : gr;
        uint32_t *matched = forward ? mf : mr;
        uint32_t *big = forward ? bigf : bigr;
        uint32_t *gcount = small + (forward ? kGcF : kGcR);
        uint32_t *bcount = small + (forward ? kBigF : kBigR);
        int p = prof_begin(CIG_STAGE_GROUP);
        // make_keys_del fills both kf and kr; only build them once per phase.
        if (forward || opt.algo == CIG_PR) {
            launch(make_keys_del, grid_for(nd), 256, d_du, d_dv, m, n, kf, kr, status);
            check_launch();
        }
        unsigned long long *sorted = sort_keys(keys, tmp, nd);
        CK(cudaMemsetAsync(bcount, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(matched, 0, nd * sizeof(uint32_t), stream));
        const Groups grp = build_groups(sorted, nd, groups, forward ? gendf : gendr, gcount);
        prof_end(p);
        p = prof_begin(forward ? CIG_STAGE_MUTATE : CIG_STAGE_MUTATE_REV);
        unsigned long long *stats = with_stats ? status->counters : nullptr;
        uint32_t *ccount = small + kCompactCount;
        uint32_t *ocount = small + kOrderedCount;
        CK(cudaMemsetAsync(ccount, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(ocount, 0, sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(chunks, 0, nd * sizeof(uint32_t), stream));
        CK(cudaMemsetAsync(firstpos, 0xFF, nd * sizeof(uint32_t), stream));
        // Flat path: rows whose deletion requests are all distinct.
        launch(del_classify, persistent_grid(), 256, A.desc, sorted, grp, chunks, ordered, ocount);
        {
            size_t bytes = cub_bytes;
            CK(cub::DeviceScan::InclusiveSum(cub, bytes, chunks, chunk_end, static_cast<int>(nd), stream));
        }
        launch(del_scan, persistent_grid(), kMutWarps * 32, A.view(), A.desc, sorted, grp, chunk_end, m, firstpos);
        launch(del_apply, grid_for(nd), 256, A.view(), A.desc, sorted, m, firstpos, stats);
        launch(del_finish, persistent_grid(), 256, A.desc, sorted, grp, chunks, firstpos, compact, ccount, stats);
        // Ordered path: rows with repeated requests for a destination.
        launch(mutate_delete, persistent_grid(), kMutWarps * 32, A.view(), A.desc, sorted, grp, ordered, ocount,
               matched, big, bcount, compact, ccount, stats, status);
        launch(mutate_delete_big, sms * 4, kTpbMut, A.view(), A.desc, sorted, grp, big, bcount, matched, compact,
               ccount, stats, status);
        launch(compact_rows, sms * 4, kTpbMut, A.view(), A.desc, compact, ccount);
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
        if (forward || opt.algo == CIG_PR) {
            launch(make_keys_add, grid_for(na), 256, d_au, d_av, m, n, kf, kr, status);
            check_launch();
        }
        unsigned long long *sorted = sort_keys(keys, tmp, na);
        CK(cudaMemsetAsync(bcount, 0, sizeof(uint32_t), stream));
        const Groups grp = build_groups(sorted, na, groups, forward ? gendf : gendr, gcount);
        prof_end(p);
        p = prof_begin(forward ? CIG_STAGE_ADD : CIG_STAGE_ADD_REV);
        launch(plan_add, persistent_grid(), 256, A.desc, sorted, grp, plan, A.alloc);
        launch(alloc_classes, 1, 64, A.alloc, status);
        unsigned long long *stats = with_stats ? status->counters : nullptr;
        const uint32_t *vals = forward ? d_av : d_au;
        launch(mutate_add, persistent_grid(), 256, A.view(), A.desc, sorted, grp, plan, A.alloc, vals, big, bcount,
               stats, status);
        launch(mutate_add_big, sms * 2, kTpbMut, A.view(), A.desc, sorted, grp, plan, A.alloc, vals, big, bcount,
               stats, status);
        prof_end(p);
        check_launch();
    }

    // ------------------------------------------------------------ batches
    template <int A>
    void delete_phase_dev(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd) {
        ++epoch;
        CK(cudaMemsetAsync(small + kFr, 0, 6 * sizeof(uint32_t), stream));  // frontier + affected counters
        int p = prof_begin(CIG_STAGE_SEED);
        if (nd)
            launch(seed_deletions<A>, grid_for(nd), 256, d_du, d_dv, static_cast<uint32_t>(nd), n, state,
                                                                aff_stamp, epoch, list, small + kAff, n + 1, status);
        prof_end(p);
        check_launch();
        mutate_delete_arena(fwd, d_du, d_dv, nd, true, true);
        mutate_delete_arena(rev, d_du, d_dv, nd, false, false);
        p = prof_begin(CIG_STAGE_INVAL);
        launch_coop(inval_closure<A>, kTpb, fwd.view(), state, aff_stamp, epoch, list, small + kAff, n + 1,
                    big_list(), n + 2, small + kAffTotal, status);
        prof_end(p);
        p = prof_begin(CIG_STAGE_PULL);
        launch(reset_affected<A>, persistent_grid(), 256, list, small + kAffTotal, state);
        const BigList pull_big = big_list();
        launch(pull_repair<A>, persistent_grid(), kTpb, rev.view(), state, aff_stamp, epoch, list,
                                                               small + kAffTotal, pull_big, status);
        launch(pull_deferred<A>, persistent_grid(), kTpb, rev.view(), state, aff_stamp, epoch, pull_big, status);
        launch(enqueue_affected<A>, persistent_grid(), 256, list, small + kAffTotal, state, frontier(), status);
        prof_end(p);
        check_launch();
        run_push<A>();
    }

    template <int A>
    void insert_phase_dev(const uint32_t *d_au, const uint32_t *d_av, uint64_t na) {
        CK(cudaMemsetAsync(small + kFr, 0, 3 * sizeof(uint32_t), stream));
        mutate_add_arena(fwd, d_au, d_av, na, true, true);
        mutate_add_arena(rev, d_au, d_av, na, false, false);
        int p = prof_begin(CIG_STAGE_SEED);
        if (na)
            launch(seed_insertions<A>, grid_for(na), 256, d_au, d_av, static_cast<uint32_t>(na), n, state,
                                                                 qstamp, tags, frontier(), status);
        prof_end(p);
        check_launch();
        run_push<A>();
    }

    // Copy host update arrays into the device batch buffers (pinned staging).
    void stage_pairs(const uint32_t *hu, const uint32_t *hv, uint64_t count, uint32_t *du_, uint32_t *dv_,
                     uint32_t *stage_base) {
        if (!count) return;
        if (!hu || !hv) throw CigError(CIG_ERR_ARG, "null update array");
        std::memcpy(stage_base, hu, count * sizeof(uint32_t));
        std::memcpy(stage_base + bcap, hv, count * sizeof(uint32_t));
        CK(cudaMemcpyAsync(du_, stage_base, count * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(dv_, stage_base + bcap, count * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    }

    void require_ready() {
        require_alive();
        if (!initialized) throw CigError(CIG_ERR_ARG, "call cig_init first");
    }

    void delete_phase_host(const uint32_t *hu, const uint32_t *hv, uint64_t nd, cig_batch_stats *s) {
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank applies whole batches (cig_apply_batch)");
        ensure_batch(nd);
        reset_counters();
        CK(cudaEventRecord(ev[0], stream));
        stage_pairs(hu, hv, nd, du, dv, stage);
        dispatch([&](auto tag) { delete_phase_dev<decltype(tag)::value>(du, dv, nd); });
        CK(cudaEventRecord(ev[1], stream));
        finish();
        fill_stats(s, nd, 0, true, false);
    }

    void insert_phase_host(const uint32_t *hu, const uint32_t *hv, uint64_t na, cig_batch_stats *s) {
        require_ready();
        if (opt.algo == CIG_PR) throw CigError(CIG_ERR_ARG, "PageRank applies whole batches (cig_apply_batch)");
        ensure_batch(na);
        reset_counters();
        CK(cudaEventRecord(ev[1], stream));
        stage_pairs(hu, hv, na, au, av, stage + 2 * bcap);
        dispatch([&](auto tag) { insert_phase_dev<decltype(tag)::value>(au, av, na); });
        CK(cudaEventRecord(ev[2], stream));
        CK(cudaEventRecord(ev[3], stream));
        finish();
        fill_stats(s, 0, na, false, true);
    }

    void apply_batch(const uint32_t *d_du, const uint32_t *d_dv, uint64_t nd, const uint32_t *d_au,
                     const uint32_t *d_av, uint64_t na, cig_batch_stats *s) {
        if (opt.algo == CIG_PR) {
            if (pr64)
                pr_batch<double>(d_du, d_dv, nd, d_au, d_av, na);
            else
                pr_batch<float>(d_du, d_dv, nd, d_au, d_av, na);
            CK(cudaEventRecord(ev[1], stream));
            CK(cudaEventRecord(ev[2], stream));
        } else {
            dispatch([&](auto tag) {
                constexpr int A = decltype(tag)::value;
                delete_phase_dev<A>(d_du, d_dv, nd);
                CK(cudaEventRecord(ev[1], stream));
                insert_phase_dev<A>(d_au, d_av, na);
                CK(cudaEventRecord(ev[2], stream));
            });
        }
        CK(cudaEventRecord(ev[3], stream));
        finish();
        fill_stats(s, nd, na, true, true);
    }

    void apply_batch_host(const uint32_t *hdu, const uint32_t *hdv, uint64_t nd, const uint32_t *hau,
                          const uint32_t *hav, uint64_t na, cig_batch_stats *s) {
        require_ready();
        ensure_batch(std::max(nd, na));
        reset_counters();
        CK(cudaEventRecord(ev[0], stream));
        stage_pairs(hdu, hdv, nd, du, dv, stage);
        stage_pairs(hau, hav, na, au, av, stage + 2 * bcap);
        apply_batch(du, dv, nd, au, av, na, s);
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

    void fill_stats(cig_batch_stats *s, uint64_t nd, uint64_t na, bool del, bool ins) {
        const unsigned long long *c = h_status->counters;
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
        s->kernel_launches = n_launch - launch_mark;
        float ms = 0;
        if (del) {
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            s->ms_delete = ms;
        }
        if (ins) {
            cudaEventElapsedTime(&ms, ev[1], ev[2]);
            s->ms_insert = ms;
            cudaEventElapsedTime(&ms, ev[2], ev[3]);
            s->ms_cache = ms;
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
                                                              out_parents ? tmp_u32 : nullptr);
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
        launch(value_digest, persistent_grid(), 256, state, n, small64 + 1);
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
        const uint64_t launches0 = n_launch;
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
            const BigList bl{ms_big, ms_small + 3, kBigRowCap};
            ms_seed<<<1, kMsWidth, 0, qstream>>>(ms_src, kw, ms_dist, width, algo == CIG_BFS ? ms_visit : nullptr,
                                                 fr, qstatus);
            ++n_launch;
            if (algo == CIG_BFS)
                launch_coop_on(qstream, ms_closure<kBfs>, kTpbMs, fwd.view(), ms_dist, width, ms_visit, fr, bl, n + 2,
                               qstatus);
            else
                launch_coop_on(qstream, ms_closure<kSssp>, kTpbMs, fwd.view(), ms_dist, width,
                               static_cast<unsigned long long *>(nullptr), fr, bl, n + 2, qstatus);
            ms_transpose<<<(n + kMsTile - 1) / kMsTile, 256, 0, qstream>>>(ms_dist, n, width, kw,
                                                                         out + static_cast<uint64_t>(j0) * n);
            ++n_launch;
            check_launch();
        }
        CK(cudaEventRecord(q_ev[2], qstream));
        CK(cudaStreamSynchronize(qstream));
        CK(cudaMemcpy(h_qstatus, qstatus, sizeof(Status), cudaMemcpyDeviceToHost));
        if (h_qstatus->err) {
            std::string what;
            if (h_qstatus->err & kErrRounds) what += "round bound exceeded; ";
            if (h_qstatus->err & kErrBarrier) what += "grid barrier wait limit exceeded; ";
            if (h_qstatus->err & kErrQueue) what += "work queue overflow; ";
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
            qs->kernel_launches = n_launch - launches0;
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
int guarded(cig_handle *h, F f) {
    if (!h) return CIG_ERR_ARG;
    try {
        CK(cudaSetDevice(h->device));
        f();
        return CIG_OK;
    } catch (const CigError &e) {
        h->err = e.what();
        if (e.code == CIG_ERR_DEVICE) h->dead = true;
        return e.code;
    } catch (const std::bad_alloc &) {
        h->err = "host allocation failed";
        return CIG_ERR_NOMEM;
    } catch (const std::exception &e) {
        h->err = e.what();
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
        info->segments_resident = std::min<uint64_t>(h->resident, std::min<uint64_t>(al.seg_bump, h->fwd.seg_total));
        info->cache_capacity_segments = h->cache_slots;
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        info->device_bytes = total_b - free_b;
        info->pinned_bytes = h->fwd.seg_total * kSegEdges * sizeof(uint32_t);
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

}  // extern "C"
