// mutate.cuh - GPU batch maintenance of an adjacency arena.
//
// Semantics follow the reference's source-local chunk store exactly
// (include/groute/graphs/source_local_chunk_store.h:219-391, 670-848) so that
// rows stay identical, element for element:
//   deletion phase: for every source, a destination requested k times loses
//     its first min(k, present) occurrences; survivors keep their order
//     (BuildDeletionPlan / ShouldDelete / CompactSourceInPlace);
//   addition phase: destinations are appended in input order; a row that
//     outgrows its power-of-two block moves to a larger block
//     (RewriteSourceToNewBlock).
// The batch is grouped by source with a device radix sort of 64-bit keys
// (source << 32 | destination) for deletions and (source << 32 | input index)
// for additions; the latter keeps input order inside a source, as the
// reference's stable radix sort does (effective_update_batch.h:48-73).
//
// Design differences from the reference (same rows):
//   - a deleted entry is overwritten with a tombstone instead of shifting
//     the rest of the row; the scan of a row stops once every requested
//     deletion of that row has been found, so a batch reads about half of
//     each touched row and writes one word per deletion;
//   - a row is compacted (tombstones dropped, order kept) when it relocates
//     or when tombstones reach a quarter of its length;
//   - grouping, matching, allocation and appends all run on the GPU.
#pragma once

#include <cub/block/block_radix_sort.cuh>
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "posindex.cuh"

namespace cig {

constexpr uint32_t kKeyShift = 32;
constexpr unsigned long long kKeyNone = ~0ull;
constexpr uint32_t kWarpRowMax = 4096;  // larger rows use the block path
constexpr int kMutWarps = 8;            // warps per block of the warp-path kernels
constexpr int kTpbMut = 256;            // threads per block of the block-path kernels

__device__ __forceinline__ uint32_t key_src(unsigned long long k) { return static_cast<uint32_t>(k >> kKeyShift); }
__device__ __forceinline__ uint32_t key_low(unsigned long long k) { return static_cast<uint32_t>(k); }

// Device-side block allocator: per class a partially used segment
// [cur_next, cur_end) and a global bump pointer over whole segments.
// Blocks left by relocation are not reused.
struct ArenaAlloc {
    unsigned long long seg_bump;
    unsigned long long seg_total;
    unsigned long long cur_next[kNumClasses];
    unsigned long long cur_end[kNumClasses];
    unsigned long long base_cur[kNumClasses];
    unsigned long long base_new[kNumClasses];
    uint32_t demand[kNumClasses];
    uint32_t avail[kNumClasses];
};

__device__ __forceinline__ uint32_t class_for(uint32_t deg) {
    if (deg <= (1u << kMinClass)) return kMinClass;
    return 32u - __clz(deg - 1u);
}

__device__ __forceinline__ unsigned long long alloc_offset(const ArenaAlloc *al, uint32_t cls, uint32_t rank) {
    if (cls <= kSegShift && rank < al->avail[cls])
        return al->base_cur[cls] + (static_cast<unsigned long long>(rank) << cls);
    const uint32_t r = cls <= kSegShift ? rank - al->avail[cls] : rank;
    return al->base_new[cls] + (static_cast<unsigned long long>(r) << cls);
}

// Keys for the deletion phase.  Invalid records (id out of range) sort last;
// they remove nothing and are reported as missing deletes.
__global__ void make_keys_del(const uint32_t *du, const uint32_t *dv, uint32_t nd, uint32_t n,
                              unsigned long long *kf, unsigned long long *kr, Status *) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t u = du[i], v = dv[i];
    if (u < n && v < n) {
        kf[i] = (static_cast<unsigned long long>(u) << kKeyShift) | v;
        kr[i] = (static_cast<unsigned long long>(v) << kKeyShift) | u;
    } else {
        kf[i] = kKeyNone;
        kr[i] = kKeyNone;
    }
}

// Keys for the addition phase: (source << 32 | index) keeps input order.
__global__ void make_keys_add(const uint32_t *au, const uint32_t *av, uint32_t na, uint32_t n,
                              unsigned long long *kf, unsigned long long *kr, Status *st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= na) return;
    const uint32_t u = au[i], v = av[i];
    if (u < n && v < n) {
        kf[i] = (static_cast<unsigned long long>(u) << kKeyShift) | i;
        kr[i] = (static_cast<unsigned long long>(v) << kKeyShift) | i;
    } else {
        kf[i] = kKeyNone;
        kr[i] = kKeyNone;
        atomicAdd(&st->counters[kCntInvalid], 1ull);
    }
}

// Source groups of a sorted key array, in key order: group g spans keys
// [start[g], end[g]).  Built by group_flags, a device exclusive scan of the
// flags and group_scatter, so a group's end is one load away.
struct Groups {
    const uint32_t *start;
    const uint32_t *end;
    const uint32_t *count;
};

__global__ void group_flags(const unsigned long long *keys, uint32_t m, uint32_t *flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const unsigned long long k = keys[i];
    flags[i] = (k != kKeyNone && (i == 0 || key_src(keys[i - 1]) != key_src(k))) ? 1u : 0u;
}

__global__ void group_scatter(const unsigned long long *keys, uint32_t m, const uint32_t *flags, const uint32_t *pos,
                              uint32_t *start, uint32_t *end, uint32_t *count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const unsigned long long k = keys[i];
    if (k == kKeyNone) return;
    if (flags[i]) {
        start[pos[i]] = i;
        if (pos[i] > 0) end[pos[i] - 1] = i;
    }
    if (i + 1 == m || keys[i + 1] == kKeyNone) {  // last valid key closes the last group
        end[pos[i] + flags[i] - 1] = i + 1;
        *count = pos[i] + flags[i];
    }
}

// ---------------------------------------------------------------- one sort per batch
// The four key sets of a whole batch (forward and reverse deletion keys,
// forward and reverse addition keys) are packed into one array and sorted
// by one radix sort: key = set << 2F | first << F | second with F bits per
// field (2^F > n and > the phase sizes), so the sort has 2 + 2F significant
// bits instead of four sorts of 32 + log2(n) bits.  An invalid record gets
// all-ones fields and sorts to the end of its set.  Sets occupy [0, nd),
// [nd, 2nd), [2nd, 2nd+na), [2nd+na, 2nd+2na).
struct PackedSets {
    uint32_t off[5];
    uint32_t f;  // field width F
};

__global__ void make_keys_batch(const uint32_t *du, const uint32_t *dv, uint32_t nd, const uint32_t *au,
                                const uint32_t *av, uint32_t na, uint32_t n, PackedSets ps,
                                unsigned long long *out, Status *st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = ps.off[4];
    if (i >= total) return;
    const uint32_t f = ps.f;
    const unsigned long long none = (1ull << f) - 1;
    uint32_t set, first, second;
    bool ok;
    if (i < ps.off[2]) {
        set = i < ps.off[1] ? 0u : 1u;
        const uint32_t j = i - ps.off[set];
        const uint32_t u = du[j], v = dv[j];
        ok = u < n && v < n;
        first = set == 0 ? u : v;
        second = set == 0 ? v : u;
    } else {
        set = i < ps.off[3] ? 2u : 3u;
        const uint32_t j = i - ps.off[set];
        const uint32_t u = au[j], v = av[j];
        ok = u < n && v < n;
        first = set == 2 ? u : v;
        second = j;
        if (!ok && set == 2) atomicAdd(&st->counters[kCntInvalid], 1ull);
    }
    const unsigned long long a = ok ? first : none, b = ok ? second : none;
    out[i] = (static_cast<unsigned long long>(set) << (2 * f)) | (a << f) | b;
}

// Small batches (at most kSmallSortKeys packed keys): one block sorts them
// in shared memory, instead of a device-wide radix sort whose passes are
// each a few microseconds of launch and latency.
constexpr int kSmallSortThreads = 256;
constexpr int kSmallSortItems = 16;
constexpr uint32_t kSmallSortKeys = kSmallSortThreads * kSmallSortItems;

__global__ void __launch_bounds__(kSmallSortThreads)
    sort_small(const unsigned long long *in, uint32_t total, int end_bit, unsigned long long *out) {
    using Sort = cub::BlockRadixSort<unsigned long long, kSmallSortThreads, kSmallSortItems>;
    __shared__ typename Sort::TempStorage tmp;
    unsigned long long k[kSmallSortItems];
#pragma unroll
    for (int j = 0; j < kSmallSortItems; ++j) {
        const uint32_t i = threadIdx.x * kSmallSortItems + j;
        k[j] = i < total ? in[i] : ~0ull;
    }
    Sort(tmp).Sort(k, 0, end_bit);
#pragma unroll
    for (int j = 0; j < kSmallSortItems; ++j) {
        const uint32_t i = threadIdx.x * kSmallSortItems + j;
        if (i < total) out[i] = k[j];
    }
}

// Sorted packed keys -> the usual (first << 32 | second) keys of each set,
// and group flags (first key of every source run inside its set).
__global__ void unpack_keys_batch(const unsigned long long *sorted, PackedSets ps, unsigned long long *k0,
                                  unsigned long long *k1, unsigned long long *k2, unsigned long long *k3,
                                  uint32_t *flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ps.off[4]) return;
    const uint32_t f = ps.f;
    const unsigned long long mask = (1ull << f) - 1;
    const unsigned long long k = sorted[i];
    const uint32_t set = static_cast<uint32_t>(k >> (2 * f)) & 3u;  // & 3: a small-sort pad (~0) reads as set 3
    const unsigned long long a = (k >> f) & mask, b = k & mask;
    const bool ok = a != mask;
    unsigned long long *dst = set == 0 ? k0 : set == 1 ? k1 : set == 2 ? k2 : k3;
    dst[i - ps.off[set]] = ok ? ((a << kKeyShift) | b) : kKeyNone;
    flags[i] = (ok && (i == ps.off[set] || (sorted[i - 1] >> f) != (k >> f))) ? 1u : 0u;
}

// Groups of the four sets from one exclusive scan of the flags; group
// indices and key positions are relative to the set.
struct SetGroups {
    uint32_t *start[4];
    uint32_t *end[4];
    uint32_t *count[4];
};

__global__ void group_scatter_batch(const unsigned long long *sorted, PackedSets ps, const uint32_t *flags,
                                    const uint32_t *pos, SetGroups sg) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ps.off[4]) return;
    const uint32_t f = ps.f;
    const unsigned long long mask = (1ull << f) - 1;
    const unsigned long long k = sorted[i];
    if (((k >> f) & mask) == mask) return;  // invalid record
    const uint32_t set = static_cast<uint32_t>(k >> (2 * f)) & 3u;  // & 3: a small-sort pad (~0) reads as set 3
    const uint32_t s0 = ps.off[set], s1 = ps.off[set + 1];
    const uint32_t base = pos[s0];
    const uint32_t local = i - s0;
    const uint32_t g = pos[i] - base;
    if (flags[i]) {
        sg.start[set][g] = local;
        if (g > 0) sg.end[set][g - 1] = local;
    }
    if (i + 1 == s1 || ((sorted[i + 1] >> f) & mask) == mask) {  // last valid key of the set
        sg.end[set][g + flags[i] - 1] = local + 1;
        *sg.count[set] = g + flags[i];
    }
}

// Deletion run of key `key` inside the group [gs, ge): the index of the
// run's first key (a unique run id) and its requested count.
__device__ __forceinline__ bool find_run(const unsigned long long *keys, uint32_t gs, uint32_t ge,
                                         unsigned long long key, uint32_t &run, uint32_t &req) {
    uint32_t lo = gs, hi = ge;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo >= ge || keys[lo] != key) return false;
    uint32_t e = lo + 1;
    while (e < ge && keys[e] == key) ++e;
    run = lo;
    req = e - lo;
    return true;
}

__device__ __forceinline__ void write_slot(const AdjView &view, unsigned long long off, uint32_t value) {
    *view.wptr(off) = value;
}

// Record the tombstones a row received; queue it for compaction when they
// reach a quarter of its length.
__device__ __forceinline__ void finish_row(RowDesc *desc, uint32_t u, const RowDesc &d, uint32_t removed,
                                           uint32_t *compact, uint32_t *compact_count) {
    if (!removed) return;
    const uint32_t tombs = rd_tombs(d) + removed;
    desc[u].meta = rd_meta(rd_cls(d), tombs);
    if (4ull * tombs >= d.len || tombs >= kMaxTombs / 2) compact[atomicAdd(compact_count, 1u)] = u;
}

// ---------------------------------------------------------------- deletion

// Rows of at most kWarpRowMax slots, at most 32 keys: lane j holds key j;
// run multiplicities and matched counts live in the run-head lanes.
// Returns the number of tombstones written.
__device__ __forceinline__ uint32_t warp_tomb_regs(const AdjView &view, const RowDesc &d,
                                                   const unsigned long long *keys, uint32_t gs, uint32_t m) {
    const uint32_t lane = lane_id();
    const bool kvalid = lane < m;
    const uint32_t kd = kvalid ? key_low(keys[gs + lane]) : 0u;
    const uint32_t vmask = __ballot_sync(kFull, kvalid);
    const uint32_t peers = __match_any_sync(kFull, kd) & vmask;
    const uint32_t req_here = kvalid ? __popc(peers) : 0u;
    uint32_t mcount = 0;
    uint32_t left = m;  // requests not yet satisfied (uniform)
    const uint32_t *src = view.at(d.off);
    uint32_t *dst = nullptr;
    uint4 q = make_uint4(0, 0, 0, 0);
    if (4u * lane < d.len) q = *reinterpret_cast<const uint4 *>(src + 4u * lane);
    for (uint32_t base = 0; base < d.len && left; base += 128u) {
        const uint32_t k0 = base + 4u * lane;
        const uint32_t e[4] = {q.x, q.y, q.z, q.w};
        // prefetch the next chunk while this one is matched
        if (base + 128u + 4u * lane < d.len) q = *reinterpret_cast<const uint4 *>(src + base + 128u + 4u * lane);
        int run[4] = {-1, -1, -1, -1};
        for (uint32_t j = 0; j < m; ++j) {
            const uint32_t kj = __shfl_sync(kFull, kd, j);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (run[s] < 0 && k0 + s < d.len && e[s] == kj) run[s] = static_cast<int>(j);
        }
        uint32_t cm[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) cm[s] = __ballot_sync(kFull, run[s] >= 0);
        uint32_t any = cm[0] | cm[1] | cm[2] | cm[3];
        bool del[4] = {false, false, false, false};
        while (any) {  // position order: lane-major, then s
            const uint32_t l = __ffs(any) - 1;
            any &= any - 1;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if ((cm[s] >> l) & 1u) {
                    const uint32_t r = static_cast<uint32_t>(__shfl_sync(kFull, run[s], l));
                    const uint32_t req = __shfl_sync(kFull, req_here, r);
                    const uint32_t seen = __shfl_sync(kFull, mcount, r);
                    if (lane == r) mcount = seen + 1;
                    if (seen < req) {
                        --left;
                        if (lane == l) del[s] = true;
                    }
                }
            }
        }
        if (del[0] | del[1] | del[2] | del[3]) {
            if (!dst) dst = view.wptr(d.off);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (del[s]) dst[k0 + s] = kTomb;
        }
        __syncwarp();
    }
    return m - left;
}

// Any number of keys: binary search in the sorted group keys in global
// memory; matched[run] counts the occurrences of a run seen so far.
__device__ __forceinline__ uint32_t warp_tomb_global(const AdjView &view, const RowDesc &d, uint32_t u,
                                                     const unsigned long long *keys, uint32_t gs, uint32_t ge,
                                                     uint32_t *matched) {
    const uint32_t lane = lane_id();
    const unsigned long long uhi = static_cast<unsigned long long>(u) << kKeyShift;
    uint32_t left = ge - gs, done = 0;
    for (uint32_t base = 0; base < d.len && left; base += 32u) {
        const uint32_t k = base + lane;
        const bool valid = k < d.len;
        const uint32_t x = valid ? *view.at(d.off + k) : kTomb;
        uint32_t run = 0xFFFFFFFFu, req = 0;
        const bool cand = x != kTomb && find_run(keys, gs, ge, uhi | x, run, req);
        bool del = false;
        if (__ballot_sync(kFull, cand)) {
            const uint32_t peers = __match_any_sync(kFull, run);
            const uint32_t before = __popc(peers & lanemask_lt());
            uint32_t seen = 0;
            if (cand) seen = matched[run];
            del = cand && seen + before < req;
            __syncwarp();
            if (cand && before == 0) matched[run] = seen + __popc(peers);
            __syncwarp();
        }
        const uint32_t dm = __ballot_sync(kFull, del);
        if (del) write_slot(view, d.off + k, kTomb);
        left -= __popc(dm);
        done += __popc(dm);
    }
    return done;
}

// Deletion phase, one warp per source group; rows above kWarpRowMax go to
// the block path.  Launched with kMutWarps * 32 threads per block.
__global__ void __launch_bounds__(kMutWarps * 32)
    mutate_delete(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr, const uint32_t *list,
                  const uint32_t *list_count, uint32_t *matched, uint32_t *big, uint32_t *big_count,
                  uint32_t *compact, uint32_t *compact_count, unsigned long long *stats, Status *st) {
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nl = *list_count;
    unsigned long long removed = 0, changed = 0;
    for (uint32_t li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < nl; li += warps) {
        const uint32_t g = list[li];
        const uint32_t gs = gr.start[g];
        const uint32_t ge = gr.end[g];
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        if (d.len > kWarpRowMax) {
            if (lane == 0) big[atomicAdd(big_count, 1u)] = g;
            continue;
        }
        const uint32_t done = (ge - gs <= 32u) ? warp_tomb_regs(view, d, keys, gs, ge - gs)
                                               : warp_tomb_global(view, d, u, keys, gs, ge, matched);
        if (lane == 0) {
            finish_row(desc, u, d, done, compact, compact_count);
            removed += done;
            changed += done != 0;
        }
    }
    if (lane == 0 && stats) {
        if (removed) atomicAdd(&stats[kCntRemoved], removed);
        if (changed) atomicAdd(&stats[kCntChanged], changed);
    }
}

// Rows above kWarpRowMax: one block per row, tiles of kTpbMut x 8 slots
// (two 16-byte loads per thread), the group's keys and matched counts in
// shared memory (up to kBigKeys keys, beyond that in global memory), a
// 4096-bit filter in front of the key search; candidates resolved in
// position order by one thread; the scan stops once every request of the
// row is satisfied.
constexpr int kBigItems = 8;
constexpr uint32_t kBigKeys = 2048;
constexpr uint32_t kFilterBits = 4096;

__device__ __forceinline__ uint32_t filter_hash(uint32_t x) { return (x * 0x9E3779B1u) >> 20; }  // 12 bits

__global__ void __launch_bounds__(kTpbMut)
    mutate_delete_big(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr, const uint32_t *big,
                      const uint32_t *big_count, uint32_t *matched, uint32_t *compact, uint32_t *compact_count,
                      unsigned long long *stats, Status *st) {
    __shared__ uint32_t skey[kBigKeys];
    __shared__ uint32_t scount[kBigKeys];
    __shared__ uint32_t filter[kFilterBits / 32];
    __shared__ uint8_t cand_bits[kTpbMut];
    __shared__ uint8_t del_bits[kTpbMut];
    __shared__ uint16_t cand_run[kTpbMut * kBigItems];
    __shared__ uint32_t g_run[kTpbMut * kBigItems];
    __shared__ uint32_t cand_warp[kTpbMut / 32];
    __shared__ uint32_t left;
    const uint32_t tid = threadIdx.x;
    const uint32_t nb = *big_count;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t gs = gr.start[big[b]];
        const uint32_t ge = gr.end[big[b]];
        const uint32_t gm = ge - gs;
        const bool in_smem = gm <= kBigKeys;
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const unsigned long long uhi = static_cast<unsigned long long>(u) << kKeyShift;
        for (uint32_t i = tid; i < kFilterBits / 32; i += kTpbMut) filter[i] = 0;
        if (tid == 0) left = gm;
        __syncthreads();
        for (uint32_t j = tid; j < gm; j += kTpbMut) {
            const uint32_t x = key_low(keys[gs + j]);
            if (in_smem) {
                skey[j] = x;
                scount[j] = 0;
            }
            const uint32_t h = filter_hash(x);
            atomicOr(&filter[h >> 5], 1u << (h & 31u));
        }
        __syncthreads();
        for (uint32_t base = 0; base < d.len; base += kTpbMut * kBigItems) {
            const uint32_t k0 = base + tid * kBigItems;
            uint32_t e[kBigItems];
#pragma unroll
            for (int h = 0; h < kBigItems; h += 4) {
                if (k0 + h < d.len) {
                    const uint4 q = *reinterpret_cast<const uint4 *>(view.at(d.off + k0 + h));
                    e[h] = q.x;
                    e[h + 1] = q.y;
                    e[h + 2] = q.z;
                    e[h + 3] = q.w;
                } else {
                    e[h] = e[h + 1] = e[h + 2] = e[h + 3] = kTomb;
                }
            }
            uint32_t cb = 0;
#pragma unroll
            for (int s = 0; s < kBigItems; ++s) {
                if (k0 + s >= d.len || e[s] == kTomb) continue;
                const uint32_t h = filter_hash(e[s]);
                if (!((filter[h >> 5] >> (h & 31u)) & 1u)) continue;
                if (in_smem) {
                    uint32_t lo = 0, hi = gm;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (skey[mid] < e[s])
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    if (lo < gm && skey[lo] == e[s]) {
                        cb |= 1u << s;
                        cand_run[tid * kBigItems + s] = static_cast<uint16_t>(lo);
                    }
                } else {
                    uint32_t run, req;
                    if (find_run(keys, gs, ge, uhi | e[s], run, req)) {
                        cb |= 1u << s;
                        g_run[tid * kBigItems + s] = run;
                    }
                }
            }
            cand_bits[tid] = static_cast<uint8_t>(cb);
            del_bits[tid] = 0;
            const uint32_t wmask = __ballot_sync(kFull, cb != 0);
            if ((tid & 31u) == 0) cand_warp[tid >> 5] = wmask;
            if (__syncthreads_or(cb != 0)) {
                if (tid == 0) {
                    // Visit only the threads that hold candidates, in position order.
                    uint32_t l = left;
                    for (uint32_t wi = 0; wi < kTpbMut / 32; ++wi) {
                        for (uint32_t tm = cand_warp[wi]; tm; tm &= tm - 1) {
                            const uint32_t t = wi * 32 + __ffs(tm) - 1;
                            uint32_t b = cand_bits[t];
                            uint32_t dbits = 0;
                            while (b) {
                                const uint32_t s = __ffs(b) - 1;
                                b &= b - 1;
                                bool del;
                                if (in_smem) {
                                    const uint32_t r = cand_run[t * kBigItems + s];
                                    uint32_t e2 = r + 1;
                                    while (e2 < gm && skey[e2] == skey[r]) ++e2;
                                    del = scount[r] < e2 - r;
                                    scount[r] += 1;
                                } else {
                                    const uint32_t r = g_run[t * kBigItems + s];
                                    uint32_t e2 = r + 1;
                                    while (e2 < ge && keys[e2] == keys[r]) ++e2;
                                    del = matched[r] < e2 - r;
                                    matched[r] += 1;
                                }
                                if (del) {
                                    dbits |= 1u << s;
                                    --l;
                                }
                            }
                            del_bits[t] = static_cast<uint8_t>(dbits);
                        }
                    }
                    left = l;
                }
                __syncthreads();
                const uint32_t db = del_bits[tid];
#pragma unroll
                for (int s = 0; s < kBigItems; ++s)
                    if ((db >> s) & 1u) write_slot(view, d.off + k0 + s, kTomb);
            }
            __syncthreads();
            if (left == 0) break;
        }
        if (tid == 0) {
            const uint32_t done = gm - left;
            finish_row(desc, u, d, done, compact, compact_count);
            if (done && stats) {
                atomicAdd(&stats[kCntRemoved], static_cast<unsigned long long>(done));
                atomicAdd(&stats[kCntChanged], 1ull);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- flat deletion
//
// When no destination is requested twice for the same source in a batch
// (every run has one key), the entry to tombstone for a key is simply the
// first live occurrence, i.e. the minimum matching position, which an
// atomicMin finds in any order.  Such rows are scanned in 512-entry warp
// chunks spread evenly over the whole grid (a hub row no longer serialises
// on one block); rows with repeated requests keep the position-ordered
// kernels above.
constexpr uint32_t kDelChunk = 512;
constexpr uint32_t kSmemKeys = 256;

// Classify groups: chunk count for flat rows, ordered list for the rest.
// `chunks` must be zero beyond the group count (it is scanned whole).
// Kinds of deletion groups: rows with repeated requests take the ordered
// kernels; rows with distinct requests the flat scan, or the position index
// when the row is indexed (posindex.cuh).
enum : uint8_t { kGroupOrdered = 0, kGroupChunked = 1, kGroupIndexed = 2 };

// Also clears the phase's per-key arrays (the scan chunk counts past the
// groups, the first-match positions, the ordered path's match counts) for
// the m keys, in place of three memsets.
__global__ void del_classify(const RowDesc *desc, const unsigned long long *keys, Groups gr, uint32_t *chunks,
                             uint8_t *gtype, uint32_t *ordered, uint32_t *ordered_count, PosIndex ix,
                             uint32_t *indexed, uint32_t *indexed_count, uint32_t m, uint32_t *firstpos,
                             uint32_t *matched) {
    const uint32_t ng = *gr.count;
    const uint32_t rounded = (ng + 31u) & ~31u;
    const uint32_t lane = lane_id();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        firstpos[i] = kInf;
        matched[i] = 0u;
        if (i >= ng) chunks[i] = 0u;
    }
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < rounded; g += gridDim.x * blockDim.x) {
        bool dup = false, by_index = false;
        uint32_t gs = 0, ge = 0;
        if (g < ng) {
            gs = gr.start[g];
            ge = gr.end[g];
            // Repeated requests are adjacent in the sorted keys; a lane checks
            // its own group when it is short, the warp checks long ones (hub
            // rows draw hundreds of deletions) together below.
            if (ge - gs <= 32u)
                for (uint32_t i = gs; i + 1 < ge && !dup; ++i) dup = keys[i] == keys[i + 1];
        }
        uint32_t longs = __ballot_sync(kFull, g < ng && ge - gs > 32u);
        while (longs) {
            const int l = __ffs(longs) - 1;
            longs &= longs - 1;
            const uint32_t ls = __shfl_sync(kFull, gs, l);
            const uint32_t le = __shfl_sync(kFull, ge, l);
            bool any = false;
            for (uint32_t i = ls + lane; i + 1 < le; i += 32u) any |= keys[i] == keys[i + 1];
            any = __any_sync(kFull, any);
            if (lane == static_cast<uint32_t>(l)) dup = any;
        }
        if (g < ng) {
            const uint32_t u = key_src(keys[gs]);
            by_index = !dup && idx_row(ix, u);
            gtype[g] = dup ? kGroupOrdered : by_index ? kGroupIndexed : kGroupChunked;
            chunks[g] = (dup || by_index) ? 0u : (desc[u].len + kDelChunk - 1) / kDelChunk;
        }
        warp_enqueue(dup, g, ordered, ordered_count, 0xFFFFFFFFu, nullptr);
        warp_enqueue(by_index, g, indexed, indexed_count, 0xFFFFFFFFu, nullptr);
    }
}

// Indexed rows with distinct requests: the first live position of every key
// from the index; the entry loses one occurrence and, when more remain, moves
// to the next one (a scan from the deleted position on, rare: parallel
// edges).  The tombstone is written here at once (the position is final),
// and the position is recorded with kApplied set so that del_apply skips
// it.  A warp deals the keys of its groups of up to kLaneKeys keys one per
// lane (del_index); larger groups get a warp each, and groups of more than
// kHugeKeys keys the whole grid (del_index_wide).
constexpr uint32_t kLaneKeys = 4;
constexpr uint32_t kHugeKeys = 256;
constexpr uint32_t kApplied = 0x80000000u;  // firstpos flag: tombstone already written

// `count_tomb`: add the tombstone to the row's descriptor here (callers that
// serve many keys of one row add their warp's total once instead).
__device__ __forceinline__ uint32_t del_index_key(const AdjView &view, RowDesc *desc, const RowDesc &d, uint32_t u,
                                                  uint32_t v, uint32_t *fp, const PosIndex &ix, Status *st,
                                                  bool count_tomb = true) {
    const unsigned long long s = idx_find(ix, (static_cast<unsigned long long>(u) << 32) | v);
    if (s == ~0ull) return 0u;  // not in the row: a missing delete
    const uint2 e = ix.val[s];
    if (e.y == 0u || e.x >= d.len) {
        if (e.y != 0u) set_error(st, kErrInternal, 0x1d2u);
        return 0u;
    }
    *fp = e.x | kApplied;
    write_slot(view, d.off + e.x, kTomb);
    if (count_tomb) atomicAdd(&desc[u].meta, 1u << 6);
    if (e.y == 1u) {
        ix.val[s] = make_uint2(kInf, 0u);
        ix.keys[s] = kIdxDeleted;
    } else {
        uint32_t q = e.x + 1;
        while (q < d.len && *view.at(d.off + q) != v) ++q;
        if (q >= d.len) set_error(st, kErrInternal, 0x1d3u);
        ix.val[s] = make_uint2(q < d.len ? q : kInf, e.y - 1u);
    }
    return 1u;
}

// The keys of one lane, N at a time (live[j]: key j is served): the key,
// descriptor, first index probe and its value slot of every key are read
// before any of them is used, so the lane waits for one chain of dependent
// loads instead of N.  The first probe almost always decides (the tables
// stay at most half full); a collision continues with idx_find_from.
template <int N>
__device__ __forceinline__ uint32_t del_index_keys(const AdjView &view, RowDesc *desc,
                                                   const unsigned long long *keys, const uint32_t (&ks)[N],
                                                   const bool (&live)[N], uint32_t *firstpos, const PosIndex &ix,
                                                   Status *st) {
    unsigned long long key[N], slot[N], seen[N];
    RowDesc d[N];
    uint2 e[N];
#pragma unroll
    for (int j = 0; j < N; ++j) key[j] = live[j] ? keys[ks[j]] : 0ull;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const uint32_t u = key_src(key[j]);
        if (live[j]) d[j] = desc[u];
        key[j] = (static_cast<unsigned long long>(u) << 32) | key_low(key[j]);
        slot[j] = idx_mix(key[j]) & ix.mask;
        seen[j] = kIdxEmpty + 0ull;
        if (live[j]) seen[j] = *reinterpret_cast<volatile unsigned long long *>(ix.keys + slot[j]);
        e[j] = live[j] ? ix.val[slot[j]] : make_uint2(0u, 0u);
    }
    uint32_t removed = 0;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        if (!live[j]) continue;
        if (seen[j] != key[j]) {
            if (seen[j] == kIdxEmpty) continue;  // not in the row: a missing delete
            slot[j] = idx_find_from(ix, key[j], (slot[j] + 1) & ix.mask, 1);
            if (slot[j] == ~0ull) continue;
            e[j] = ix.val[slot[j]];
        }
        const uint32_t u = static_cast<uint32_t>(key[j] >> 32), v = static_cast<uint32_t>(key[j]);
        if (e[j].y == 0u || e[j].x >= d[j].len) {
            if (e[j].y != 0u) set_error(st, kErrInternal, 0x1d2u);
            continue;
        }
        firstpos[ks[j]] = e[j].x | kApplied;
        write_slot(view, d[j].off + e[j].x, kTomb);
        atomicAdd(&desc[u].meta, 1u << 6);
        if (e[j].y == 1u) {
            ix.val[slot[j]] = make_uint2(kInf, 0u);
            ix.keys[slot[j]] = kIdxDeleted;
        } else {
            uint32_t q = e[j].x + 1;
            while (q < d[j].len && *view.at(d[j].off + q) != v) ++q;
            if (q >= d[j].len) set_error(st, kErrInternal, 0x1d3u);
            ix.val[slot[j]] = make_uint2(q < d[j].len ? q : kInf, e[j].y - 1u);
        }
        ++removed;
    }
    return removed;
}

__global__ void __launch_bounds__(256, 4)
    del_index(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr,
                          const uint32_t *list, const uint32_t *count, uint32_t *firstpos, PosIndex ix,
                          uint32_t *wide, uint32_t *wide_count, uint32_t *huge, uint32_t *huge_count,
                          unsigned long long *stats, Status *st) {
    const uint32_t lane = lane_id();
    uint32_t removed = 0;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nl = *count;
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < nl; base += warps * 32u) {
        const uint32_t i = base + lane;
        uint32_t g = 0, gs = 0, nk = 0;
        if (i < nl) {
            g = list[i];
            gs = gr.start[g];
            nk = gr.end[g] - gs;
        }
        // The warp's small groups (up to kLaneKeys keys) are concatenated (a
        // warp scan of their sizes) and their keys dealt one per lane, at
        // most kLaneKeys steps; distinct keys of a row are independent.
        const bool small_g = i < nl && nk <= kLaneKeys;
        const uint32_t mine = small_g ? nk : 0u;
        uint32_t incl = mine;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const uint32_t excl = incl - mine;
        const uint32_t total = __shfl_sync(kFull, incl, 31);  // at most 32 * kLaneKeys
        uint32_t ks[kLaneKeys];
        bool live[kLaneKeys];
#pragma unroll
        for (int j = 0; j < static_cast<int>(kLaneKeys); ++j) {
            const uint32_t e = 32u * j + lane;
            ks[j] = 0;
            live[j] = false;
            if (32u * j < total) {  // warp-uniform
                uint32_t lo = 0, hi = 32;  // the last lane whose keys start at or before e
#pragma unroll
                for (int step = 0; step < 5; ++step) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (__shfl_sync(kFull, excl, mid) <= e)
                        lo = mid;
                    else
                        hi = mid;
                }
                ks[j] = __shfl_sync(kFull, gs, lo) + (e - __shfl_sync(kFull, excl, lo));
                live[j] = e < total;
            }
        }
        removed += del_index_keys<kLaneKeys>(view, desc, keys, ks, live, firstpos, ix, st);
        // Larger groups go to del_index_wide: up to kHugeKeys keys one warp
        // per group, more (hub rows, where uniform deletions over the edges
        // concentrate) across the whole grid in 32-key chunks.
        warp_enqueue(i < nl && nk > kLaneKeys && nk <= kHugeKeys, g, wide, wide_count, nl, st);
        warp_enqueue(i < nl && nk > kHugeKeys, g, huge, huge_count, nl, st);
    }
    if (stats) warp_count(&stats[kCntRemoved], removed);
}

__global__ void del_index_wide(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr,
                               const uint32_t *wide, const uint32_t *wide_count, const uint32_t *huge,
                               const uint32_t *huge_count, uint32_t *firstpos, PosIndex ix,
                               unsigned long long *stats, Status *st) {
    const uint32_t lane = lane_id();
    uint32_t removed = 0;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = *wide_count;
    for (uint32_t i = wid; i < nw; i += warps) {
        const uint32_t g = wide[i];
        const uint32_t gs = gr.start[g];
        const uint32_t nk = gr.end[g] - gs;
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        uint32_t tombs = 0;
        for (uint32_t j = lane; j < nk; j += 32u)
            tombs += del_index_key(view, desc, d, u, key_low(keys[gs + j]), firstpos + gs + j, ix, st, false);
        tombs = __reduce_add_sync(kFull, tombs);
        if (lane == 0 && tombs) atomicAdd(&desc[u].meta, tombs << 6);
        removed += lane == 0 ? tombs : 0u;
    }
    // Huge groups: chunk c of the concatenated 32-key chunks goes to warp
    // c mod warps; every warp walks the (short) list in the same order.
    const uint32_t nh = *huge_count;
    uint64_t prefix = 0;
    for (uint32_t h = 0; h < nh; ++h) {
        const uint32_t g = huge[h];
        const uint32_t gs = gr.start[g];
        const uint32_t nk = gr.end[g] - gs;
        const uint64_t chunks = (nk + 31u) / 32u;
        uint64_t c = prefix + (wid + warps - static_cast<uint32_t>(prefix % warps)) % warps;
        if (c < prefix + chunks) {
            const uint32_t u = key_src(keys[gs]);
            const RowDesc d = desc[u];
            uint32_t tombs = 0;
            for (; c < prefix + chunks; c += warps) {
                const uint32_t j = static_cast<uint32_t>(c - prefix) * 32u + lane;
                if (j < nk)
                    tombs += del_index_key(view, desc, d, u, key_low(keys[gs + j]), firstpos + gs + j, ix, st, false);
            }
            tombs = __reduce_add_sync(kFull, tombs);
            if (lane == 0 && tombs) atomicAdd(&desc[u].meta, tombs << 6);
            removed += lane == 0 ? tombs : 0u;
        }
        prefix += chunks;
    }
    if (stats) warp_count(&stats[kCntRemoved], removed);
}

// After the ordered kernels: the entries of every key of an ordered group on
// an indexed row are recounted from the row (rare: repeated requests).
__global__ void idx_fix_ordered(AdjView view, const RowDesc *desc, const unsigned long long *keys, Groups gr,
                                const uint32_t *ordered, const uint32_t *ordered_count, PosIndex ix, Status *st) {
    const uint32_t no = *ordered_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < no; i += gridDim.x * blockDim.x) {
        const uint32_t g = ordered[i];
        const uint32_t gs = gr.start[g];
        const uint32_t ge = gr.end[g];
        const uint32_t u = key_src(keys[gs]);
        if (!idx_row(ix, u)) continue;
        const RowDesc d = desc[u];
        for (uint32_t j = gs; j < ge; ++j) {
            if (j > gs && keys[j] == keys[j - 1]) continue;  // one pass per distinct key
            const uint32_t v = key_low(keys[j]);
            const unsigned long long s = idx_find(ix, (static_cast<unsigned long long>(u) << 32) | v);
            if (s == ~0ull) continue;
            uint32_t first = kInf, live = 0;
            for (uint32_t q = 0; q < d.len; ++q)
                if (*view.at(d.off + q) == v) {
                    if (first == kInf) first = q;
                    ++live;
                }
            ix.val[s] = make_uint2(first, live);
            if (!live) ix.keys[s] = kIdxDeleted;
        }
    }
}

// Chunk runs are dealt round-robin to the warps: run r (kDelRun consecutive
// 512-entry chunks) goes to warp r mod warps, so the chunks of one long row
// spread over the whole grid while a warp still reuses a row's keys for a
// few chunks.  `chunk_map[c]` is the group of chunk c (del_chunk_map);
// `chunk_end` is the inclusive prefix sum of `chunks` over scan_n entries.
// Each chunk records the first live match of every key (atomicMin).
//
// Membership test per row entry, by the row's number of requests: up to
// kDelCmpKeys, compare against the keys held in lanes (about 9 instructions
// per request per 4 entries, no divergence); beyond, a per-warp bit filter in
// shared memory (32 bits per request rounded up to a power of two,
// 1024..16384 bits, one multiplicative hash) built once per group, and a
// binary search on a filter hit.  (Filters for rows of 3..8 requests, in
// shared memory or in a 64-bit register, measured 40-50 % slower on the
// whole scan: their hits diverge inside the warp.)
constexpr uint32_t kDelCmpKeys = 8;
constexpr uint32_t kDelFilterWords = 512;

__device__ __forceinline__ uint32_t del_hash(uint32_t y, uint32_t shift) { return (y * 2654435761u) >> shift; }

constexpr uint32_t kDelRun = 4;

// chunk_map[c] = group of chunk c; one warp per group, lanes over its chunks.
__global__ void del_chunk_map(Groups gr, const uint32_t *chunk_end, uint32_t *chunk_map) {
    const uint32_t ng = *gr.count;
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ng; g += warps) {
        const uint32_t c0 = g ? chunk_end[g - 1] : 0u, c1 = chunk_end[g];
        for (uint32_t c = c0 + lane; c < c1; c += 32u) chunk_map[c] = g;
    }
}

__global__ void __launch_bounds__(kMutWarps * 32)
    del_scan(AdjView view, const RowDesc *desc, const unsigned long long *keys, Groups gr, const uint32_t *chunk_end,
             const uint32_t *chunk_map, uint32_t scan_n, uint32_t *firstpos, unsigned long long *stats,
             uint32_t *seg_hot) {
    __shared__ uint32_t skeys[kMutWarps][kSmemKeys];
    __shared__ uint32_t sfilt[kMutWarps][kDelFilterWords];
    uint32_t *sk = skeys[threadIdx.x >> 5];
    uint32_t *filt = sfilt[threadIdx.x >> 5];
    const uint32_t lane = lane_id();
    const uint32_t total = scan_n ? chunk_end[scan_n - 1] : 0u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t g_ready = ~0u;  // group whose keys are loaded in kd / filt / sk
    uint32_t gs = 0, ge = 0, nk = 0, kd = 0, fshift = 18;
    RowDesc d{};
    unsigned long long uhi = 0;
    uint32_t scanned = 0, scanned_cached = 0;
    for (uint32_t c = wid * kDelRun; c < total; c += (c % kDelRun == kDelRun - 1) ? (warps - 1) * kDelRun + 1 : 1) {
        const uint32_t g = chunk_map[c];
        if (g != g_ready) {
            __syncwarp();
            g_ready = g;
            gs = gr.start[g];
            ge = gr.end[g];
            nk = ge - gs;
            const uint32_t u = key_src(keys[gs]);
            d = desc[u];
            uhi = static_cast<unsigned long long>(u) << kKeyShift;
            kd = lane < nk ? key_low(keys[gs + lane]) : 0u;
            if (nk > kDelCmpKeys) {
                // words = nk rounded up to a power of two in [32, 512]
                const uint32_t words = min(kDelFilterWords, max(32u, 1u << (32 - __clz(nk - 1))));
                fshift = 32u - (5u + (31u - __clz(words)));  // hash -> log2(32 * words) bits
                for (uint32_t j = lane; j < words; j += 32u) filt[j] = 0u;
                __syncwarp();
                for (uint32_t j = lane; j < nk; j += 32u) {
                    const uint32_t y = key_low(keys[gs + j]);
                    const uint32_t h = del_hash(y, fshift);
                    atomicOr(filt + (h >> 5), 1u << (h & 31u));
                    if (nk <= kSmemKeys) sk[j] = y;
                }
            }
            __syncwarp();
        }
        const uint32_t k0 = (c - (g ? chunk_end[g - 1] : 0u)) * kDelChunk;
        // A 512-entry chunk never straddles a segment (segments hold 2^14).
        const uint32_t *src = view.at(d.off + k0);
        const uint32_t len_here = min(kDelChunk, d.len - k0);
        scanned += len_here;
        if (view.cached(d.off + k0)) scanned_cached += len_here;
        if (seg_hot && lane == 0) atomicAdd(seg_hot + ((d.off + k0) >> kSegShift), len_here);
        // Short rows (most groups) end after one or two 128-entry steps.
        const uint32_t steps = (len_here + 127u) / 128u;
        uint4 q[kDelChunk / 128u];
#pragma unroll
        for (uint32_t s = 0; s < kDelChunk / 128u; ++s) {
            const uint32_t kk = k0 + 128u * s + 4u * lane;
            q[s] = (s < steps && kk < d.len) ? *reinterpret_cast<const uint4 *>(src + 128u * s + 4u * lane)
                                             : make_uint4(kTomb, kTomb, kTomb, kTomb);
        }
#pragma unroll
        for (uint32_t s = 0; s < kDelChunk / 128u; ++s) {
            if (s >= steps) continue;  // warp-uniform; keeps the loop unrolled (q[] in registers)
            const uint32_t kk = k0 + 128u * s + 4u * lane;
            uint32_t e[4] = {q[s].x, q[s].y, q[s].z, q[s].w};
#pragma unroll
            for (int t = 0; t < 4; ++t)
                if (kk + t >= d.len) e[t] = kTomb;
            if (nk <= kDelCmpKeys) {
                int hit[4] = {-1, -1, -1, -1};
                for (uint32_t j = 0; j < nk; ++j) {
                    const uint32_t kj = __shfl_sync(kFull, kd, j);
#pragma unroll
                    for (int t = 0; t < 4; ++t)
                        if (e[t] == kj) hit[t] = static_cast<int>(j);
                }
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (hit[t] >= 0 && e[t] != kTomb) atomicMin(firstpos + gs + hit[t], kk + t);
            } else {
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    if (e[t] == kTomb) continue;
                    const uint32_t h = del_hash(e[t], fshift);
                    if (!((filt[h >> 5] >> (h & 31u)) & 1u)) continue;
                    int hit = -1;
                    if (nk <= kSmemKeys) {
                        uint32_t a = 0, b = nk;
                        while (a < b) {
                            const uint32_t mid = (a + b) >> 1;
                            if (sk[mid] < e[t])
                                a = mid + 1;
                            else
                                b = mid;
                        }
                        if (a < nk && sk[a] == e[t]) hit = static_cast<int>(a);
                    } else {
                        uint32_t run, req;
                        if (find_run(keys, gs, ge, uhi | e[t], run, req)) hit = static_cast<int>(run - gs);
                    }
                    if (hit >= 0) atomicMin(firstpos + gs + hit, kk + t);
                }
            }
        }
    }
    if (stats) {
        // lane 0 of every warp holds the warp's totals (all lanes counted the same chunks)
        if (lane == 0 && scanned) atomicAdd(&stats[kCntDelScanned], static_cast<unsigned long long>(scanned));
        if (lane == 0 && scanned_cached)
            atomicAdd(&stats[kCntDelScannedCached], static_cast<unsigned long long>(scanned_cached));
    }
}

// Tombstone the first match of every key found by del_scan.
__global__ void del_apply(AdjView view, RowDesc *desc, const unsigned long long *keys, uint32_t m,
                          const uint32_t *firstpos, unsigned long long *stats) {
    uint32_t removed = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (m + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += stride) {
        if (i < m) {
            const uint32_t p = firstpos[i];
            if (p != kInf && !(p & kApplied)) {
                const uint32_t u = key_src(keys[i]);
                write_slot(view, desc[u].off + p, kTomb);
                atomicAdd(&desc[u].meta, 1u << 6);
                ++removed;
            }
        }
    }
    if (stats) warp_count(&stats[kCntRemoved], removed);
}

// Queue flat rows whose tombstones reached a quarter of their length.
__global__ void del_finish(const RowDesc *desc, const unsigned long long *keys, Groups gr, const uint8_t *gtype,
                           const uint32_t *firstpos, uint32_t *compact, uint32_t *compact_count,
                           unsigned long long *stats) {
    const uint32_t ng = *gr.count;
    const uint32_t rounded = (ng + 31u) & ~31u;
    uint32_t changed = 0;
    // Warp-aggregated appends and counts: ~10^5 rows per batch would
    // otherwise queue on one counter address.
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < rounded; g += gridDim.x * blockDim.x) {
        bool want = false;
        uint32_t u = 0;
        if (g < ng && gtype[g] != kGroupOrdered) {  // flat group (scanned or indexed)
            const uint32_t gs = gr.start[g];
            const uint32_t ge = gr.end[g];
            bool any = false;
            for (uint32_t i = gs; i < ge && !any; ++i) any = firstpos[i] != kInf;
            if (any) {
                ++changed;
                u = key_src(keys[gs]);
                const RowDesc d = desc[u];
                const uint32_t tombs = rd_tombs(d);
                want = 4ull * tombs >= d.len || tombs >= kMaxTombs / 2;
            }
        }
        warp_enqueue(want, u, compact, compact_count, 0xFFFFFFFFu, nullptr);
    }
    if (stats) warp_count(&stats[kCntChanged], changed);
}

// ---------------------------------------------------------------- index upkeep
// The live entries of an indexed row moved (compaction, relocation): the
// first positions of its keys are recomputed over the row's first `len`
// slots at `off` (two passes, reset then minimum).  Block-wide and warp-wide
// forms; all threads of the block (warp) call.
// One pass over the entries t, t + stride, ... of the row: `set` false
// clears every key's first position, true lowers it to the entry's
// position.  Four entries per thread at a time, their row reads and index
// probes in flight together.
__device__ __forceinline__ void idx_reposition_pass(const AdjView &view, const PosIndex &ix, uint32_t u,
                                                    uint64_t off, uint32_t len, uint32_t t, uint32_t stride, bool set,
                                                    Status *st) {
    constexpr int N = 4;
    for (uint32_t base = t; base < len; base += N * stride) {
        uint32_t v[N];
        bool live[N];
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const uint32_t k = base + j * stride;
            live[j] = k < len;
            v[j] = live[j] ? __ldcg(view.at(off + k)) : 0u;
        }
        unsigned long long slot[N];
        idx_find_n<N>(ix, u, v, live, slot, st);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            if (slot[j] == ~0ull) continue;
            if (set)
                atomicMin(&ix.val[slot[j]].x, base + j * stride);
            else
                atomicExch(&ix.val[slot[j]].x, kInf);
        }
    }
}

__device__ __forceinline__ void idx_reposition_block(const AdjView &view, const PosIndex &ix, uint32_t u,
                                                     uint64_t off, uint32_t len, Status *st) {
    idx_reposition_pass(view, ix, u, off, len, threadIdx.x, blockDim.x, false, st);
    __syncthreads();
    idx_reposition_pass(view, ix, u, off, len, threadIdx.x, blockDim.x, true, st);
    __syncthreads();
}

__device__ __forceinline__ void idx_reposition_warp(const AdjView &view, const PosIndex &ix, uint32_t u,
                                                    uint64_t off, uint32_t len, Status *st) {
    const uint32_t lane = lane_id();
    __syncwarp();
    idx_reposition_pass(view, ix, u, off, len, lane, 32u, false, st);
    __syncwarp();
    idx_reposition_pass(view, ix, u, off, len, lane, 32u, true, st);
    __syncwarp();
}

// ---------------------------------------------------------------- compaction

// Drop the tombstones of the queued rows in place (order kept).  One block
// per row; tiles of kTpbMut x 8 slots, block scan, survivors staged in
// shared memory and stored with coalesced writes.
__global__ void __launch_bounds__(kTpbMut) compact_rows(AdjView view, RowDesc *desc, const uint32_t *list,
                                                         const uint32_t *count, PosIndex ix, Status *st) {
    using BlockScan = cub::BlockScan<uint32_t, kTpbMut>;
    __shared__ typename BlockScan::TempStorage scan_tmp;
    __shared__ uint32_t stage[kTpbMut * kBigItems];
    const uint32_t tid = threadIdx.x;
    const uint32_t nc = *count;
    for (uint32_t c = blockIdx.x; c < nc; c += gridDim.x) {
        const uint32_t u = list[c];
        const RowDesc d = desc[u];
        uint32_t w = 0;
        for (uint32_t base = 0; base < d.len; base += kTpbMut * kBigItems) {
            const uint32_t k0 = base + tid * kBigItems;
            uint32_t e[kBigItems];
#pragma unroll
            for (int h = 0; h < kBigItems; h += 4) {
                if (k0 + h < d.len) {
                    const uint4 q = *reinterpret_cast<const uint4 *>(view.at(d.off + k0 + h));
                    e[h] = q.x;
                    e[h + 1] = q.y;
                    e[h + 2] = q.z;
                    e[h + 3] = q.w;
                } else {
                    e[h] = e[h + 1] = e[h + 2] = e[h + 3] = kTomb;
                }
            }
            uint32_t kc = 0;
#pragma unroll
            for (int s = 0; s < kBigItems; ++s) kc += (k0 + s < d.len && e[s] != kTomb) ? 1u : 0u;
            uint32_t prefix, total;
            BlockScan(scan_tmp).ExclusiveSum(kc, prefix, total);
            uint32_t pos = prefix;
#pragma unroll
            for (int s = 0; s < kBigItems; ++s)
                if (k0 + s < d.len && e[s] != kTomb) stage[pos++] = e[s];
            __syncthreads();  // every load of this tile is done before any store
            const uint32_t tile_valid = min(static_cast<uint32_t>(kTpbMut * kBigItems), d.len - base);
            if (w != base || total != tile_valid)
                for (uint32_t i = tid; i < total; i += kTpbMut) write_slot(view, d.off + w + i, stage[i]);
            w += total;
            __syncthreads();
        }
        if (tid == 0) desc[u] = RowDesc{d.off, w, rd_meta(rd_cls(d), 0)};
        __syncthreads();
        if (idx_row(ix, u)) idx_reposition_block(view, ix, u, d.off, w, st);
    }
}

// ---------------------------------------------------------------- addition

// Addition plan: rows that outgrow their block get a class (sized for the
// live entries plus the additions, since relocation drops tombstones) and a
// rank in that class.
__global__ void plan_add(const RowDesc *desc, const unsigned long long *keys, Groups gr, unsigned long long *plan,
                         ArenaAlloc *al) {
    const uint32_t ng = *gr.count;
    const uint32_t rounded = (ng + 31u) & ~31u;
    const uint32_t lane = lane_id();
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < rounded; g += gridDim.x * blockDim.x) {
        unsigned long long p = kKeyNone;
        bool move = false;
        uint32_t cls = 0;
        if (g < ng) {
            const uint32_t gs = gr.start[g];
            const uint32_t ge = gr.end[g];
            const RowDesc d = desc[key_src(keys[gs])];
            const unsigned long long used = static_cast<unsigned long long>(d.len) + (ge - gs);
            const unsigned long long live = static_cast<unsigned long long>(rd_live(d)) + (ge - gs);
            if (live > 0xFFFFFFFFull) {
                p = kKeyNone - 1;  // degree overflow, reported by the apply kernel
            } else if (rd_cls(d) == 0 || used > (1ull << rd_cls(d))) {
                cls = class_for(static_cast<uint32_t>(live));
                move = true;
            }
        }
        // Ranks within a class, one atomic per class present in the warp
        // (tens of thousands of moving rows share a handful of classes).
        const uint32_t movers = __ballot_sync(kFull, move);
        if (move) {
            const uint32_t peers = __match_any_sync(movers, cls);
            const uint32_t leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&al->demand[cls], static_cast<uint32_t>(__popc(peers)));
            base = __shfl_sync(peers, base, leader);
            p = (static_cast<unsigned long long>(cls) << 32) | (base + __popc(peers & lanemask_lt()));
        }
        if (g < ng) plan[g] = p;
    }
}

// Serve this batch's demand per class (one thread per class).
__global__ void alloc_classes(ArenaAlloc *al, Status *st) {
    const uint32_t c = threadIdx.x;
    if (c >= kNumClasses) return;
    const uint32_t need = al->demand[c];
    al->demand[c] = 0;
    al->avail[c] = 0;
    if (need == 0) return;
    if (c <= kSegShift) {
        const unsigned long long cur = al->cur_next[c], end = al->cur_end[c];
        const unsigned long long room = (end - cur) >> c;
        al->base_cur[c] = cur;
        if (need <= room) {
            al->avail[c] = need;
            al->cur_next[c] = cur + (static_cast<unsigned long long>(need) << c);
            return;
        }
        al->avail[c] = static_cast<uint32_t>(room);
        const unsigned long long rest = need - room;
        const unsigned long long per_seg = 1ull << (kSegShift - c);
        const unsigned long long nseg = (rest + per_seg - 1) / per_seg;
        const unsigned long long s0 = atomicAdd(&al->seg_bump, nseg);
        if (s0 + nseg > al->seg_total) {
            set_error(st, kErrArena, c);
            return;
        }
        al->base_new[c] = s0 << kSegShift;
        al->cur_next[c] = al->base_new[c] + (rest << c);
        al->cur_end[c] = (s0 + nseg) << kSegShift;
    } else {
        const unsigned long long nseg = static_cast<unsigned long long>(need) << (c - kSegShift);
        const unsigned long long s0 = atomicAdd(&al->seg_bump, nseg);
        if (s0 + nseg > al->seg_total) {
            set_error(st, kErrArena, c);
            return;
        }
        al->base_new[c] = s0 << kSegShift;
    }
}

// Addition phase.  mutate_add gives each lane a group of its own when the
// lane can serve it alone (at most kLaneAdds appends, and a moving row of at
// most kLaneRow slots, read into registers with independent loads: rows in
// host memory cost one round trip, not one per entry), so the common
// one-request groups run 32 to a warp.  The other groups are appended to a
// list that mutate_add_warp serves one warp per group over the whole grid
// (rows above kWarpRowMax that must move go on to the block path,
// mutate_add_big).  Serving them inside the warp that found them left the
// busiest warps a serial queue of up to 32 row copies while most of the grid
// had no group at all.  `vals` is add_v for the forward arena and add_u for
// the reverse arena.  A moving row is copied without its tombstones.
constexpr uint32_t kLaneAdds = 8;
constexpr uint32_t kLaneRow = 8;

__global__ void __launch_bounds__(256, 4)
    mutate_add(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr,
                           const unsigned long long *plan, const ArenaAlloc *al, const uint32_t *vals,
                           uint32_t *coop_list, uint32_t *coop_count, unsigned long long *stats, PosIndex ix,
                           Status *st) {
    if (ld_volatile(&st->err) & kErrArena) return;
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t ng = *gr.count;
    uint32_t changed = 0, moved = 0, moved_entries = 0;  // per lane
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < ng; base += warps * 32u) {
        const uint32_t g = base + lane;
        bool coop = false;
        if (g < ng) {
            const unsigned long long p = plan[g];
            const uint32_t gs = gr.start[g];
            const uint32_t a = gr.end[g] - gs;
            if (p == kKeyNone - 1) {
                set_error(st, kErrInternal, g);
            } else if (a > kLaneAdds) {
                coop = true;
            } else {
                const uint32_t u = key_src(keys[gs]);
                const RowDesc d = desc[u];
                const bool indexed = idx_row(ix, u);
                // The appended values first, with independent loads (the
                // stores below could alias them as far as the compiler knows).
                uint32_t add[kLaneAdds];
#pragma unroll
                for (uint32_t j = 0; j < kLaneAdds; ++j) add[j] = j < a ? vals[key_low(keys[gs + j])] : 0u;
                if (p == kKeyNone) {
                    // A block of at most one segment: one slot lookup for the
                    // row's end, then plain stores.
                    if (rd_cls(d) <= kSegShift) {
                        uint32_t *wp = view.wptr(d.off + d.len);
#pragma unroll
                        for (uint32_t j = 0; j < kLaneAdds; ++j)
                            if (j < a) wp[j] = add[j];
                    } else {
                        for (uint32_t j = 0; j < a; ++j) write_slot(view, d.off + d.len + j, add[j]);
                    }
                    if (indexed) idx_add_n<kLaneAdds>(ix, u, add, d.len, a, st);
                    desc[u] = RowDesc{d.off, d.len + a, d.meta};
                    changed += 1;
                } else if (d.len > kLaneRow) {
                    coop = true;
                } else {
                    const uint32_t cls = static_cast<uint32_t>(p >> 32);
                    const unsigned long long off = alloc_offset(al, cls, static_cast<uint32_t>(p));
                    // Old block (<= kLaneRow slots) and new block (<= 16 slots)
                    // each lie in one segment: one slot lookup apiece.
                    uint32_t row[kLaneRow];
                    const uint32_t *src = d.len ? view.at(d.off) : nullptr;
#pragma unroll
                    for (uint32_t k = 0; k < kLaneRow; ++k) row[k] = k < d.len ? src[k] : kTomb;
                    uint32_t *wp = view.wptr(off);
                    uint32_t w = 0;
#pragma unroll
                    for (uint32_t k = 0; k < kLaneRow; ++k)
                        if (row[k] != kTomb) wp[w++] = row[k];
#pragma unroll
                    for (uint32_t j = 0; j < kLaneAdds; ++j)
                        if (j < a) wp[w + j] = add[j];
                    desc[u] = RowDesc{off, w + a, rd_meta(cls, 0)};
                    moved_entries += w;
                    if (indexed) {
                        for (uint32_t k = 0; k < w; ++k) idx_pos_reset(ix, u, __ldcg(wp + k), st);
                        for (uint32_t k = 0; k < w; ++k) idx_pos_set(ix, u, __ldcg(wp + k), k);
                        for (uint32_t j = 0; j < a; ++j) idx_add(ix, u, add[j], w + j, st);
                    }
                    moved += 1;
                    changed += 1;
                }
            }
        }
        // Groups a lane cannot serve alone go to the warp-per-group kernel,
        // which spreads them over every warp of the grid.
        warp_enqueue(coop, g, coop_list, coop_count, ng, st);
    }
    if (stats) {
        warp_count(&stats[kCntChanged], changed);
        warp_count(&stats[kCntRelocated], moved);
        warp_count(&stats[kCntMovedEntries], moved_entries);
    }
}


// The groups mutate_add left to whole warps (more than kLaneAdds appends, or
// a moving row of more than kLaneRow entries), one warp per group over the
// whole grid: rows of up to kWarpRowMax entries move here, larger ones go to
// mutate_add_big.
__global__ void mutate_add_warp(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr,
                                const unsigned long long *plan, const ArenaAlloc *al, const uint32_t *vals,
                                const uint32_t *coop_list, const uint32_t *coop_count, uint32_t *big,
                                uint32_t *big_count, unsigned long long *stats, PosIndex ix, Status *st) {
    if (ld_volatile(&st->err) & kErrArena) return;
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nc = *coop_count;
    uint32_t changed = 0, moved = 0, moved_entries = 0;  // lane 0 counts
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += warps) {
        const uint32_t gb = coop_list[i];
        const unsigned long long p = plan[gb];
        const uint32_t gs = gr.start[gb];
        const uint32_t ge = gr.end[gb];
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const uint32_t a = ge - gs;
        if (p == kKeyNone) {
            const bool indexed = idx_row(ix, u);
            for (uint32_t j = lane; j < a; j += 32u) {
                const uint32_t v = vals[key_low(keys[gs + j])];
                write_slot(view, d.off + d.len + j, v);
                if (indexed) idx_add(ix, u, v, d.len + j, st);
            }
            if (lane == 0) desc[u] = RowDesc{d.off, d.len + a, d.meta};
        } else {
            if (d.len > kWarpRowMax) {
                if (lane == 0) big[atomicAdd(big_count, 1u)] = gb;
                continue;
            }
            const uint32_t cls = static_cast<uint32_t>(p >> 32);
            const unsigned long long off = alloc_offset(al, cls, static_cast<uint32_t>(p));
            // Copy the survivors in order, 256 entries per step: each lane
            // issues two independent 16-byte loads (the old block lies in
            // one segment and starts on a 16-byte boundary) before any
            // store, so a zero-copy row costs one host round trip per
            // 256 entries instead of one per 32.
            const uint32_t *src = view.at(d.off);
            uint32_t w = 0;
            for (uint32_t b0 = 0; b0 < d.len; b0 += 256u) {
                uint32_t e[8];
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    const uint32_t k = b0 + 128u * h + 4u * lane;
                    uint4 q = make_uint4(kTomb, kTomb, kTomb, kTomb);
                    if (k < d.len) q = *reinterpret_cast<const uint4 *>(src + k);
                    e[4 * h] = k < d.len ? q.x : kTomb;
                    e[4 * h + 1] = k + 1u < d.len ? q.y : kTomb;
                    e[4 * h + 2] = k + 2u < d.len ? q.z : kTomb;
                    e[4 * h + 3] = k + 3u < d.len ? q.w : kTomb;
                }
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    uint32_t c = 0;
#pragma unroll
                    for (uint32_t j = 0; j < 4; ++j) c += e[4 * h + j] != kTomb ? 1u : 0u;
                    uint32_t incl = c;
#pragma unroll
                    for (uint32_t o = 1; o < 32u; o <<= 1) {
                        const uint32_t t = __shfl_up_sync(kFull, incl, o);
                        if (lane >= o) incl += t;
                    }
                    uint32_t pos = w + incl - c;
#pragma unroll
                    for (uint32_t j = 0; j < 4; ++j)
                        if (e[4 * h + j] != kTomb) write_slot(view, off + pos++, e[4 * h + j]);
                    w += __shfl_sync(kFull, incl, 31);
                }
            }
            if (lane == 0) moved_entries += w;
            for (uint32_t j = lane; j < a; j += 32u) write_slot(view, off + w + j, vals[key_low(keys[gs + j])]);
            if (lane == 0) desc[u] = RowDesc{off, w + a, rd_meta(cls, 0)};
            if (idx_row(ix, u)) {
                // survivors moved: reposition them; then count the appended entries
                idx_reposition_warp(view, ix, u, off, w, st);
                for (uint32_t j = lane; j < a; j += 32u) idx_add(ix, u, vals[key_low(keys[gs + j])], w + j, st);
            }
            if (lane == 0) moved += 1;
        }
        if (lane == 0) changed += 1;
    }
    if (stats) {
        warp_count(&stats[kCntChanged], changed);
        warp_count(&stats[kCntRelocated], moved);
        warp_count(&stats[kCntMovedEntries], moved_entries);
    }
}

__global__ void __launch_bounds__(kTpbMut)
    mutate_add_big(AdjView view, RowDesc *desc, const unsigned long long *keys, Groups gr,
                   const unsigned long long *plan, const ArenaAlloc *al, const uint32_t *vals, const uint32_t *big,
                   const uint32_t *big_count, unsigned long long *stats, PosIndex ix, Status *st) {
    using BlockScan = cub::BlockScan<uint32_t, kTpbMut>;
    __shared__ typename BlockScan::TempStorage scan_tmp;
    if (ld_volatile(&st->err) & kErrArena) return;
    const uint32_t nb = *big_count;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t g = big[b];
        const unsigned long long p = plan[g];
        const uint32_t gs = gr.start[g];
        const uint32_t ge = gr.end[g];
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const uint32_t a = ge - gs;
        const uint32_t cls = static_cast<uint32_t>(p >> 32);
        const unsigned long long off = alloc_offset(al, cls, static_cast<uint32_t>(p));
        uint32_t w = 0;
        for (uint32_t base = 0; base < d.len; base += kTpbMut) {
            const uint32_t k = base + threadIdx.x;
            const uint32_t x = k < d.len ? *view.at(d.off + k) : kTomb;
            uint32_t prefix, total;
            BlockScan(scan_tmp).ExclusiveSum(x != kTomb ? 1u : 0u, prefix, total);
            if (x != kTomb) write_slot(view, off + w + prefix, x);
            w += total;
            __syncthreads();
        }
        for (uint32_t j = threadIdx.x; j < a; j += kTpbMut) write_slot(view, off + w + j, vals[key_low(keys[gs + j])]);
        __syncthreads();
        if (idx_row(ix, u)) {
            idx_reposition_block(view, ix, u, off, w, st);
            for (uint32_t j = threadIdx.x; j < a; j += kTpbMut) idx_add(ix, u, vals[key_low(keys[gs + j])], w + j, st);
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            desc[u] = RowDesc{off, w + a, rd_meta(cls, 0)};
            if (stats) {
                atomicAdd(&stats[kCntChanged], 1ull);
                atomicAdd(&stats[kCntRelocated], 1ull);
                atomicAdd(&stats[kCntMovedEntries], static_cast<unsigned long long>(w));
            }
        }
    }
}

}  // namespace cig
