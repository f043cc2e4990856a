// mutate.cuh - GPU batch maintenance of an adjacency arena.
//
// Semantics follow the reference's source-local chunk store exactly
// (include/groute/graphs/source_local_chunk_store.h:219-391, 670-848) so that
// rows stay identical, element for element:
//   deletion phase: for every source, a destination requested k times loses
//     its first min(k, present) occurrences; survivors keep their order
//     (BuildDeletionPlan / ShouldDelete / CompactSourceInPlace);
//   addition phase: destinations are appended in input order; a row that
//     outgrows its power-of-two block moves to a block of the next class
//     (RewriteSourceToNewBlock).
// The batch is grouped by source with a device radix sort of 64-bit keys
// (source << 32 | destination) for deletions and (source << 32 | input index)
// for additions; the latter keeps input order inside a source, as the
// reference's stable radix sort does (effective_update_batch.h:48-73).
//
// Design differences: the grouping, deletion matching, compaction,
// allocation and appends all run on the GPU; the forward arena is written
// through to both the pinned host copy and the HBM cache copy of the segment.
#pragma once

#include <cub/block/block_scan.cuh>

#include "common.cuh"

namespace cig {

constexpr uint32_t kKeyShift = 32;
constexpr unsigned long long kKeyNone = ~0ull;
constexpr uint32_t kWarpRowMax = 4096;  // larger rows use the block path

__device__ __forceinline__ uint32_t key_src(unsigned long long k) { return static_cast<uint32_t>(k >> kKeyShift); }
__device__ __forceinline__ uint32_t key_low(unsigned long long k) { return static_cast<uint32_t>(k); }

// Device-side block allocator: per class a partially used segment
// [cur_next, cur_end) and a global bump pointer over whole segments.
// Retired blocks are not reused (see ArenaAlloc users).
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

// Group heads of a sorted key array (one group per source).
__global__ void find_groups(const unsigned long long *keys, uint32_t m, uint32_t *groups, uint32_t *gcount) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool head = false;
    if (i < m) {
        const unsigned long long k = keys[i];
        head = k != kKeyNone && (i == 0 || key_src(keys[i - 1]) != key_src(k));
    }
    if (__any_sync(kFull, i < m)) {
        const uint32_t mask = __ballot_sync(kFull, head);
        if (mask) {
            const uint32_t leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (lane_id() == leader) base = atomicAdd(gcount, __popc(mask));
            base = __shfl_sync(kFull, base, leader);
            if (head) groups[base + __popc(mask & lanemask_lt())] = i;
        }
    }
}

// End of the group starting at `start`: first index whose source differs.
__device__ __forceinline__ uint32_t group_end(const unsigned long long *keys, uint32_t m, uint32_t start) {
    const uint32_t src = key_src(keys[start]);
    uint32_t lo = start + 1, hi = m;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const unsigned long long k = keys[mid];
        if (k != kKeyNone && key_src(k) == src)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Deletion run of destination x inside the group [gs, ge): returns the index
// of the run's first key (a unique run id) and its requested count.
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
    uint32_t *p, *mirror;
    view.targets(off, p, mirror);
    *p = value;
    if (mirror) *mirror = value;
}

// Deletion phase, one warp per source group; rows above kWarpRowMax go to
// the block path.  `matched[run]` counts occurrences of a run already seen.
__global__ void mutate_delete(AdjView view, RowDesc *desc, const unsigned long long *keys, uint32_t m,
                              const uint32_t *groups, const uint32_t *gcount, uint32_t *matched, uint32_t *big,
                              uint32_t *big_count, unsigned long long *stats, Status *st) {
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t ng = *gcount;
    unsigned long long removed = 0, changed = 0;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ng; g += warps) {
        const uint32_t gs = groups[g];
        const uint32_t ge = group_end(keys, m, gs);
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        if (d.deg > kWarpRowMax) {
            if (lane == 0) big[atomicAdd(big_count, 1u)] = gs;
            continue;
        }
        const unsigned long long uhi = static_cast<unsigned long long>(u) << kKeyShift;
        uint32_t w = 0;
        for (uint32_t base = 0; base < d.deg; base += 32u) {
            const uint32_t k = base + lane;
            const bool valid = k < d.deg;
            const uint32_t x = valid ? *view.at(d.off + k) : 0u;
            uint32_t run = 0xFFFFFFFFu, req = 0;
            const bool cand = valid && find_run(keys, gs, ge, uhi | x, run, req);
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
            const bool keep = valid && !del;
            const uint32_t km = __ballot_sync(kFull, keep);
            const uint32_t pos = w + __popc(km & lanemask_lt());
            __syncwarp();
            if (keep && pos != k) write_slot(view, d.off + pos, x);
            w += __popc(km);
        }
        if (lane == 0) {
            desc[u].deg = w;
            removed += d.deg - w;
            changed += (w != d.deg);
        }
    }
    if (lane == 0 && stats) {
        if (removed) atomicAdd(&stats[kCntRemoved], removed);
        if (changed) atomicAdd(&stats[kCntChanged], changed);
    }
}

// Deletion phase for rows above kWarpRowMax: one block per row, tiles of
// kTpbMut entries, candidates resolved in position order by one thread,
// block scan for the in-place compaction.
constexpr int kTpbMut = 256;

__global__ void __launch_bounds__(kTpbMut) mutate_delete_big(AdjView view, RowDesc *desc,
                                                              const unsigned long long *keys, uint32_t m,
                                                              const uint32_t *big, const uint32_t *big_count,
                                                              uint32_t *matched, unsigned long long *stats,
                                                              Status *st) {
    using BlockScan = cub::BlockScan<uint32_t, kTpbMut>;
    __shared__ typename BlockScan::TempStorage scan_tmp;
    __shared__ uint32_t cand_bits[kTpbMut / 32];
    __shared__ uint32_t del_bits[kTpbMut / 32];
    __shared__ uint32_t cand_run[kTpbMut];
    __shared__ uint32_t cand_req[kTpbMut];
    const uint32_t tid = threadIdx.x;
    const uint32_t nb = *big_count;
    for (uint32_t g = blockIdx.x; g < nb; g += gridDim.x) {
        const uint32_t gs = big[g];
        const uint32_t ge = group_end(keys, m, gs);
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const unsigned long long uhi = static_cast<unsigned long long>(u) << kKeyShift;
        uint32_t w = 0;
        for (uint32_t base = 0; base < d.deg; base += kTpbMut) {
            const uint32_t k = base + tid;
            const bool valid = k < d.deg;
            const uint32_t x = valid ? *view.at(d.off + k) : 0u;
            uint32_t run = 0, req = 0;
            const bool cand = valid && find_run(keys, gs, ge, uhi | x, run, req);
            cand_run[tid] = run;
            cand_req[tid] = req;
            const uint32_t bits = __ballot_sync(kFull, cand);
            if ((tid & 31u) == 0) {
                cand_bits[tid >> 5] = bits;
                del_bits[tid >> 5] = 0;
            }
            __syncthreads();
            if (tid == 0) {
                for (uint32_t wi = 0; wi < kTpbMut / 32; ++wi) {
                    uint32_t b = cand_bits[wi];
                    while (b) {
                        const uint32_t bit = __ffs(b) - 1;
                        b &= b - 1;
                        const uint32_t p = wi * 32 + bit;
                        const uint32_t r = cand_run[p];
                        const uint32_t seen = matched[r];
                        if (seen < cand_req[p]) del_bits[wi] |= 1u << bit;
                        matched[r] = seen + 1;
                    }
                }
            }
            __syncthreads();
            const bool del = (del_bits[tid >> 5] >> (tid & 31u)) & 1u;
            const uint32_t keep = (valid && !del) ? 1u : 0u;
            uint32_t prefix, total;
            BlockScan(scan_tmp).ExclusiveSum(keep, prefix, total);
            __syncthreads();
            if (keep && w + prefix != k) write_slot(view, d.off + w + prefix, x);
            w += total;
            __syncthreads();
        }
        if (tid == 0) {
            desc[u].deg = w;
            if (d.deg != w && stats) {
                atomicAdd(&stats[kCntRemoved], static_cast<unsigned long long>(d.deg - w));
                atomicAdd(&stats[kCntChanged], 1ull);
            }
        }
        __syncthreads();
    }
}

// Addition plan: rows that outgrow their block get a class and a rank.
__global__ void plan_add(const RowDesc *desc, const unsigned long long *keys, uint32_t m, const uint32_t *groups,
                         const uint32_t *gcount, unsigned long long *plan, ArenaAlloc *al) {
    const uint32_t ng = *gcount;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        const uint32_t gs = groups[g];
        const uint32_t ge = group_end(keys, m, gs);
        const RowDesc d = desc[key_src(keys[gs])];
        const unsigned long long nd = static_cast<unsigned long long>(d.deg) + (ge - gs);
        unsigned long long p = kKeyNone;
        if (nd > 0xFFFFFFFFull) {
            p = kKeyNone - 1;  // degree overflow, reported by the apply kernel
        } else if (d.cls == 0 || nd > (1ull << d.cls)) {
            const uint32_t cls = class_for(static_cast<uint32_t>(nd));
            const uint32_t rank = atomicAdd(&al->demand[cls], 1u);
            p = (static_cast<unsigned long long>(cls) << 32) | rank;
        }
        plan[g] = p;
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

// Addition phase, one warp per group (rows above kWarpRowMax that must move
// go to the block path).  `vals` is add_v for the forward arena and add_u
// for the reverse arena.
__global__ void mutate_add(AdjView view, RowDesc *desc, const unsigned long long *keys, uint32_t m,
                           const uint32_t *groups, const uint32_t *gcount, const unsigned long long *plan,
                           const ArenaAlloc *al, const uint32_t *vals, uint32_t *big, uint32_t *big_count,
                           unsigned long long *stats, Status *st) {
    if (ld_volatile(&st->err) & kErrArena) return;
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t ng = *gcount;
    unsigned long long changed = 0, moved = 0;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ng; g += warps) {
        const unsigned long long p = plan[g];
        if (p == kKeyNone - 1) {
            if (lane == 0) set_error(st, kErrInternal, g);
            continue;
        }
        const uint32_t gs = groups[g];
        const uint32_t ge = group_end(keys, m, gs);
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const uint32_t a = ge - gs;
        unsigned long long off = d.off;
        uint32_t cls = d.cls;
        if (p != kKeyNone) {
            if (d.deg > kWarpRowMax) {
                if (lane == 0) big[atomicAdd(big_count, 1u)] = g;
                continue;
            }
            cls = static_cast<uint32_t>(p >> 32);
            off = alloc_offset(al, cls, static_cast<uint32_t>(p));
            for (uint32_t k = lane; k < d.deg; k += 32u) write_slot(view, off + k, *view.at(d.off + k));
            moved += 1;
        }
        for (uint32_t j = lane; j < a; j += 32u) write_slot(view, off + d.deg + j, vals[key_low(keys[gs + j])]);
        if (lane == 0) desc[u] = RowDesc{off, d.deg + a, cls};
        changed += 1;
    }
    if (lane == 0 && stats) {
        if (changed) atomicAdd(&stats[kCntChanged], changed);
        if (moved) atomicAdd(&stats[kCntRelocated], moved);
    }
}

__global__ void __launch_bounds__(kTpbMut) mutate_add_big(AdjView view, RowDesc *desc,
                                                          const unsigned long long *keys, uint32_t m,
                                                          const uint32_t *groups, const unsigned long long *plan,
                                                          const ArenaAlloc *al, const uint32_t *vals,
                                                          const uint32_t *big, const uint32_t *big_count,
                                                          unsigned long long *stats, Status *st) {
    if (ld_volatile(&st->err) & kErrArena) return;
    const uint32_t nb = *big_count;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t g = big[b];
        const unsigned long long p = plan[g];
        const uint32_t gs = groups[g];
        const uint32_t ge = group_end(keys, m, gs);
        const uint32_t u = key_src(keys[gs]);
        const RowDesc d = desc[u];
        const uint32_t a = ge - gs;
        const uint32_t cls = static_cast<uint32_t>(p >> 32);
        const unsigned long long off = alloc_offset(al, cls, static_cast<uint32_t>(p));
        for (uint32_t k = threadIdx.x; k < d.deg; k += kTpbMut) write_slot(view, off + k, *view.at(d.off + k));
        for (uint32_t j = threadIdx.x; j < a; j += kTpbMut) write_slot(view, off + d.deg + j, vals[key_low(keys[gs + j])]);
        __syncthreads();
        if (threadIdx.x == 0) {
            desc[u] = RowDesc{off, d.deg + a, cls};
            if (stats) {
                atomicAdd(&stats[kCntChanged], 1ull);
                atomicAdd(&stats[kCntRelocated], 1ull);
            }
        }
    }
}

}  // namespace cig
