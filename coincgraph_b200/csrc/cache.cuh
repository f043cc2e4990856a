// cache.cuh - device-side segment table of the HBM edge cache.
//
// The forward arena is cut into 64 KiB segments; `seg_slot` maps each to a
// slot of the HBM cache pool or to -1 (served zero-copy from pinned host
// memory).  This table is owned and changed by the GPU alone, once per batch
// (after the insertion phase), so a batch never waits on the host for a
// residency decision:
//   - hotness: every row read or rewritten adds its length to `hot` of its
//     segment; the service folds it into a decayed `score` (score/2 + hot);
//   - new segments handed out by the block allocator take a free slot at
//     once (their rows were just written, so they are hot), and the service
//     keeps `reserve` slots free for them by evicting the coldest resident
//     segments (a histogram of log2(score) picks the threshold);
//   - host segments whose score passed admit_score are copied in, at most
//     kMaxAdmit per batch, into slots freed from cold segments;
//   - an evicted segment is written back first if it is dirty.
// The reference keeps per-vertex hotness in a 4-batch uint8 window, sorts
// vertices by it and re-packs the cached rows when the admitted set changes
// (include/framework/variants/driver.cuh:53-247, 691-770; framework.cuh:
// 599-798); residency here is per segment, so admission is a slot copy and
// the arena layout never changes.
#pragma once

#include "common.cuh"

namespace cig {

constexpr uint32_t kAdmitScore = 8192;   // default: ~half a segment of entries read recently
constexpr uint32_t kColdScore = 1u << 30;  // default cap: segments scoring this much are never evicted
constexpr int kScoreBuckets = 33;          // bucket of a score: 32 - clz(score)
constexpr uint32_t kMaxAdmit = 64;       // admissions per batch (4 MiB over the host link)
constexpr uint32_t kMaxEvict = 1024;     // evictions per batch
constexpr uint32_t kNewScore = 16384;    // score of a freshly allocated segment

enum SegCtl : int {
    kCtlFreeTop = 0,    // entries on the free-slot stack
    kCtlBumpSeen = 1,   // allocator bump pointer when slots were last handed out
    kCtlNewLast = 2,    // segments created since the last service
    kCtlVictims = 3,    // cold resident segments found this service
    kCtlAdmits = 4,     // hot host segments found this service
    kCtlEvictNeed = 5,  // evictions this service
    kCtlReserve = 6,    // free slots kept for new segments
    kCtlThreshold = 7,  // victims: bucket below this ...
    kCtlExtra = 8,      // ... plus this many from the threshold bucket
    kCtlExtraTaken = 9,
    kCtlHist = 16,      // kScoreBuckets counters of resident scores
    kCtlCount = 16 + kScoreBuckets
};

struct SegTable {
    int32_t *seg_slot;    // per segment: slot or -1
    int32_t *slot_seg;    // per slot: owning segment or -1
    uint8_t *seg_dirty;   // per segment: HBM copy newer than the host copy
    uint32_t *score;      // per segment
    uint32_t *hot;        // per segment, since the last service
    uint32_t *free_slots; // stack
    uint32_t *victims;    // this service's evictions (slots)
    uint32_t *admits;     // this service's admissions (segments)
    uint32_t *ctl;        // SegCtl
    uint32_t nslots;
    uint32_t nsegs;
    uint32_t admit_score;  // host segments at or above are admitted
    uint32_t cold_score;   // resident segments below may be evicted
};

__device__ __forceinline__ void seg_touch(uint32_t *hot, uint64_t off, uint32_t len) {
    if (hot && len) atomicAdd(hot + (off >> kSegShift), len);
}

// Slots for the segments the allocator created since the last call.
// One thread; a handful of segments per batch.
__global__ void seg_assign_new(SegTable t, const unsigned long long *seg_bump, Status *st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t bump = static_cast<uint32_t>(min(*seg_bump, static_cast<unsigned long long>(t.nsegs)));
    const uint32_t seen = t.ctl[kCtlBumpSeen];
    uint32_t top = t.ctl[kCtlFreeTop];
    for (uint32_t s = seen; s < bump; ++s) {
        t.score[s] = kNewScore;
        if (t.seg_slot[s] >= 0 || top == 0) continue;
        const uint32_t slot = t.free_slots[--top];
        t.seg_slot[s] = static_cast<int32_t>(slot);
        t.slot_seg[slot] = static_cast<int32_t>(s);
        t.seg_dirty[s] = 0;
        atomicAdd(&st->counters[kCntSegLoaded], 1ull);
    }
    t.ctl[kCtlFreeTop] = top;
    t.ctl[kCtlNewLast] += bump > seen ? bump - seen : 0u;
    t.ctl[kCtlBumpSeen] = max(seen, bump);
}

__device__ __forceinline__ uint32_t score_bucket(uint32_t sc) { return 32u - __clz(sc); }

// Decay scores, histogram the resident ones (evictable: below cold_score)
// and list admission candidates among hot host segments.  Grid-stride.
__global__ void seg_rescore(SegTable t, uint32_t bump) {
    __shared__ uint32_t hist[kScoreBuckets];
    for (uint32_t b = threadIdx.x; b < kScoreBuckets; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < bump; s += gridDim.x * blockDim.x) {
        const uint32_t h = t.hot[s];
        if (h) t.hot[s] = 0;
        const uint32_t sc = (t.score[s] >> 1) + min(h, 1u << 24);
        t.score[s] = sc;
        if (t.seg_slot[s] >= 0) {
            if (sc < t.cold_score) atomicAdd(hist + score_bucket(sc), 1u);
        } else if (sc >= t.admit_score) {
            const uint32_t i = atomicAdd(t.ctl + kCtlAdmits, 1u);
            if (i < kMaxAdmit) t.admits[i] = s;
        }
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < kScoreBuckets; b += blockDim.x)
        if (hist[b]) atomicAdd(t.ctl + kCtlHist + b, hist[b]);
}

// How many to evict: enough to keep `reserve` slots free for new segments
// (twice the last batches' count, 16..1024) plus the admissions; the
// coldest first: whole buckets below a threshold, then part of it.
__global__ void seg_plan(SegTable t) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t reserve = min(1024u, max(16u, 2u * t.ctl[kCtlNewLast]));
    t.ctl[kCtlNewLast] = 0;
    t.ctl[kCtlReserve] = reserve;
    const uint32_t want = reserve + min(t.ctl[kCtlAdmits], kMaxAdmit);
    const uint32_t top = t.ctl[kCtlFreeTop];
    uint32_t need = min(want > top ? want - top : 0u, kMaxEvict);
    uint32_t below = 0, b = 0;
    for (; b < static_cast<uint32_t>(kScoreBuckets); ++b) {
        const uint32_t c = t.ctl[kCtlHist + b];
        if (below + c >= need) break;
        below += c;
    }
    if (b == static_cast<uint32_t>(kScoreBuckets)) need = below;  // fewer evictable segments than wanted
    t.ctl[kCtlThreshold] = b;
    t.ctl[kCtlExtra] = need - below;
    t.ctl[kCtlExtraTaken] = 0;
    t.ctl[kCtlEvictNeed] = need;
}

// The victims chosen by seg_plan.  Grid-stride over segments.
__global__ void seg_pick(SegTable t, uint32_t bump) {
    const uint32_t thr = t.ctl[kCtlThreshold], extra = t.ctl[kCtlExtra], need = t.ctl[kCtlEvictNeed];
    if (!need) return;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < bump; s += gridDim.x * blockDim.x) {
        const int32_t slot = t.seg_slot[s];
        if (slot < 0) continue;
        const uint32_t sc = t.score[s];
        if (sc >= t.cold_score) continue;
        const uint32_t b = score_bucket(sc);
        bool take = b < thr;
        if (!take && b == thr && extra) take = atomicAdd(t.ctl + kCtlExtraTaken, 1u) < extra;
        if (take) {
            const uint32_t i = atomicAdd(t.ctl + kCtlVictims, 1u);
            if (i < need) t.victims[i] = static_cast<uint32_t>(slot);
        }
    }
}

// One block copies one 64 KiB segment: each thread has eight 16-byte loads
// in flight before it stores them, so a copy from host memory (about 2 us
// away) takes two round trips instead of sixteen.
__device__ __forceinline__ void copy_segment(uint4 *dst, const uint4 *src) {
    constexpr uint32_t kVec = kSegEdges / 4, kDepth = 8;
    for (uint32_t i0 = 0; i0 < kVec; i0 += kDepth * blockDim.x) {
        uint4 r[kDepth];
#pragma unroll
        for (uint32_t j = 0; j < kDepth; ++j) {
            const uint32_t i = i0 + j * blockDim.x + threadIdx.x;
            r[j] = i < kVec ? src[i] : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (uint32_t j = 0; j < kDepth; ++j) {
            const uint32_t i = i0 + j * blockDim.x + threadIdx.x;
            if (i < kVec) dst[i] = r[j];
        }
    }
}

// One block per victim slot: write back if dirty, unmap, free the slot.
__global__ void seg_evict(SegTable t, const uint32_t *cache, uint32_t *host, Status *st) {
    const uint32_t nv = min(t.ctl[kCtlEvictNeed], t.ctl[kCtlVictims]);
    for (uint32_t v = blockIdx.x; v < nv; v += gridDim.x) {
        const uint32_t slot = t.victims[v];
        const int32_t seg = t.slot_seg[slot];
        if (seg < 0) continue;
        if (t.seg_dirty[seg])
            copy_segment(reinterpret_cast<uint4 *>(host + (static_cast<uint64_t>(seg) << kSegShift)),
                         reinterpret_cast<const uint4 *>(cache + (static_cast<uint64_t>(slot) << kSegShift)));
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence_system();
            t.seg_dirty[seg] = 0;
            t.seg_slot[seg] = -1;
            t.slot_seg[slot] = -1;
            const uint32_t pos = atomicAdd(t.ctl + kCtlFreeTop, 1u);
            if (pos < t.nslots)
                t.free_slots[pos] = slot;
            else
                set_error(st, kErrInternal, pos);
            atomicAdd(&st->counters[kCntSegEvicted], 1ull);
        }
        __syncthreads();
    }
}

// One block per admission candidate while free slots above the reserve
// last: copy the host segment into a slot and map it.
__global__ void seg_admit(SegTable t, uint32_t *cache, const uint32_t *host, Status *st) {
    __shared__ int32_t slot_s;
    const uint32_t na = min(t.ctl[kCtlAdmits], kMaxAdmit);
    const uint32_t reserve = t.ctl[kCtlReserve];
    for (uint32_t a = blockIdx.x; a < na; a += gridDim.x) {
        const uint32_t seg = t.admits[a];
        if (threadIdx.x == 0 && t.seg_slot[seg] < 0) {
            slot_s = -1;
            // Take a slot only while more than `reserve` remain.
            uint32_t top = ld_volatile(t.ctl + kCtlFreeTop);
            while (top > reserve) {
                const uint32_t prev = atomicCAS(t.ctl + kCtlFreeTop, top, top - 1);
                if (prev == top) {
                    slot_s = static_cast<int32_t>(t.free_slots[top - 1]);
                    break;
                }
                top = prev;
            }
        }
        if (threadIdx.x == 0 && t.seg_slot[seg] >= 0) slot_s = -1;
        __syncthreads();
        const int32_t slot = slot_s;
        if (slot >= 0) {
            copy_segment(reinterpret_cast<uint4 *>(cache + (static_cast<uint64_t>(slot) << kSegShift)),
                         reinterpret_cast<const uint4 *>(host + (static_cast<uint64_t>(seg) << kSegShift)));
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                t.seg_dirty[seg] = 0;
                t.slot_seg[slot] = static_cast<int32_t>(seg);
                t.seg_slot[seg] = slot;
                atomicAdd(&st->counters[kCntSegLoaded], 1ull);
            }
        }
        __syncthreads();
    }
}

}  // namespace cig
