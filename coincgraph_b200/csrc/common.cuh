// common.cuh - shared device definitions for libcig (sm_100a).
//
// Adjacency layout.  Each vertex owns one power-of-two block of edge slots
// (at least 4), as the reference's source-local chunk store does
// (include/groute/graphs/source_local_chunk_store.h:125-145).  Blocks live in
// an "arena" addressed by a 64-bit edge offset.  The arena is cut into
// 64 KiB segments (2^14 uint32 slots); a block of 2^c slots with c <= 14 is
// aligned to its size and therefore never straddles a segment, larger blocks
// cover whole segments.  The forward arena lives in pinned, mapped host memory
// (the authoritative copy, read zero-copy) and a device segment table maps a
// segment either to a 64 KiB slot of the HBM edge cache or to "host".  The
// reverse arena (in-edges, for deletion repair) is device-only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cig {

constexpr uint32_t kSegShift = 14;
constexpr uint64_t kSegEdges = 1ull << kSegShift;
constexpr uint64_t kSegMask = kSegEdges - 1;
constexpr uint32_t kMinClass = 2;  // 4-slot minimum block (RequiredChunkCapacity)
constexpr uint32_t kNumClasses = 40;
constexpr uint32_t kInf = 0xFFFFFFFFu;
constexpr uint64_t kInf64 = ~0ull;
constexpr uint32_t kFull = 0xFFFFFFFFu;

// Device error codes (bit flags in Status::err).
enum : uint32_t {
    kErrQueue = 1u << 0,     // a work queue overflowed
    kErrArena = 1u << 1,     // arena exhausted
    kErrRounds = 1u << 2,    // round bound exceeded
    kErrBarrier = 1u << 3,   // grid barrier wait limit exceeded
    kErrNonFinite = 1u << 4, // PR produced a non-finite value
    kErrInternal = 1u << 5,
    kErrBounds = 1u << 6,    // an index out of range (bounds-check build only)
};

// A deleted entry is overwritten with kTomb (never a vertex id: ids are
// below n <= 2^32 - 1).  Survivors keep their relative order, so a row with
// its tombstones removed is exactly the row the reference keeps; tombstones
// are dropped when the row is compacted or relocated.
constexpr uint32_t kTomb = 0xFFFFFFFFu;
constexpr uint32_t kMaxTombs = (1u << 26) - 1;

struct RowDesc {
    uint64_t off;   // first slot of the block in the arena
    uint32_t len;   // used slots (live entries + tombstones)
    uint32_t meta;  // bits 0-5: class (block holds 2^cls slots, 0 = no block); bits 6-31: tombstones
};
static_assert(sizeof(RowDesc) == 16, "RowDesc must stay 16 bytes");

__host__ __device__ __forceinline__ uint32_t rd_cls(const RowDesc &d) { return d.meta & 63u; }
__host__ __device__ __forceinline__ uint32_t rd_tombs(const RowDesc &d) { return d.meta >> 6; }
__host__ __device__ __forceinline__ uint32_t rd_live(const RowDesc &d) { return d.len - (d.meta >> 6); }
__host__ __device__ __forceinline__ uint32_t rd_meta(uint32_t cls, uint32_t tombs) { return cls | (tombs << 6); }

// Device view of one arena.  For the forward arena `seg_slot` maps segments
// to cache slots (-1 = host); for a device-only arena it is null and `dev`
// holds the whole arena.  The cache is write-back: a resident segment's HBM
// copy is authoritative and `seg_dirty` marks segments whose host copy is
// stale (copied back before any host-side read or eviction).
struct Status;
__device__ __forceinline__ void report_bounds(Status *st, uint64_t index);

struct AdjView {
    const RowDesc *desc;
    uint32_t *dev;            // cache pool (forward) or arena (device-only)
    uint32_t *host;           // mapped host arena (forward) or null
    const int32_t *seg_slot;  // null for a device-only arena
    uint8_t *seg_dirty;       // null for a device-only arena
#ifdef CIG_BOUNDS_CHECK
    // Bounds-check build: arena slots and vertex ids in range (0 = not
    // checked); a violation sets kErrBounds in `bst` and the access is
    // redirected to slot 0 / dropped, so the kernel finishes and the host
    // reports the error.
    uint64_t nslots = 0;
    uint32_t nverts = 0;
    Status *bst = nullptr;
    __device__ __forceinline__ uint64_t chk(uint64_t off) const {
        if (nslots && off >= nslots) {
            report_bounds(bst, off);
            return 0;
        }
        return off;
    }
    // A row entry used as a vertex id: out of range reads as a tombstone.
    __device__ __forceinline__ uint32_t vid(uint32_t y) const {
        if (nverts && y != 0xFFFFFFFFu && y >= nverts) {
            report_bounds(bst, y);
            return 0xFFFFFFFFu;
        }
        return y;
    }
#else
    __device__ __forceinline__ uint64_t chk(uint64_t off) const { return off; }
    __device__ __forceinline__ uint32_t vid(uint32_t y) const { return y; }
#endif

    __device__ __forceinline__ uint32_t *at(uint64_t off) const {
        off = chk(off);
        if (!seg_slot) return dev + off;
        const int32_t s = __ldg(seg_slot + (off >> kSegShift));
        return s >= 0 ? dev + ((static_cast<uint64_t>(s) << kSegShift) | (off & kSegMask)) : host + off;
    }
    __device__ __forceinline__ bool cached(uint64_t off) const {
        off = chk(off);
        return !seg_slot || __ldg(seg_slot + (off >> kSegShift)) >= 0;
    }
    // The authoritative copy of slot `off` for writing; marks a resident
    // segment dirty.  Valid for the whole segment containing `off`.
    __device__ __forceinline__ uint32_t *wptr(uint64_t off) const {
        off = chk(off);
        if (!seg_slot) return dev + off;
        const uint64_t seg = off >> kSegShift;
        const int32_t s = seg_slot[seg];
        if (s < 0) return host + off;
        if (!seg_dirty[seg]) seg_dirty[seg] = 1;
        return dev + ((static_cast<uint64_t>(s) << kSegShift) | (off & kSegMask));
    }
};

struct Status {
    uint32_t err;
    uint32_t err_info;
    uint32_t barrier_count;
    uint32_t barrier_gen;
    unsigned long long counters[40];
    uint32_t cc_shift;  // CC: depth bits of a value (label << cc_shift | depth); 0 otherwise
    uint32_t cc_pad;
};

enum Counter : int {
    kCntRounds = 0,
    kCntEdges = 1,
    kCntEdgesCached = 2,
    kCntExpanded = 3,
    kCntAffected = 4,
    kCntSeeds = 5,
    kCntMissing = 6,
    kCntInvalid = 7,
    kCntChanged = 8,
    kCntRelocated = 9,
    kCntSegLoaded = 10,
    kCntSegEvicted = 11,
    kCntPrRounds = 12,
    kCntRemoved = 13,
    kCntSrcEdges = 14,  // multi-source queries: sum of (source bits x row length) over expanded rows
    // Per-kernel groups of 4: edges, edges from HBM, rows expanded, hits.
    kCntPush = 16,
    kCntInval = 20,
    kCntPull = 24,
    kCntPr = 28,
    // Flat deletion scan (forward and reverse rows): row entries read, of
    // which from HBM.
    kCntDelScanned = 32,
    kCntDelScannedCached = 33,
    // Forward row entries copied by relocations (addition phase).
    kCntMovedEntries = 34,
};

// Hint: bring the line holding `p` into L2 (no register result, no wait).
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) {
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

__device__ __forceinline__ void set_error(Status *st, uint32_t code, uint32_t info = 0) {
    if ((atomicOr(&st->err, code) & code) == 0) st->err_info = info;
}

__device__ __forceinline__ void report_bounds(Status *st, uint64_t index) {
    if (st) set_error(st, kErrBounds, static_cast<uint32_t>(index));
}

// Warp-aggregated append: one atomicAdd per warp.  All 32 lanes must call.
__device__ __forceinline__ void warp_enqueue(bool want, uint32_t item, uint32_t *queue, uint32_t *count,
                                             uint32_t capacity, Status *st) {
    const uint32_t mask = __ballot_sync(kFull, want);
    if (!mask) return;
    const uint32_t lane = lane_id();
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(kFull, base, leader);
    if (want) {
        const uint32_t pos = base + __popc(mask & lanemask_lt());
        if (pos < capacity)
            queue[pos] = item;
        else
            set_error(st, kErrQueue, pos);
    }
}

// Append up to N items per lane (item[j] where want[j]) with one warp scan
// and one atomic per warp.
template <int N>
__device__ __forceinline__ void warp_enqueue_n(const bool (&want)[N], const uint32_t (&item)[N], uint32_t *queue,
                                               uint32_t *count, uint32_t capacity, Status *st) {
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < N; ++j) c += want[j] ? 1u : 0u;
    if (!__any_sync(kFull, c != 0u)) return;
    const uint32_t lane = lane_id();
    uint32_t incl = c;
#pragma unroll
    for (uint32_t o = 1; o < 32u; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    uint32_t base = 0;
    if (lane == 31) base = atomicAdd(count, incl);
    base = __shfl_sync(kFull, base, 31);
    uint32_t pos = base + incl - c;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        if (want[j]) {
            if (pos < capacity)
                queue[pos] = item[j];
            else
                set_error(st, kErrQueue, pos);
            ++pos;
        }
    }
}

// Warp-aggregated counter add.
__device__ __forceinline__ void warp_count(unsigned long long *counter, uint32_t value) {
    uint32_t sum = __reduce_add_sync(kFull, value);
    if (lane_id() == 0 && sum) atomicAdd(counter, static_cast<unsigned long long>(sum));
}

// Grid-wide barrier for cooperatively launched kernels.  Waits are bounded:
// after ~2 s without progress the waiting block records kErrBarrier and
// returns false; every later barrier then returns false at once.
constexpr long long kBarrierTimeoutCycles = 4000000000LL;

__device__ __forceinline__ bool grid_barrier(Status *st) {
    __syncthreads();
    __shared__ uint32_t ok;
    if (threadIdx.x == 0) {
        ok = 1;
        const uint32_t gen = atomicAdd(&st->barrier_gen, 0);
        __threadfence();
        const uint32_t arrived = atomicAdd(&st->barrier_count, 1);
        if (arrived == gridDim.x - 1) {
            atomicExch(&st->barrier_count, 0);
            __threadfence();
            atomicAdd(&st->barrier_gen, 1);
        } else {
            const long long start = clock64();
            while (ld_volatile(&st->barrier_gen) == gen) {
                if (ld_volatile(&st->err) & kErrBarrier) break;
                if (clock64() - start > kBarrierTimeoutCycles) {
                    set_error(st, kErrBarrier, blockIdx.x);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        if (ld_volatile(&st->err) & kErrBarrier) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// Edge weights of the reference samples: BFS 1 (samples/hybrid_bfs/
// hybrid_bfs.cu:41-47), SSSP (src+dst)%128+1 (include/framework/variants/
// api.cuh:26-28), CC 0 (samples/hybrid_cc/hybrid_cc.cu:51-57).
// kSsspU: SSSP with weights uniform in [1, 255] (CIG_FLAG_WEIGHT_U255).
enum Algo : int { kBfs = 0, kSssp = 1, kCc = 2, kPr = 3, kSsspU = 4 };

// Weight of edge (u, v) in [1, 255] for kSsspU: 1 + lowbias32(u*G + v*H)
// mod 255, where lowbias32 is C. Wellons' published 32-bit integer hash
// ("Prospecting for hash functions", 2018).  A function of the edge, so the
// weight needs no storage and moves with the row; the reference itself never
// stores file weights (its chunk store holds destinations only).
__host__ __device__ __forceinline__ uint32_t weight_u255(uint32_t u, uint32_t v) {
    uint32_t x = u * 0x9E3779B1u + v * 0x85EBCA77u;
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return 1u + x % 255u;
}

template <int A>
__device__ __forceinline__ uint32_t edge_weight(uint32_t u, uint32_t v) {
    if (A == kBfs) return 1u;
    if (A == kCc) return 0u;
    if (A == kSsspU) return weight_u255(u, v);
    return ((u + v) & 127u) + 1u;  // (u+v) mod 2^32 keeps the residue mod 128
}

__device__ __forceinline__ uint32_t cc_step(uint32_t v, uint32_t shift);

// Value of y relaxed from x with value dx (CC: one more hop from the seed).
template <int A>
__device__ __forceinline__ uint32_t relax_value(uint32_t dx, uint32_t x, uint32_t y, uint32_t ccs) {
    if (A == kCc) return cc_step(dx, ccs);
    return dx + edge_weight<A>(x, y);
}

__device__ __forceinline__ uint32_t val_of(unsigned long long s) { return static_cast<uint32_t>(s >> 32); }

// CC values carry a depth below the label: value = label << shift | depth,
// where depth counts the hops from the component's seed (the vertex whose id
// is the label) along parents and saturates at the low-bit mask.  The
// lexicographic minimum (label, depth, parent) makes every unsaturated
// parent chain strictly shorter towards the seed, so a parent is a rooted
// witness and a deletion invalidates only the subtree below it; saturated
// vertices (and shift 0, for graphs of more than 2^31 vertices) fall back to
// invalidating every equal-label out-neighbour.  Labels (value >> shift) are
// the reference's values.
__device__ __forceinline__ uint32_t cc_step(uint32_t v, uint32_t shift) {
    const uint32_t m = (1u << shift) - 1u;
    return (v & m) == m ? v : v + 1u;
}
__device__ __forceinline__ bool cc_saturated(uint32_t v, uint32_t shift) {
    const uint32_t m = (1u << shift) - 1u;
    return (v & m) == m;
}
__device__ __forceinline__ uint32_t par_of(unsigned long long s) { return static_cast<uint32_t>(s); }
__device__ __forceinline__ unsigned long long pack(uint32_t value, uint32_t parent) {
    return (static_cast<unsigned long long>(value) << 32) | parent;
}

}  // namespace cig
