// posindex.cuh - position index of hub rows.
//
// The reference deletes the first occurrence of (u, v) from u's row, whose
// order is the file/insertion order, so a deletion must find v's first
// position in an unordered row.  For most rows the flat scan (del_scan) is
// cheap; hub rows are not: on R-MAT s24 they made up most of the ~87 M row
// entries a 100 k-deletion batch scanned.  Rows whose block class was at
// least a threshold when the index was last built (`rowbit`)
// therefore keep, in one open-addressing hash table per arena, an entry per
// distinct (u, v): the position of v's first live occurrence in u's row and
// the number of live occurrences.  Deletions look positions up; appends,
// relocations and compactions keep the entries current.
//
// Table: keys (u << 32 | v), EMPTY / DELETED sentinels, linear probing with
// a bounded probe length (kIdxProbe; running past it is reported as
// kErrInternal, never a fault).  Values {pos, count} start as {kInf, 0} in
// every slot, so an insert is a key CAS followed by atomicMin / atomicAdd
// with no initialisation race.  A slot is never reused after DELETED (so a
// probe never meets an EMPTY slot before its key); the host sizes the table
// with room for as many inserts as it has entries and rebuilds it before the
// keys inserted since the last build can take the load factor past one half.
#pragma once

#include "common.cuh"

namespace cig {

constexpr unsigned long long kIdxEmpty = ~0ull;
constexpr unsigned long long kIdxDeleted = ~0ull - 1ull;
constexpr uint32_t kIdxCls = 5;       // default: rows in blocks of >= 32 slots are indexed
constexpr uint32_t kIdxProbe = 4096;  // probe bound

struct PosIndex {
    unsigned long long *keys;  // null: no index for this arena
    uint2 *val;                // x: first live position, y: live occurrences
    unsigned long long mask;   // capacity - 1 (power of two)
    const uint32_t *rowbit;    // bit v: row v is indexed
};

__device__ __forceinline__ unsigned long long idx_mix(unsigned long long k) {
    // SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom number generators", 2014)
    k ^= k >> 30;
    k *= 0xBF58476D1CE4E5B9ull;
    k ^= k >> 27;
    k *= 0x94D049BB133111EBull;
    return k ^ (k >> 31);
}

__device__ __forceinline__ bool idx_row(const PosIndex &ix, uint32_t v) {
    return ix.keys && ((__ldg(ix.rowbit + (v >> 5)) >> (v & 31u)) & 1u);
}

// Slot of `key`, or ~0 when absent; the probe starts at slot `s`, its
// `first`-th step.
__device__ __forceinline__ unsigned long long idx_find_from(const PosIndex &ix, unsigned long long key,
                                                            unsigned long long s, uint32_t first) {
    for (uint32_t i = first; i < kIdxProbe; ++i, s = (s + 1) & ix.mask) {
        const unsigned long long k = *reinterpret_cast<volatile unsigned long long *>(ix.keys + s);
        if (k == key) return s;
        if (k == kIdxEmpty) return ~0ull;
    }
    return ~0ull;
}

// Slot of `key`, or ~0 when absent.
__device__ __forceinline__ unsigned long long idx_find(const PosIndex &ix, unsigned long long key) {
    unsigned long long s = idx_mix(key) & ix.mask;
    for (uint32_t i = 0; i < kIdxProbe; ++i, s = (s + 1) & ix.mask) {
        const unsigned long long k = *reinterpret_cast<volatile unsigned long long *>(ix.keys + s);
        if (k == key) return s;
        if (k == kIdxEmpty) return ~0ull;
    }
    return ~0ull;
}

// Slot of `key`, inserting it when absent; ~0 (and an error) when the probe
// bound is reached.
__device__ __forceinline__ unsigned long long idx_insert(const PosIndex &ix, unsigned long long key, Status *st) {
    unsigned long long s = idx_mix(key) & ix.mask;
    for (uint32_t i = 0; i < kIdxProbe; ++i, s = (s + 1) & ix.mask) {
        unsigned long long k = *reinterpret_cast<volatile unsigned long long *>(ix.keys + s);
        if (k == kIdxEmpty) k = atomicCAS(ix.keys + s, kIdxEmpty, key);
        if (k == kIdxEmpty || k == key) return s;
    }
    set_error(st, kErrInternal, 0x1d0u);
    return ~0ull;
}

// The slots of the keys (u, v[j]) of an indexed row for the live j, ~0 for
// the others: the first probe of every key is in flight together; a
// collision continues with idx_find_from.  A live key that is absent sets
// an internal error (the row holds it, so the index must).
template <int N>
__device__ __forceinline__ void idx_find_n(const PosIndex &ix, uint32_t u, const uint32_t (&v)[N],
                                           const bool (&live)[N], unsigned long long (&slot)[N], Status *st) {
    unsigned long long key[N], seen[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
        key[j] = (static_cast<unsigned long long>(u) << 32) | v[j];
        slot[j] = idx_mix(key[j]) & ix.mask;
        seen[j] = key[j];
        if (live[j]) seen[j] = *reinterpret_cast<volatile unsigned long long *>(ix.keys + slot[j]);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
        if (!live[j]) {
            slot[j] = ~0ull;
        } else if (seen[j] != key[j]) {
            slot[j] = seen[j] == kIdxEmpty ? ~0ull : idx_find_from(ix, key[j], (slot[j] + 1) & ix.mask, 1);
            if (slot[j] == ~0ull) set_error(st, kErrInternal, 0x1d1u);
        }
    }
}

// The first a of v[0..N) appear (again) at positions p0, p0 + 1, ... of
// indexed row u: every key's first probe (a load, then a compare-and-swap
// where the slot is empty) is in flight together; a collision continues
// with idx_insert.
template <int N>
__device__ __forceinline__ void idx_add_n(const PosIndex &ix, uint32_t u, const uint32_t (&v)[N], uint32_t p0,
                                          uint32_t a, Status *st) {
    unsigned long long key[N], slot[N], seen[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
        key[j] = (static_cast<unsigned long long>(u) << 32) | v[j];
        slot[j] = idx_mix(key[j]) & ix.mask;
        seen[j] = key[j];
        if (static_cast<uint32_t>(j) < a)
            seen[j] = *reinterpret_cast<volatile unsigned long long *>(ix.keys + slot[j]);
    }
#pragma unroll
    for (int j = 0; j < N; ++j)
        if (static_cast<uint32_t>(j) < a && seen[j] == kIdxEmpty)
            seen[j] = atomicCAS(ix.keys + slot[j], kIdxEmpty, key[j]);
#pragma unroll
    for (int j = 0; j < N; ++j) {
        if (static_cast<uint32_t>(j) >= a) continue;
        if (seen[j] != kIdxEmpty && seen[j] != key[j]) slot[j] = idx_insert(ix, key[j], st);
        if (slot[j] == ~0ull) continue;
        atomicMin(&ix.val[slot[j]].x, p0 + j);
        atomicAdd(&ix.val[slot[j]].y, 1u);
    }
}

// v appears (again) at position p of indexed row u.
__device__ __forceinline__ void idx_add(const PosIndex &ix, uint32_t u, uint32_t v, uint32_t p, Status *st) {
    const unsigned long long s = idx_insert(ix, (static_cast<unsigned long long>(u) << 32) | v, st);
    if (s == ~0ull) return;
    atomicMin(&ix.val[s].x, p);
    atomicAdd(&ix.val[s].y, 1u);
}

// Positions of an indexed row changed (compaction, relocation): every live
// entry's first position is recomputed in two passes separated by a
// barrier of the caller: reset, then atomicMin of the new positions.
__device__ __forceinline__ void idx_pos_reset(const PosIndex &ix, uint32_t u, uint32_t v, Status *st) {
    const unsigned long long s = idx_find(ix, (static_cast<unsigned long long>(u) << 32) | v);
    if (s == ~0ull) {
        set_error(st, kErrInternal, 0x1d1u);
        return;
    }
    atomicExch(&ix.val[s].x, kInf);
}

__device__ __forceinline__ void idx_pos_set(const PosIndex &ix, uint32_t u, uint32_t v, uint32_t p) {
    const unsigned long long s = idx_find(ix, (static_cast<unsigned long long>(u) << 32) | v);
    if (s != ~0ull) atomicMin(&ix.val[s].x, p);
}

// ---------------------------------------------------------------- kernels

__global__ void idx_init(PosIndex ix) {
    for (unsigned long long s = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; s <= ix.mask;
         s += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        ix.keys[s] = kIdxEmpty;
        ix.val[s] = make_uint2(kInf, 0u);
    }
}

// Slots of the rows of every block class (64 bins), from which the host
// picks the smallest class threshold whose table fits its memory share.
__global__ void idx_class_slots(const RowDesc *desc, uint32_t n, unsigned long long *hist) {
    __shared__ unsigned long long h[64];
    for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const RowDesc d = desc[v];
        if (d.len) atomicAdd(&h[rd_cls(d)], static_cast<unsigned long long>(d.len));
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Rows of class >= min_cls: set their bit and list them.
__global__ void idx_pick_rows(const RowDesc *desc, uint32_t n, uint32_t min_cls, uint32_t *rowbit, uint32_t *list,
                              uint32_t *count, uint32_t cap, Status *st) {
    const uint32_t rounded = (n + 31u) & ~31u;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < rounded; v += gridDim.x * blockDim.x) {
        const bool big = v < n && rd_cls(desc[v]) >= min_cls;
        const uint32_t bits = __ballot_sync(kFull, big);
        if (lane_id() == 0 && v < n) rowbit[v >> 5] = bits;
        warp_enqueue(big, v, list, count, cap, st);
    }
}

// Entries of the listed rows; one block per row.
__global__ void idx_build(AdjView view, const RowDesc *desc, const uint32_t *list, const uint32_t *count,
                          PosIndex ix, Status *st) {
    // Rows of at least kIdxBlockRow entries: a block each; shorter rows (most
    // of them) a warp each, so that lanes are not left idle on short rows.
    constexpr uint32_t kIdxBlockRow = 512;
    const uint32_t nr = *count;
    for (uint32_t r = blockIdx.x; r < nr; r += gridDim.x) {
        const uint32_t u = list[r];
        const RowDesc d = desc[u];
        if (d.len < kIdxBlockRow) continue;
        for (uint32_t k = threadIdx.x; k < d.len; k += blockDim.x) {
            const uint32_t v = *view.at(d.off + k);
            if (v != kTomb) idx_add(ix, u, v, k, st);
        }
    }
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nr; r += warps) {
        const uint32_t u = list[r];
        const RowDesc d = desc[u];
        if (d.len >= kIdxBlockRow) continue;
        for (uint32_t k = lane; k < d.len; k += 32u) {
            const uint32_t v = *view.at(d.off + k);
            if (v != kTomb) idx_add(ix, u, v, k, st);
        }
    }
}

}  // namespace cig
