// query.cuh - multi-source BFS and SSSP with 64-wide bitmask frontiers.
//
// One wave serves up to 64 sources.  Per vertex the wave keeps a 64-bit mask
// of the sources whose value at that vertex changed in the last round, so a
// row is read once per round for all of those sources (the "MS-BFS" idea of
// Then et al., "The More the Merrier: Efficient Multi-Source Graph
// Traversal", VLDB 2014, applied to label-correcting SSSP as well).  Values
// are stored vertex-major, `width` words per vertex (the wave width, 1..64),
// so the sources of one vertex share cache lines; a transpose kernel writes
// the k x n source-major result.
//
// The reference answers one source per engine run (BFS/SSSP Start,
// include/framework/framework.cuh:1151-1182); these queries give the same
// depths and distances (the values are unique) for many sources at once,
// over the same adjacency (cache or zero-copy rows) and edge weights.
#pragma once

#include "common.cuh"
#include "expand.cuh"
#include "traverse.cuh"

namespace cig {

constexpr uint32_t kMsWidth = 64;
constexpr int kTpbMs = 256;

struct MsFrontier {
    uint32_t *q0;
    uint32_t *q1;
    uint32_t *cnt;                // 3 round counters, as for the push closure
    unsigned long long *mask0;    // source masks read in even rounds
    unsigned long long *mask1;    // ... in odd rounds
    uint32_t cap;
};

// BFS: a source bit reaches y the first time any round carries it there;
// `visit` holds the bits that already reached each vertex, so a bit is set
// (and its depth written) exactly once.
struct MsBfsOp {
    uint32_t *dist;
    uint32_t width;
    unsigned long long *visit;
    unsigned long long *mask_out;
    uint32_t level;
    uint32_t *q_out;
    uint32_t *q_count;
    uint32_t q_cap;
    Status *st;

    __device__ __forceinline__ bool edge(bool valid, uint32_t, unsigned long long m, uint32_t y) const {
        bool want = false, hit = false;
        if (valid) {
            const unsigned long long cand = m & ~__ldcg(visit + y);
            if (cand) {
                const unsigned long long nb = cand & ~atomicOr(visit + y, cand);
                if (nb) {
                    hit = true;
                    uint32_t *row = dist + static_cast<uint64_t>(y) * width;
                    for (unsigned long long b = nb; b; b &= b - 1) row[__ffsll(static_cast<long long>(b)) - 1] = level;
                    want = atomicOr(mask_out + y, nb) == 0ull;
                }
            }
        }
        warp_enqueue(want, y, q_out, q_count, q_cap, st);
        return hit;
    }
};

// SSSP (or BFS with unit weights): label-correcting relaxation per source
// bit; a bit is carried to y for the next round when it lowered y's value.
template <int A>
struct MsRelaxOp {
    uint32_t *dist;
    uint32_t width;
    unsigned long long *mask_out;
    uint32_t *q_out;
    uint32_t *q_count;
    uint32_t q_cap;
    Status *st;

    __device__ __forceinline__ bool edge(bool valid, uint32_t x, unsigned long long m, uint32_t y) const {
        bool want = false;
        unsigned long long add = 0;
        if (valid) {
            const uint32_t w = edge_weight<A>(x, y);
            const uint32_t *rx = dist + static_cast<uint64_t>(x) * width;
            uint32_t *ry = dist + static_cast<uint64_t>(y) * width;
            for (unsigned long long b = m; b; b &= b - 1) {
                const int i = __ffsll(static_cast<long long>(b)) - 1;
                const uint32_t nd = __ldcg(rx + i) + w;
                if (nd < __ldcg(ry + i) && nd < atomicMin(ry + i, nd)) add |= 1ull << i;
            }
            if (add) want = atomicOr(mask_out + y, add) == 0ull;
        }
        warp_enqueue(want, y, q_out, q_count, q_cap, st);
        return add != 0ull;
    }
};

// Seeds of one wave: source j of the wave gets bit j, value 0, and its
// vertex is queued once (several bits may share a vertex).
__global__ void ms_seed(const uint32_t *sources, uint32_t k, uint32_t *dist, uint32_t width,
                        unsigned long long *visit, MsFrontier fr, Status *st) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const uint32_t s = sources[j];
    dist[static_cast<uint64_t>(s) * width + j] = 0u;
    if (visit) atomicOr(visit + s, 1ull << j);
    if (atomicOr(fr.mask0 + s, 1ull << j) == 0ull) {
        const uint32_t pos = atomicAdd(fr.cnt + 0, 1u);
        if (pos < fr.cap)
            fr.q0[pos] = s;
        else
            set_error(st, kErrQueue, pos);
    }
}

// Direction switching of the BFS wave (Beamer, Asanovic and Patterson,
// "Direction-optimizing breadth-first search", SC 2012, on a bitmask
// frontier): a round runs bottom-up when the frontier holds more than
// `on` vertices (or, once bottom-up, at least `off`); 0 disables it.
struct MsPull {
    AdjView rev;             // in-edges (desc null: no bottom-up)
    uint32_t n;
    unsigned long long full; // the wave's source bits
    uint32_t on, off;
};

// Bottom-up round: every vertex still missing source bits ORs the frontier
// masks of its in-neighbours (stopping once nothing is missing) and takes
// the new bits; one thread per vertex, so `visit` needs no atomics.
__device__ __forceinline__ void ms_bottom_up(const MsPull &pl, uint32_t *dist, uint32_t width,
                                             unsigned long long *visit, const unsigned long long *m_in,
                                             unsigned long long *m_out, uint32_t level, uint32_t *q_out,
                                             uint32_t *q_cnt, uint32_t cap, Status *st, ExpandCounters &cnt) {
    const uint32_t rounded = (pl.n + 31u) & ~31u;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < rounded; w += gridDim.x * blockDim.x) {
        bool want = false;
        if (w < pl.n) {
            const unsigned long long vis = __ldcg(visit + w);
            const unsigned long long missing = pl.full & ~vis;
            if (missing) {
                const RowDesc d = pl.rev.desc[w];
                unsigned long long acc = 0;
                uint32_t k = 0;
                for (; k < d.len && (acc & missing) != missing; ++k) {
                    const uint32_t u = __ldg(pl.rev.at(d.off + k));
                    if (u != kTomb) acc |= __ldcg(m_in + u);
                }
                cnt.edges += k;
                cnt.edges_cached += k;
                cnt.rows += d.len ? 1u : 0u;
                const unsigned long long nb = acc & missing;
                if (nb) {
                    visit[w] = vis | nb;
                    uint32_t *row = dist + static_cast<uint64_t>(w) * width;
                    for (unsigned long long b = nb; b; b &= b - 1) row[__ffsll(static_cast<long long>(b)) - 1] = level;
                    m_out[w] = nb;
                    want = true;
                    ++cnt.hits;
                }
            }
        }
        warp_enqueue(want, w, q_out, q_cnt, cap, st);
    }
}

// Persistent multi-source closure (cooperative launch): round r expands the
// vertices queued in round r-1 with the source bits that reached them.
// BFS (kBfs with `visit`) is level-synchronous: round r writes depth r+1,
// top-down or (with `pl`) bottom-up.
template <int A>
__global__ void __launch_bounds__(kTpbMs) ms_closure(AdjView fwd, uint32_t *dist, uint32_t width,
                                                     unsigned long long *visit, MsFrontier fr, BigList big,
                                                     uint32_t max_rounds, MsPull pl, Status *st) {
    __shared__ ExpandSmem<kTpbMs, unsigned long long> sm;
    ExpandCounters cnt;
    unsigned long long src_edges = 0;
    bool pull = false;  // every block takes the same decisions from the same counts
    const bool can_pull = A == kBfs && visit && pl.rev.desc && pl.on;
    uint32_t r = 0;
    for (;; ++r) {
        const uint32_t n_in = ld_volatile(fr.cnt + (r % 3));
        if (n_in == 0) break;
        if (r >= max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) set_error(st, kErrRounds, r);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fr.cnt[(r + 2) % 3] = 0;
            big.cnt[(r + 2) % 3] = 0;
        }
        const uint32_t *in = (r & 1) ? fr.q1 : fr.q0;
        uint32_t *out = (r & 1) ? fr.q0 : fr.q1;
        unsigned long long *m_in = (r & 1) ? fr.mask1 : fr.mask0;
        unsigned long long *m_out = (r & 1) ? fr.mask0 : fr.mask1;
        if (can_pull) pull = n_in > (pull ? pl.off : pl.on);
        if (pull) {
            ms_bottom_up(pl, dist, width, visit, m_in, m_out, r + 1, out, fr.cnt + ((r + 1) % 3), fr.cap, st, cnt);
            if (!grid_barrier(st)) break;
            // The frontier masks were read, not taken: clear them before
            // the next round writes into this array.
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_in; i += gridDim.x * blockDim.x)
                m_in[__ldcg(in + i)] = 0ull;
            if (!grid_barrier(st)) break;
            continue;
        }
        const Defer df{big.rows, big.cnt + (r % 3), big.cap, big.split};
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpbMs) {
            const uint32_t i = base + spread_rank<kTpbMs>() * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t x = 0, deg = 0;
            uint64_t off = 0;
            unsigned long long m = 0;
            if (has) {
                x = __ldcg(in + i);
                // Nobody writes m_in this round: take the bits and clear them.
                m = __ldcg(m_in + x);
                m_in[x] = 0ull;
                const RowDesc d = fwd.desc[x];
                deg = d.len;
                off = d.off;
                has = m != 0ull && deg > 0;
                if (has) src_edges += static_cast<unsigned long long>(__popcll(m)) * deg;
            }
            // (Warp-only tiers, expand_rows_warp, measured the same for BFS and
            // 12 % slower for SSSP waves than the block tiers.)
            if (A == kBfs && visit) {
                const MsBfsOp op{dist, width, visit, m_out, r + 1, out, fr.cnt + ((r + 1) % 3), fr.cap, st};
                expand_rows<kTpbMs>(fwd, has, x, m, off, deg, op, sm, cnt, df);
            } else {
                const MsRelaxOp<A> op{dist, width, m_out, out, fr.cnt + ((r + 1) % 3), fr.cap, st};
                expand_rows<kTpbMs>(fwd, has, x, m, off, deg, op, sm, cnt, df);
            }
        }
        if (!grid_barrier(st)) break;
        const uint32_t nbig = min(ld_volatile(big.cnt + (r % 3)), big.cap);
        if (nbig) {
            if (A == kBfs && visit) {
                const MsBfsOp op{dist, width, visit, m_out, r + 1, out, fr.cnt + ((r + 1) % 3), fr.cap, st};
                expand_deferred<kTpbMs, unsigned long long>(fwd, big.rows, nbig, op, cnt);
            } else {
                const MsRelaxOp<A> op{dist, width, m_out, out, fr.cnt + ((r + 1) % 3), fr.cap, st};
                expand_deferred<kTpbMs, unsigned long long>(fwd, big.rows, nbig, op, cnt);
            }
            if (!grid_barrier(st)) break;
        }
    }
    flush_counters(st, cnt, kCntPush);
    {
        unsigned long long s = src_edges;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
        if (lane_id() == 0 && s) atomicAdd(&st->counters[kCntSrcEdges], s);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->counters[kCntRounds], static_cast<unsigned long long>(r));
}

// Source-major output: out[j * n + v] = dist[v * width + j] for j < k,
// through a shared-memory tile so that both sides are coalesced.
constexpr uint32_t kMsTile = 32;

__global__ void ms_transpose(const uint32_t *dist, uint32_t n, uint32_t width, uint32_t k, uint32_t *out) {
    __shared__ uint32_t tile[kMsTile][kMsWidth + 1];
    const uint32_t v0 = blockIdx.x * kMsTile;
    const uint32_t rows = min(kMsTile, n - v0);
    // The tile's vertices are contiguous in `dist`: rows x width words.
    const uint64_t base = static_cast<uint64_t>(v0) * width;
    for (uint32_t e = threadIdx.x; e < rows * width; e += blockDim.x) tile[e / width][e % width] = dist[base + e];
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < kMsTile * k; e += blockDim.x) {
        const uint32_t j = e / kMsTile, vv = e % kMsTile;
        if (vv < rows) out[static_cast<uint64_t>(j) * n + v0 + vv] = tile[vv][j];
    }
}

// Digest of every row of a k x n result (the function of value_digest, so a
// query row and a maintained state with the same values agree).
__global__ void ms_row_digest(const uint32_t *rows, uint32_t n, unsigned long long *out) {
    const uint32_t j = blockIdx.y;
    const uint32_t *row = rows + static_cast<uint64_t>(j) * n;
    unsigned long long acc = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t d = row[v];
        if (d != kInf) acc += digest_mix((static_cast<unsigned long long>(v) << 32) | d);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane_id() == 0 && acc) atomicAdd(out + j, acc);
}

}  // namespace cig
