// expand.cuh - load-balanced neighbour-list expansion for one thread block.
//
// Every thread of the block brings at most one row (a frontier vertex and its
// adjacency block).  Rows are served in three tiers so that work per lane
// stays even whatever the degree mix (scan-based gather, Merrill, Garland and
// Grimshaw, "Scalable GPU graph traversal", PPoPP 2012):
//   1. rows with >= TPB entries: the whole block strides over the row;
//   2. rows with >= 32 entries: the owning warp strides over the row;
//   3. smaller rows: each warp concatenates its lanes' rows with a warp scan
//      and hands out the combined edge list 32 entries at a time.
// The reference balances with CTAWorkSchedulerNew
// (include/groute/device/cta_scheduler_hybrid.cuh:55-237); this is a new
// design (tiers, a scan instead of per-row scheduling) that keeps every
// Op::edge call warp-synchronous so that ops can use warp-aggregated queue
// appends.
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"

namespace cig {

// P is the per-row payload handed to Op::edge: a 32-bit value for the
// maintained algorithms, a 64-bit source mask for multi-source queries.
template <int TPB, class P = uint32_t>
struct ExpandSmem {
    uint32_t owner;
    uint32_t b_x, b_deg;
    P b_payload;
    unsigned long long b_off;
    uint32_t f_scan[TPB];
    uint32_t f_x[TPB];
    P f_payload[TPB];
    const uint32_t *f_ptr[TPB];
};

struct ExpandCounters {
    uint32_t edges = 0;
    uint32_t edges_cached = 0;
    uint32_t rows = 0;
    uint32_t hits = 0;  // edges whose op changed state (relaxations, claims)
};

// Add a thread's counters to the batch totals and to one kernel's group of
// four slots (edges, edges served from HBM, rows, hits).  All lanes call.
__device__ __forceinline__ void flush_counters(Status *st, const ExpandCounters &c, int group) {
    warp_count(&st->counters[kCntEdges], c.edges);
    warp_count(&st->counters[kCntEdgesCached], c.edges_cached);
    warp_count(&st->counters[kCntExpanded], c.rows);
    warp_count(&st->counters[group + 0], c.edges);
    warp_count(&st->counters[group + 1], c.edges_cached);
    warp_count(&st->counters[group + 2], c.rows);
    warp_count(&st->counters[group + 3], c.hits);
}

// Rows with at least `split` entries (default kSplitDeg) are not expanded by the block that
// holds them: they are appended to a list that every block of the grid
// then expands in kSplitChunk-entry chunks (expand_deferred), so that one
// hub row does not serialise a whole round on one block.
constexpr uint32_t kSplitDeg = 4096;
constexpr uint32_t kSplitChunk = 1024;

struct BigRow {
    unsigned long long off;
    unsigned long long payload;
    uint32_t x, deg;
};

struct Defer {
    BigRow *rows;     // null: expand every row in place
    uint32_t *count;
    uint32_t cap;
    uint32_t split;   // rows of at least this many entries are deferred
};

// Ops whose first access per edge is a plain load of a word of the edge's
// target (its state word) expose it as `peek(y)` and take the loaded word in
// `edge_peeked(valid, x, payload, y, word)`.  The sweeps then issue the loads
// of a thread's entries together before any of them is used, instead of one
// dependent load per edge() call.  Ops without peek() run edge() per entry.
template <class Op, class = void>
struct has_peek : std::false_type {};
template <class Op>
struct has_peek<Op, std::void_t<decltype(std::declval<const Op &>().peek(0u))>> : std::true_type {};

// Ops that declare kMulti also take a thread's N entries at once
// (edges<N>(valid, x, payload, y, peeked)): their atomics are then in flight
// together and their queue appends share one warp scan, instead of N
// rounds of atomic, ballot and append.
template <class Op, class = void>
struct has_multi : std::false_type {};
template <class Op>
struct has_multi<Op, std::void_t<decltype(Op::kMulti)>> : std::true_type {};

// N entries of one thread: entry j is edge x[j] -> y[j] with payload pl[j],
// live when v[j].
template <int N, class Op, class P>
__device__ __forceinline__ uint32_t edges_n(const Op &op, const bool (&v)[N], const uint32_t (&x)[N],
                                            const P (&pl)[N], const uint32_t (&y)[N]) {
    uint32_t hits = 0;
    if constexpr (has_peek<Op>::value) {
        using W = decltype(op.peek(0u));
        W w[N];
#pragma unroll
        for (int j = 0; j < N; ++j) w[j] = v[j] ? op.peek(y[j]) : W{};
        if constexpr (has_multi<Op>::value) {
            hits = op.template edges<N>(v, x, pl, y, w);
        } else {
#pragma unroll
            for (int j = 0; j < N; ++j) hits += op.edge_peeked(v[j], x[j], pl[j], y[j], w[j]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < N; ++j) hits += op.edge(v[j], x[j], pl[j], y[j]);
    }
    return hits;
}

// The four entries of a 16-byte row load: entry j is live when it lies
// before `deg` (relative index k + j) and is not a tombstone.
template <class Op, class P>
__device__ __forceinline__ uint32_t edge4(const Op &op, uint4 q, uint32_t k, uint32_t deg, uint32_t x, P payload) {
    const bool v[4] = {k < deg && q.x != kTomb, k + 1u < deg && q.y != kTomb, k + 2u < deg && q.z != kTomb,
                       k + 3u < deg && q.w != kTomb};
    const uint32_t xs[4] = {x, x, x, x};
    const P ps[4] = {payload, payload, payload, payload};
    const uint32_t ys[4] = {q.x, q.y, q.z, q.w};
    return edges_n<4>(op, v, xs, ps, ys);
}

// Sweep of one row by `lanes` threads (a warp or a block; `t` = the
// thread's rank among them).  Rows start on a 16-byte boundary in the
// arenas (a block of 2^c >= 4 slots is aligned to its size), so each thread
// reads four consecutive entries with one 16-byte load: a warp moves 128
// entries, 512 bytes, per step, and a zero-copy row crosses the host link
// in full 16-byte requests.  The load of a thread's next step is issued
// before the current step's entries are used, so on rows of several steps
// the row reads overlap the state reads.  Entries past `deg` (still inside
// the block, whose size is a multiple of 4) are masked.  A row that is not
// 16-byte aligned (a caller's plain CSR) is read one entry per thread.
// Every thread of the group runs the same number of steps (Op::edge is
// warp-synchronous).
template <uint32_t lanes, class Op, class P>
__device__ __forceinline__ void sweep_row(const AdjView &view, const uint32_t *rp, uint32_t deg, uint32_t t,
                                          uint32_t x, P payload, const Op &op, ExpandCounters &cnt) {
    const bool aligned = (reinterpret_cast<uintptr_t>(rp) & 15u) == 0;
    if constexpr (has_peek<Op>::value && has_multi<Op>::value) {
        if (aligned) {
            // Two steps in flight: while a step's entries are relaxed, the
            // next step's state words are being read and the one after
            // that's row entries.
            using W = decltype(op.peek(0u));
            const uint4 tomb4 = make_uint4(kTomb, kTomb, kTomb, kTomb);
            const uint32_t xs[4] = {x, x, x, x};
            const P ps[4] = {payload, payload, payload, payload};
            auto live = [&](uint4 &q, uint32_t k, bool (&v)[4], uint32_t (&ys)[4]) {
                ys[0] = view.vid(q.x);
                ys[1] = view.vid(q.y);
                ys[2] = view.vid(q.z);
                ys[3] = view.vid(q.w);
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = k + j < deg && ys[j] != kTomb;
            };
            uint32_t k = 4u * t;
            uint4 q = k < deg ? __ldg(reinterpret_cast<const uint4 *>(rp + k)) : tomb4;
            bool v[4];
            uint32_t ys[4];
            W w[4];
            live(q, k, v, ys);
#pragma unroll
            for (int j = 0; j < 4; ++j) w[j] = v[j] ? op.peek(ys[j]) : W{};
            uint32_t kn = k + 4u * lanes;
            uint4 qn = kn < deg ? __ldg(reinterpret_cast<const uint4 *>(rp + kn)) : tomb4;
            for (uint32_t base = 0; base < deg; base += 4u * lanes) {
                bool vn[4];
                uint32_t yn[4];
                W wn[4];
                live(qn, kn, vn, yn);
#pragma unroll
                for (int j = 0; j < 4; ++j) wn[j] = vn[j] ? op.peek(yn[j]) : W{};
                const uint32_t knn = kn + 4u * lanes;
                const uint4 qnn = knn < deg ? __ldg(reinterpret_cast<const uint4 *>(rp + knn)) : tomb4;
                cnt.hits += op.template edges<4>(v, xs, ps, ys, w);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    v[j] = vn[j];
                    ys[j] = yn[j];
                    w[j] = wn[j];
                }
                qn = qnn;
                kn = knn;
            }
            return;
        }
    }
    if (aligned) {
        const uint4 tomb4 = make_uint4(kTomb, kTomb, kTomb, kTomb);
        uint32_t k = 4u * t;
        uint4 q = k < deg ? __ldg(reinterpret_cast<const uint4 *>(rp + k)) : tomb4;
        for (uint32_t base = 0; base < deg; base += 4u * lanes) {
            const uint32_t kn = k + 4u * lanes;
            const uint4 qn = kn < deg ? __ldg(reinterpret_cast<const uint4 *>(rp + kn)) : tomb4;
            q.x = view.vid(q.x);
            q.y = view.vid(q.y);
            q.z = view.vid(q.z);
            q.w = view.vid(q.w);
            cnt.hits += edge4(op, q, k, deg, x, payload);
            q = qn;
            k = kn;
        }
    } else {
        for (uint32_t base = 0; base < deg; base += lanes) {
            const uint32_t k = base + t;
            const bool valid = k < deg;
            const uint32_t y = valid ? view.vid(__ldg(rp + k)) : 0u;
            cnt.hits += op.edge(valid && y != kTomb, x, payload, y);
        }
    }
}

// Rank of the calling thread in a block's share of a work list, dealt out
// warp by warp: rank k sits in warp k mod (TPB/32), lane k / (TPB/32).  A
// round often hands a block only a few items (a few dozen at most); with the
// plain rank (= threadIdx.x) they would all land in warp 0, which would then
// serve their rows one after another while the other warps idle.  Dealt
// out, the first TPB/32 items go to different warps and their chains of
// dependent row and state reads run side by side.
template <int TPB>
__device__ __forceinline__ uint32_t spread_rank() {
    return (threadIdx.x & 31u) * static_cast<uint32_t>(TPB / 32) + (threadIdx.x >> 5);
}

// Op must provide: __device__ bool edge(bool valid, uint32_t x, P payload, uint32_t y) const;
// returning true when the edge changed state.
// edge() is called by all 32 lanes of a warp together (valid=false on padding lanes).
template <int TPB, class Op, class P>
__device__ __forceinline__ void expand_rows(const AdjView &view, bool has, uint32_t x, P payload,
                                            uint64_t off, uint32_t deg, const Op &op, ExpandSmem<TPB, P> &sm,
                                            ExpandCounters &cnt, const Defer &defer = Defer{nullptr, nullptr, 0, 0}) {
    const uint32_t lane = lane_id();
    const uint32_t warp = threadIdx.x >> 5;
    if (has) {
        cnt.rows += 1;
        cnt.edges += deg;
        if (view.cached(off)) cnt.edges_cached += deg;
    }
    if (has && defer.rows && deg >= defer.split) {
        const uint32_t i = atomicAdd(defer.count, 1u);
        if (i < defer.cap) {
            defer.rows[i] = BigRow{off, static_cast<unsigned long long>(payload), x, deg};
            has = false;
        }
    }

    // Tier 1: block-wide rows.  Rows larger than one segment are resolved
    // per element (view.at), everything else is read from one base pointer.
    bool big = has && deg >= static_cast<uint32_t>(TPB);
    while (__syncthreads_or(big)) {
        if (big) sm.owner = threadIdx.x;
        __syncthreads();
        if (sm.owner == threadIdx.x) {
            sm.b_x = x;
            sm.b_payload = payload;
            sm.b_deg = deg;
            sm.b_off = off;
            big = false;
        }
        __syncthreads();
        const uint32_t bx = sm.b_x, bdeg = sm.b_deg;
        const P bp = sm.b_payload;
        const uint64_t boff = sm.b_off;
        if (bdeg <= kSegEdges) {
            sweep_row<TPB>(view, view.at(boff), bdeg, threadIdx.x, bx, bp, op, cnt);
        } else {
            for (uint32_t base = 0; base < bdeg; base += TPB) {
                const uint32_t k = base + threadIdx.x;
                const bool valid = k < bdeg;
                const uint32_t y = valid ? view.vid(__ldg(view.at(boff + k))) : 0u;
                cnt.hits += op.edge(valid && y != kTomb, bx, bp, y);
            }
        }
        __syncthreads();
    }

    // Tier 2: warp-wide rows (32 <= deg < TPB, always inside one segment).
    bool med = has && deg >= 32u && deg < static_cast<uint32_t>(TPB);
    uint32_t mmask;
    while ((mmask = __ballot_sync(kFull, med)) != 0u) {
        const uint32_t leader = __ffs(mmask) - 1;
        const uint32_t wx = __shfl_sync(kFull, x, leader);
        const P wp = __shfl_sync(kFull, payload, leader);
        const uint32_t wdeg = __shfl_sync(kFull, deg, leader);
        const uint64_t woff = __shfl_sync(kFull, static_cast<unsigned long long>(off), leader);
        if (lane == leader) med = false;
        sweep_row<32u>(view, view.at(woff), wdeg, lane, wx, wp, op, cnt);
    }

    // Tier 3: small rows gathered through a warp scan.
    const uint32_t mydeg = (has && deg < 32u) ? deg : 0u;
    uint32_t incl = mydeg;
#pragma unroll
    for (uint32_t o = 1; o < 32u; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (total == 0) return;
    const uint32_t wb = warp * 32u;
    sm.f_scan[wb + lane] = incl - mydeg;
    sm.f_x[wb + lane] = x;
    sm.f_payload[wb + lane] = payload;
    sm.f_ptr[wb + lane] = mydeg ? view.at(off) : nullptr;
    __syncwarp();
    // Two entries per lane per step: both row reads, then (for ops with
    // peek) both state reads, are in flight together.
    for (uint32_t base = 0; base < total; base += 64u) {
        uint32_t ox[2], y[2];
        P pl[2];
        bool valid[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint32_t e = base + 32u * j + lane;
            valid[j] = e < total;
            ox[j] = 0;
            y[j] = 0;
            pl[j] = 0;
            if (valid[j]) {
                // Last lane whose exclusive prefix is <= e owns edge e.
                uint32_t lo = 0, hi = 32;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (sm.f_scan[wb + mid] <= e)
                        lo = mid;
                    else
                        hi = mid;
                }
                ox[j] = sm.f_x[wb + lo];
                pl[j] = sm.f_payload[wb + lo];
                y[j] = __ldg(sm.f_ptr[wb + lo] + (e - sm.f_scan[wb + lo]));
            }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            y[j] = valid[j] ? view.vid(y[j]) : 0u;
            valid[j] = valid[j] && y[j] != kTomb;
        }
        cnt.hits += edges_n<2>(op, valid, ox, pl, y);
    }
    __syncwarp();
}

// Expand the deferred rows: chunk g of the concatenated chunk sequence goes
// to block g mod gridDim.x.  Every block walks the (short) list in the same
// order, so the assignment needs no coordination.  Block-uniform loops.
template <int TPB, class P = uint32_t, class Op>
__device__ __forceinline__ void expand_deferred(const AdjView &view, const BigRow *rows, uint32_t nrows,
                                                const Op &op, ExpandCounters &cnt) {
    const uint32_t grid = gridDim.x;
    uint64_t prefix = 0;
    for (uint32_t i = 0; i < nrows; ++i) {
        const BigRow r = rows[i];
        const uint64_t chunks = (r.deg + kSplitChunk - 1) / kSplitChunk;
        uint64_t g = prefix + (blockIdx.x + grid - static_cast<uint32_t>(prefix % grid)) % grid;
        for (; g < prefix + chunks; g += grid) {
            // A chunk (1024 entries, a multiple of 4) never straddles a
            // segment boundary: one pointer serves it.
            const uint32_t base = static_cast<uint32_t>(g - prefix) * kSplitChunk;
            const uint32_t len = min(kSplitChunk, r.deg - base);
            sweep_row<TPB>(view, view.at(r.off + base), len, threadIdx.x, r.x, static_cast<P>(r.payload), op, cnt);
        }
        prefix += chunks;
    }
}

}  // namespace cig
