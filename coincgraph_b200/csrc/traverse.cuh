// traverse.cuh - incremental BFS / SSSP / CC kernels.
//
// Vertex state is one 64-bit word per vertex: (value << 32) | parent, where
// value is the BFS depth, SSSP distance or CC label and parent the in-
// neighbour the value came from.  atomicMin on the packed word updates value
// and parent together, so a parent is always a witness of its value and ties
// resolve to the smallest parent id.  The reference keeps value, buffer and
// parent in three arrays and repairs parents with a CAS loop
// (samples/hybrid_sssp/hybrid_sssp.cu:110-127); the results it guarantees
// (unique depths, distances and labels) are the same.
//
// Per batch (reference flow: include/framework/framework.cuh:2752-2894 for
// deletions, :2139-2348 for insertions):
//   deletion:  seed_deletions -> inval_closure -> reset_affected -> pull_repair
//              -> enqueue_affected -> push_closure
//   insertion: seed_insertions -> push_closure
#pragma once

#include "common.cuh"
#include "expand.cuh"

namespace cig {

constexpr int kTpb = 256;

// Frontier for the push closure: ping-pong queues and three round counters
// (round r reads cnt[r%3], appends to cnt[(r+1)%3] and clears cnt[(r+2)%3]).
struct Frontier {
    uint32_t *q0;
    uint32_t *q1;
    uint32_t *cnt;  // 3 counters
    uint32_t cap;
};

// Tag space for per-round queue de-duplication; advanced on the device.
struct TagState {
    uint32_t next_tag;
    uint32_t pad;
};

// ---------------------------------------------------------------- ops

// Relax x -> y with the value of x (push).  CombineValueBuffer +
// AccumulateBuffer of the samples (hybrid_sssp.cu:84-127, hybrid_cc.cu:
// 87-127): improve y, and queue it once per round if its value decreased.
template <int A>
struct PushOp {
    uint32_t ccs;  // CC depth bits (Status::cc_shift)
    unsigned long long *state;
    uint32_t *qstamp;
    uint32_t tag;
    uint32_t *q_out;
    uint32_t *q_count;
    uint32_t q_cap;
    Status *st;
    const RowDesc *desc;  // rows of the queued vertices: prefetched into L2 for the next hop

    __device__ __forceinline__ unsigned long long peek(uint32_t y) const { return __ldcg(state + y); }
    __device__ __forceinline__ bool edge_peeked(bool valid, uint32_t x, uint32_t dx, uint32_t y,
                                                unsigned long long sy) const {
        bool want = false, improved = false;
        if (valid) {
            const uint32_t nd = relax_value<A>(dx, x, y, ccs);
            const unsigned long long cand = pack(nd, x);
            if (cand < sy) {
                const unsigned long long old = atomicMin(state + y, cand);
                improved = nd < val_of(old);
                if (improved) want = atomicExch(qstamp + y, tag) != tag;
            }
        }
        if (want) prefetch_l2(desc + y);
        warp_enqueue(want, y, q_out, q_count, q_cap, st);
        return improved;
    }
    __device__ __forceinline__ bool edge(bool valid, uint32_t x, uint32_t dx, uint32_t y) const {
        return edge_peeked(valid, x, dx, y, valid ? peek(y) : 0ull);
    }
    static constexpr bool kMulti = true;
    template <int N>
    __device__ __forceinline__ uint32_t edges(const bool (&v)[N], const uint32_t (&x)[N], const uint32_t (&dx)[N],
                                              const uint32_t (&y)[N], const unsigned long long (&sy)[N]) const {
        unsigned long long cand[N], old[N];
        bool want[N];
        uint32_t hits = 0;
#pragma unroll
        for (int j = 0; j < N; ++j) cand[j] = pack(relax_value<A>(dx[j], x[j], y[j], ccs), x[j]);
#pragma unroll
        for (int j = 0; j < N; ++j) old[j] = (v[j] && cand[j] < sy[j]) ? atomicMin(state + y[j], cand[j]) : 0ull;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const bool improved = v[j] && cand[j] < sy[j] && val_of(cand[j]) < val_of(old[j]);
            hits += improved ? 1u : 0u;
            want[j] = improved && atomicExch(qstamp + y[j], tag) != tag;
        }
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (want[j]) prefetch_l2(desc + y[j]);
        warp_enqueue_n<N>(want, y, q_out, q_count, q_cap, st);
        return hits;
    }
};

// Deletion dependency of an out-neighbour z (state word sz) of an
// invalidated vertex x (value px).  BFS/SSSP: z's parent is x
// (IsDeletionDependency, api.cuh:43-49; the packed state makes every parent
// tight).  CC: equal labels and z is not its own seed (hybrid_cc.cu:45-49),
// since equal-label cycles may hold parents that do not lead back to the
// seed.
template <int A>
__device__ __forceinline__ bool inval_dep(uint32_t ccs, uint32_t x, uint32_t px, uint32_t z, unsigned long long sz) {
    if (A == kCc) {
        const uint32_t vz = val_of(sz);
        return z != x &&
               (par_of(sz) == x || (cc_saturated(vz, ccs) && (vz >> ccs) == (px >> ccs) && (vz >> ccs) < z));
    }
    return par_of(sz) == x;
}

// Claims the out-neighbours of invalidated vertices that depend on them.
template <int A>
struct InvalOp {
    uint32_t ccs;
    unsigned long long *state;
    uint32_t *aff_stamp;
    uint32_t epoch;
    uint32_t *list;   // append base for this round
    uint32_t *count;  // this round's append counter
    uint32_t cap;
    Status *st;
    const RowDesc *desc;  // rows of the queued vertices: prefetched into L2 for the next hop

    __device__ __forceinline__ unsigned long long peek(uint32_t z) const { return __ldcg(state + z); }
    __device__ __forceinline__ bool edge(bool valid, uint32_t x, uint32_t px, uint32_t z) const {
        return edge_peeked(valid, x, px, z, valid ? peek(z) : 0ull);
    }
    __device__ __forceinline__ bool edge_peeked(bool valid, uint32_t x, uint32_t px, uint32_t z,
                                                unsigned long long sz) const {
        bool want = false;
        if (valid && inval_dep<A>(ccs, x, px, z, sz)) want = atomicExch(aff_stamp + z, epoch) != epoch;
        if (want) prefetch_l2(desc + z);
        warp_enqueue(want, z, list, count, cap, st);
        return want;
    }
    static constexpr bool kMulti = true;
    template <int N>
    __device__ __forceinline__ uint32_t edges(const bool (&v)[N], const uint32_t (&x)[N], const uint32_t (&px)[N],
                                              const uint32_t (&z)[N], const unsigned long long (&sz)[N]) const {
        bool want[N];
        uint32_t hits = 0;
#pragma unroll
        for (int j = 0; j < N; ++j) want[j] = v[j] && inval_dep<A>(ccs, x[j], px[j], z[j], sz[j]);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            want[j] = want[j] && atomicExch(aff_stamp + z[j], epoch) != epoch;
            hits += want[j] ? 1u : 0u;
        }
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (want[j]) prefetch_l2(desc + z[j]);
        warp_enqueue_n<N>(want, z, list, count, cap, st);
        return hits;
    }
};

// Pull over the in-row of an invalidated vertex v (edge u -> v).  Replaces
// GpuAffectedPullRelax (framework.cuh:137-204): candidates from vertices
// that kept their value; CC also takes the seed label of invalidated
// in-neighbours, which are valid reaching ids.
template <int A>
struct PullOp {
    uint32_t ccs;
    unsigned long long *state;
    const uint32_t *aff_stamp;
    uint32_t epoch;

    // Both words of u at once: bit 32 = u is invalidated, low half = u's value.
    __device__ __forceinline__ unsigned long long peek(uint32_t u) const {
        const uint32_t stamp = __ldcg(aff_stamp + u);
        const uint32_t du = val_of(__ldcg(state + u));
        return (stamp == epoch ? (1ull << 32) : 0ull) | du;
    }
    __device__ __forceinline__ bool edge_peeked(bool valid, uint32_t v, uint32_t, uint32_t u,
                                                unsigned long long w) const {
        if (!valid) return false;
        unsigned long long cand;
        if (w >> 32) {
            if (A != kCc) return false;
            cand = pack(cc_step(u << ccs, ccs), u);  // u restarts as its own seed
        } else {
            const uint32_t du = static_cast<uint32_t>(w);
            if (du == kInf) return false;
            cand = pack(relax_value<A>(du, u, v, ccs), u);
        }
        if (cand >= __ldcg(state + v)) return false;
        atomicMin(state + v, cand);
        return true;
    }
    __device__ __forceinline__ bool edge(bool valid, uint32_t v, uint32_t p, uint32_t u) const {
        return edge_peeked(valid, v, p, u, valid ? peek(u) : 0ull);
    }
};

// ---------------------------------------------------------------- kernels

// Persistent push closure (cooperative launch).  Replaces RunExactGpuClosure
// (framework.cuh:342-454) and the Start loop (:1151-1182): waves of relaxation
// until no vertex improves, with bounded grid barriers and a round bound.
// Rows of at least kSplitDeg entries met in a round go to `big` (three round
// counters, as for the frontier) and are expanded by the whole grid after a
// barrier; rounds without such rows keep a single barrier.
struct BigList {
    BigRow *rows;
    uint32_t *cnt;  // 3 counters
    uint32_t cap;
    uint32_t split;  // deferral threshold (row entries), tuned per handle
};

// Block-local sweeps.  After a block has relaxed its share of a round's
// frontier, the vertices it improved go to a queue in its shared memory, and
// the block expands them itself for up to `max_sweeps` more hops,
// synchronising with __syncthreads only (a vertex that is in the next
// round's frontier by the time a sweep reads it is left to that round); what
// is left (or does not fit) goes to the next round's frontier as usual.  On high-diameter graphs, whose rounds carry
// small frontiers and cost a chain of dependent memory accesses plus a grid
// barrier each, this covers several hops per grid round.  A vertex may then
// be expanded by two blocks in one round (a redundant relaxation); the
// label-correcting fixpoint, values and smallest-id parents, is unchanged.
constexpr uint32_t kLocalCap = 1024;
constexpr uint32_t kSweepItems = 4;  // invalidation sweeps: rounds of at most this many items per block

template <int A>
struct LocalPushOp {
    uint32_t ccs;
    unsigned long long *state;
    uint32_t *qstamp;
    uint32_t tag;       // membership of the next round's frontier
    uint32_t *q_out;    // next round's frontier (overflow)
    uint32_t *q_count;
    uint32_t q_cap;
    uint32_t *lq;       // shared-memory queue of this sweep's output
    uint32_t *lq_n;
    Status *st;
    const RowDesc *desc;  // rows of the queued vertices: prefetched into L2 for the next hop

    __device__ __forceinline__ unsigned long long peek(uint32_t y) const { return __ldcg(state + y); }
    __device__ __forceinline__ bool edge(bool valid, uint32_t x, uint32_t dx, uint32_t y) const {
        return edge_peeked(valid, x, dx, y, valid ? peek(y) : 0ull);
    }
    __device__ __forceinline__ bool edge_peeked(bool valid, uint32_t x, uint32_t dx, uint32_t y,
                                                unsigned long long sy) const {
        bool want = false, improved = false;
        if (valid) {
            const uint32_t nd = relax_value<A>(dx, x, y, ccs);
            const unsigned long long cand = pack(nd, x);
            if (cand < sy) {
                const unsigned long long old = atomicMin(state + y, cand);
                improved = nd < val_of(old);
                want = improved;  // a y already in the next frontier is skipped when the sweep reads it
            }
        }
        if (want) prefetch_l2(desc + y);
        const uint32_t mask = __ballot_sync(kFull, want);
        bool spill = false;
        if (mask) {
            const uint32_t lane = lane_id();
            const uint32_t leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(lq_n, __popc(mask));
            base = __shfl_sync(kFull, base, leader);
            if (want) {
                const uint32_t pos = base + __popc(mask & lanemask_lt());
                if (pos < kLocalCap)
                    lq[pos] = y;
                else
                    spill = atomicExch(qstamp + y, tag) != tag;
            }
        }
        warp_enqueue(spill, y, q_out, q_count, q_cap, st);
        return improved;
    }
    static constexpr bool kMulti = true;
    template <int N>
    __device__ __forceinline__ uint32_t edges(const bool (&v)[N], const uint32_t (&x)[N], const uint32_t (&dx)[N],
                                              const uint32_t (&y)[N], const unsigned long long (&sy)[N]) const {
        unsigned long long cand[N], old[N];
        bool want[N], spill[N];
        uint32_t hits = 0, c = 0;
#pragma unroll
        for (int j = 0; j < N; ++j) cand[j] = pack(relax_value<A>(dx[j], x[j], y[j], ccs), x[j]);
#pragma unroll
        for (int j = 0; j < N; ++j) old[j] = (v[j] && cand[j] < sy[j]) ? atomicMin(state + y[j], cand[j]) : 0ull;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            want[j] = v[j] && cand[j] < sy[j] && val_of(cand[j]) < val_of(old[j]);
            hits += want[j] ? 1u : 0u;
            c += want[j] ? 1u : 0u;
            spill[j] = false;
            if (want[j]) prefetch_l2(desc + y[j]);
        }
        if (__any_sync(kFull, c != 0u)) {
            const uint32_t lane = lane_id();
            uint32_t incl = c;
#pragma unroll
            for (uint32_t o = 1; o < 32u; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += t;
            }
            uint32_t base = 0;
            if (lane == 31) base = atomicAdd(lq_n, incl);
            base = __shfl_sync(kFull, base, 31);
            uint32_t pos = base + incl - c;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                if (want[j]) {
                    if (pos < kLocalCap)
                        lq[pos] = y[j];
                    else
                        spill[j] = atomicExch(qstamp + y[j], tag) != tag;
                    ++pos;
                }
            }
        }
        warp_enqueue_n<N>(spill, y, q_out, q_count, q_cap, st);
        return hits;
    }
};

template <int A>
__global__ void __launch_bounds__(kTpb, 4) push_closure(AdjView fwd, unsigned long long *state, uint32_t *qstamp,
                                                     TagState *tags, Frontier fr, BigList big, uint32_t max_rounds,
                                                     uint32_t max_sweeps, uint32_t *seg_hot, Status *st) {
    __shared__ ExpandSmem<kTpb> sm;
    __shared__ uint32_t lq[2][kLocalCap];
    __shared__ uint32_t lq_n[2];
    ExpandCounters cnt;
    // next_tag itself belongs to the seeds queued before this launch.
    const uint32_t tag0 = tags->next_tag + 1;
    const uint32_t sweeps = max_sweeps;
    const uint32_t ccs = (A == kCc) ? st->cc_shift : 0u;
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
        uint32_t *out_cnt = fr.cnt + ((r + 1) % 3);
        PushOp<A> op{ccs, state, qstamp, tag0 + r, out, out_cnt, fr.cap, st, fwd.desc};
        const Defer df{big.rows, big.cnt + (r % 3), big.cap, big.split};
        if (sweeps) {
            if (threadIdx.x == 0) lq_n[0] = 0;
            __syncthreads();
        }
        // Item i goes to block i mod gridDim.x, so small frontiers still
        // spread over the whole grid, and within the block to the warps in
        // turn (spread_rank).
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpb) {
            const uint32_t i = base + spread_rank<kTpb>() * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t x = 0, dx = 0, deg = 0;
            uint64_t off = 0;
            if (has) {
                x = __ldcg(in + i);
                dx = val_of(__ldcg(state + x));
                const RowDesc d = fwd.desc[x];
                deg = d.len;
                off = d.off;
                has = dx != kInf && deg > 0;
                if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), deg);
            }
            if (sweeps)
                expand_rows<kTpb>(fwd, has, x, dx, off, deg,
                                  LocalPushOp<A>{ccs, state, qstamp, tag0 + r, out, out_cnt, fr.cap, lq[0], &lq_n[0],
                                                 st, fwd.desc},
                                  sm, cnt, df);
            else
                expand_rows<kTpb>(fwd, has, x, dx, off, deg, op, sm, cnt, df);
        }
        if (sweeps) {
            uint32_t cur = 0;
            for (uint32_t sw = 0; sw < sweeps; ++sw) {
                __syncthreads();
                const uint32_t nl = min(lq_n[cur], kLocalCap);
                if (nl == 0) break;
                if (threadIdx.x == 0) lq_n[cur ^ 1u] = 0;
                __syncthreads();
                const LocalPushOp<A> lop{ccs, state, qstamp, tag0 + r, out, out_cnt, fr.cap, lq[cur ^ 1u],
                                         &lq_n[cur ^ 1u], st, fwd.desc};
                for (uint32_t base = 0; base < nl; base += kTpb) {
                    const uint32_t i = base + spread_rank<kTpb>();
                    bool has = i < nl;
                    uint32_t x = 0, dx = 0, deg = 0;
                    uint64_t off = 0;
                    if (has) {
                        x = lq[cur][i];
                        dx = val_of(__ldcg(state + x));
                        const bool queued = __ldcg(qstamp + x) == tag0 + r;  // the next round expands it
                        const RowDesc d = fwd.desc[x];
                        deg = d.len;
                        off = d.off;
                        has = dx != kInf && deg > 0 && !queued;
                        if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), deg);
                    }
                    expand_rows<kTpb>(fwd, has, x, dx, off, deg, lop, sm, cnt, df);
                }
                cur ^= 1u;
            }
            // What the last sweep queued joins the next round's frontier.
            __syncthreads();
            const uint32_t nl = min(lq_n[cur], kLocalCap);
            for (uint32_t b0 = 0; b0 < nl; b0 += kTpb) {
                const uint32_t i = b0 + threadIdx.x;
                const uint32_t y = i < nl ? lq[cur][i] : 0u;
                const bool want = i < nl && atomicExch(qstamp + y, tag0 + r) != tag0 + r;
                warp_enqueue(want, y, out, out_cnt, fr.cap, st);
            }
        }
        if (!grid_barrier(st)) break;
        const uint32_t nbig = min(ld_volatile(big.cnt + (r % 3)), big.cap);
        if (nbig) {
            expand_deferred<kTpb>(fwd, big.rows, nbig, op, cnt);
            if (!grid_barrier(st)) break;
        }
    }
    flush_counters(st, cnt, kCntPush);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&st->counters[kCntRounds], static_cast<unsigned long long>(r));
        tags->next_tag = tag0 + r + 1;
    }
}

// Persistent invalidation closure over the affected list.  Round r processes
// list[lo, hi) and appends at list[hi + ...] counted by cnt[(r+1)%3].
// Replaces RunSyncPushDDB_del rounds (framework.cuh:2830-2853).
// Local sweeps of the invalidation closure: a vertex a block claims goes to
// the block's shared-memory queue and is expanded by the block at once, for
// up to `max_sweeps` hops (then appended to `done`); what is left after the
// last sweep, or does not fit, goes to the next round's list as usual.
// Every claimed vertex is expanded once and ends in exactly one of the two
// lists; `done` is appended to the list when the closure ends, so the
// affected list is the same set.
template <int A>
struct LocalInvalOp {
    uint32_t ccs;
    unsigned long long *state;
    uint32_t *aff_stamp;
    uint32_t epoch;
    uint32_t *list;
    uint32_t *count;
    uint32_t cap;
    uint32_t *lq;
    uint32_t *lq_n;
    Status *st;
    const RowDesc *desc;  // rows of the queued vertices: prefetched into L2 for the next hop

    __device__ __forceinline__ unsigned long long peek(uint32_t z) const { return __ldcg(state + z); }
    __device__ __forceinline__ bool edge(bool valid, uint32_t x, uint32_t px, uint32_t z) const {
        return edge_peeked(valid, x, px, z, valid ? peek(z) : 0ull);
    }
    __device__ __forceinline__ bool edge_peeked(bool valid, uint32_t x, uint32_t px, uint32_t z,
                                                unsigned long long sz) const {
        bool want = false;
        if (valid && inval_dep<A>(ccs, x, px, z, sz)) want = atomicExch(aff_stamp + z, epoch) != epoch;
        if (want) prefetch_l2(desc + z);
        const uint32_t mask = __ballot_sync(kFull, want);
        bool spill = false;
        if (mask) {
            const uint32_t lane = lane_id();
            const uint32_t leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(lq_n, __popc(mask));
            base = __shfl_sync(kFull, base, leader);
            const uint32_t pos = base + __popc(mask & lanemask_lt());
            if (want) {
                if (pos < kLocalCap)
                    lq[pos] = z;
                else
                    spill = true;
            }
        }
        warp_enqueue(spill, z, list, count, cap, st);
        return want;
    }
    static constexpr bool kMulti = true;
    template <int N>
    __device__ __forceinline__ uint32_t edges(const bool (&v)[N], const uint32_t (&x)[N], const uint32_t (&px)[N],
                                              const uint32_t (&z)[N], const unsigned long long (&sz)[N]) const {
        bool want[N], spill[N];
        uint32_t hits = 0, c = 0;
#pragma unroll
        for (int j = 0; j < N; ++j) want[j] = v[j] && inval_dep<A>(ccs, x[j], px[j], z[j], sz[j]);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            want[j] = want[j] && atomicExch(aff_stamp + z[j], epoch) != epoch;
            hits += want[j] ? 1u : 0u;
            c += want[j] ? 1u : 0u;
            spill[j] = false;
            if (want[j]) prefetch_l2(desc + z[j]);
        }
        if (__any_sync(kFull, c != 0u)) {
            const uint32_t lane = lane_id();
            uint32_t incl = c;
#pragma unroll
            for (uint32_t o = 1; o < 32u; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += t;
            }
            uint32_t base = 0;
            if (lane == 31) base = atomicAdd(lq_n, incl);
            base = __shfl_sync(kFull, base, 31);
            uint32_t pos = base + incl - c;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                if (want[j]) {
                    if (pos < kLocalCap)
                        lq[pos] = z[j];
                    else
                        spill[j] = true;
                    ++pos;
                }
            }
        }
        warp_enqueue_n<N>(spill, z, list, count, cap, st);
        return hits;
    }
};

template <int A>
__global__ void __launch_bounds__(kTpb, 4) inval_closure(AdjView fwd, unsigned long long *state, uint32_t *aff_stamp,
                                                      const uint32_t *epoch_p, uint32_t *list, uint32_t *cnt3,
                                                      uint32_t cap, BigList big, uint32_t max_rounds,
                                                      uint32_t max_sweeps, uint32_t *done, uint32_t *done_cnt,
                                                      uint32_t *aff_total, uint32_t *seg_hot, Status *st) {
    __shared__ ExpandSmem<kTpb> sm;
    __shared__ uint32_t lq[2][kLocalCap];
    __shared__ uint32_t lq_n[2];
    ExpandCounters c;
    const uint32_t ccs = (A == kCc) ? st->cc_shift : 0u;
    const uint32_t epoch = *epoch_p;
    uint32_t lo = 0, hi = ld_volatile(cnt3 + 0);
    uint32_t r = 0;
    for (;; ++r) {
        if (hi == lo) break;
        if (r >= max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) set_error(st, kErrRounds, r);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            cnt3[(r + 2) % 3] = 0;
            big.cnt[(r + 2) % 3] = 0;
        }
        InvalOp<A> op{ccs, state, aff_stamp, epoch, list + hi, cnt3 + ((r + 1) % 3), cap > hi ? cap - hi : 0u, st,
                      fwd.desc};
        const Defer df{big.rows, big.cnt + (r % 3), big.cap, big.split};
        const uint32_t n_in = hi - lo;
        // Sweeps only for small frontiers (a few items per block): on R-MAT
        // the large invalidation rounds already fill the grid, and sweeps
        // left their work to the blocks that found it (2x slower there).
        const uint32_t sweeps = n_in <= kSweepItems * gridDim.x ? max_sweeps : 0u;
        if (sweeps) {
            if (threadIdx.x == 0) lq_n[0] = 0;
            __syncthreads();
        }
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpb) {
            const uint32_t i = base + spread_rank<kTpb>() * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t x = 0, px = 0, deg = 0;
            uint64_t off = 0;
            if (has) {
                x = __ldcg(list + lo + i);
                px = (A == kCc) ? val_of(__ldcg(state + x)) : x;
                const RowDesc d = fwd.desc[x];
                deg = d.len;
                off = d.off;
                has = deg > 0;
                if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), deg);
            }
            if (sweeps)
                expand_rows<kTpb>(fwd, has, x, px, off, deg,
                                  LocalInvalOp<A>{ccs, state, aff_stamp, epoch, op.list, op.count, op.cap, lq[0],
                                                  &lq_n[0], st, fwd.desc},
                                  sm, c, df);
            else
                expand_rows<kTpb>(fwd, has, x, px, off, deg, op, sm, c, df);
        }
        if (sweeps) {
            uint32_t cur = 0;
            for (uint32_t sw = 0; sw < sweeps; ++sw) {
                __syncthreads();
                const uint32_t nl = min(lq_n[cur], kLocalCap);
                if (nl == 0) break;
                if (threadIdx.x == 0) lq_n[cur ^ 1u] = 0;
                __syncthreads();
                const LocalInvalOp<A> lop{ccs, state, aff_stamp, epoch, op.list, op.count, op.cap, lq[cur ^ 1u],
                                          &lq_n[cur ^ 1u], st, fwd.desc};
                for (uint32_t base = 0; base < nl; base += kTpb) {
                    const uint32_t i = base + spread_rank<kTpb>();
                    bool has = i < nl;
                    uint32_t x = 0, px = 0, deg = 0;
                    uint64_t off = 0;
                    if (has) x = lq[cur][i];
                    warp_enqueue(has, x, done, done_cnt, cap, st);
                    if (has) {
                        px = (A == kCc) ? val_of(__ldcg(state + x)) : x;
                        const RowDesc d = fwd.desc[x];
                        deg = d.len;
                        off = d.off;
                        has = deg > 0;
                        if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), deg);
                    }
                    expand_rows<kTpb>(fwd, has, x, px, off, deg, lop, sm, c, df);
                }
                cur ^= 1u;
            }
            // What the last sweep claimed is expanded by the next round.
            __syncthreads();
            const uint32_t nl = min(lq_n[cur], kLocalCap);
            for (uint32_t b0 = 0; b0 < nl; b0 += kTpb) {
                const uint32_t i = b0 + threadIdx.x;
                warp_enqueue(i < nl, i < nl ? lq[cur][i] : 0u, op.list, op.count, op.cap, st);
            }
        }
        if (!grid_barrier(st)) break;
        const uint32_t nbig = min(ld_volatile(big.cnt + (r % 3)), big.cap);
        if (nbig) {
            expand_deferred<kTpb>(fwd, big.rows, nbig, op, c);
            if (!grid_barrier(st)) break;
        }
        lo = hi;
        hi = hi + ld_volatile(cnt3 + ((r + 1) % 3));
    }
    if (max_sweeps) {
        // The vertices expanded by local sweeps complete the affected list.
        // Every block left the loop after the same barrier, so `done` is final.
        const uint32_t nd = ld_volatile(done_cnt);
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nd && hi + i < cap; i += gridDim.x * blockDim.x)
            list[hi + i] = __ldcg(done + i);
        if (hi + nd > cap && blockIdx.x == 0 && threadIdx.x == 0) set_error(st, kErrQueue, hi + nd);
        hi += min(nd, cap - min(hi, cap));
    }
    flush_counters(st, c, kCntInval);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *aff_total = hi;
        atomicAdd(&st->counters[kCntRounds], static_cast<unsigned long long>(r));
        atomicAdd(&st->counters[kCntAffected], static_cast<unsigned long long>(hi));
    }
}

// Deletion seeds (reset_del_edges, include/framework/variants/driver.cuh:
// 371-411), evaluated on the values before the batch.
template <int A>
__global__ void seed_deletions(const uint32_t *du, const uint32_t *dv, uint32_t nd, uint32_t n,
                               const unsigned long long *state, uint32_t *aff_stamp, const uint32_t *epoch_p,
                               uint32_t *list, uint32_t *count, uint32_t cap, Status *st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t epoch = *epoch_p;
    bool want = false;
    uint32_t v = 0;
    if (i < nd) {
        const uint32_t u = du[i];
        v = dv[i];
        if (u < n && v < n) {
            const unsigned long long sv = __ldcg(state + v);
            bool dep;
            if (A == kCc) {
                const uint32_t ccs = st->cc_shift;
                const uint32_t lu = val_of(__ldcg(state + u)) >> ccs;
                const uint32_t vv = val_of(sv);
                dep = u != v && (par_of(sv) == u || (cc_saturated(vv, ccs) && lu == (vv >> ccs) && (vv >> ccs) < v));
            } else {
                dep = par_of(sv) == u && val_of(sv) != kInf;
            }
            if (dep && __ldcg(aff_stamp + v) != epoch) want = atomicExch(aff_stamp + v, epoch) != epoch;
        }
    }
    if (__any_sync(kFull, i < nd)) warp_enqueue(want, v, list, count, cap, st);
}

// Start of a deletion phase: advance the batch epoch (the "invalidated in
// this batch" marker of aff_stamp, kept on the device so that a captured
// batch graph needs no new arguments) and clear the counters of `counters`
// (32 words) whose bit is set in `mask`, in place of one memset each.
// Launched with 32 threads.
__global__ void phase_begin(uint32_t *epoch, uint32_t *counters, uint32_t mask) {
    if (threadIdx.x == 0) *epoch += 1u;
    if (threadIdx.x < 32u && ((mask >> threadIdx.x) & 1u)) counters[threadIdx.x] = 0u;
}

// value <- initial value for every invalidated vertex (reset_affected_values,
// driver.cuh:418-433): unreached for BFS/SSSP, its own id for CC.
template <int A>
__global__ void reset_affected(const uint32_t *list, const uint32_t *total, unsigned long long *state,
                               uint32_t ccs) {
    const uint32_t n = *total;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = list[i];
        state[v] = (A == kCc) ? pack(v << ccs, kInf) : kInf64;
    }
}

template <int A>
__global__ void __launch_bounds__(kTpb, 4) pull_repair(AdjView rev, unsigned long long *state, const uint32_t *aff_stamp,
                                                    const uint32_t *epoch_p, const uint32_t *list,
                                                    const uint32_t *total, BigList big, Status *st) {
    __shared__ ExpandSmem<kTpb> sm;
    ExpandCounters c;
    const uint32_t n = *total;
    PullOp<A> op{(A == kCc) ? st->cc_shift : 0u, state, aff_stamp, *epoch_p};
    const Defer df{big.rows, big.cnt, big.cap, big.split};
    for (uint32_t base = 0; base < n; base += gridDim.x * kTpb) {
        const uint32_t i = base + spread_rank<kTpb>() * gridDim.x + blockIdx.x;
        bool has = i < n;
        uint32_t v = 0, deg = 0;
        uint64_t off = 0;
        if (has) {
            v = list[i];
            const RowDesc d = rev.desc[v];
            deg = d.len;
            off = d.off;
            has = deg > 0;
        }
        expand_rows<kTpb>(rev, has, v, 0u, off, deg, op, sm, c, df);
    }
    flush_counters(st, c, kCntPull);
}

// The in-rows that pull_repair deferred, expanded by the whole grid.
template <int A>
__global__ void __launch_bounds__(kTpb) pull_deferred(AdjView rev, unsigned long long *state, const uint32_t *aff_stamp,
                                                      const uint32_t *epoch_p, BigList big, Status *st) {
    ExpandCounters c;
    PullOp<A> op{(A == kCc) ? st->cc_shift : 0u, state, aff_stamp, *epoch_p};
    expand_deferred<kTpb>(rev, big.rows, min(*big.cnt, big.cap), op, c);
    flush_counters(st, c, kCntPull);
}

// Queue every repaired vertex that has a value (all of them for CC).
template <int A>
__global__ void enqueue_affected(const uint32_t *list, const uint32_t *total, const unsigned long long *state,
                                 Frontier fr, Status *st) {
    const uint32_t n = *total;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (n + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += stride) {
        bool want = false;
        uint32_t v = 0;
        if (i < n) {
            v = list[i];
            want = (A == kCc) || val_of(__ldcg(state + v)) != kInf;
        }
        warp_enqueue(want, v, fr.q0, fr.cnt, fr.cap, st);
    }
}

// Insertion seeds (SeedAddedEdgeFrontier, framework.cuh:238-294): relax every
// inserted edge with the value of its source after the topology update.
template <int A>
__global__ void seed_insertions(const uint32_t *au, const uint32_t *av, uint32_t na, uint32_t n,
                                unsigned long long *state, uint32_t *qstamp, const TagState *tags, Frontier fr,
                                Status *st) {
    const uint32_t tag = tags->next_tag;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    uint32_t v = 0;
    if (i < na) {
        const uint32_t u = au[i];
        v = av[i];
        if (u < n && v < n) {
            const uint32_t du = val_of(__ldcg(state + u));
            if (du != kInf) {
                const uint32_t nd = relax_value<A>(du, u, v, (A == kCc) ? st->cc_shift : 0u);
                const unsigned long long cand = pack(nd, u);
                if (cand < __ldcg(state + v)) {
                    const unsigned long long old = atomicMin(state + v, cand);
                    if (nd < val_of(old)) want = atomicExch(qstamp + v, tag) != tag;
                }
            }
        }
    }
    if (__any_sync(kFull, i < na)) warp_enqueue(want, v, fr.q0, fr.cnt, fr.cap, st);
    if (want) atomicAdd(&st->counters[kCntSeeds], 1ull);
}

// Static-solve initialisation (InitGraph, framework.cuh:991-1041).
template <int A>
__global__ void init_state(unsigned long long *state, uint32_t n, uint32_t source, uint32_t ccs) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (A == kCc)
            state[v] = pack(v << ccs, kInf);
        else
            state[v] = (v == source) ? pack(0u, kInf) : kInf64;
    }
}

// CC starts from every vertex with out-edges.
__global__ void enqueue_all_nonempty(const RowDesc *desc, uint32_t n, Frontier fr, Status *st) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (n + 31u) & ~31u;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < rounded; v += stride) {
        const bool want = v < n && rd_live(desc[v]) > 0;
        warp_enqueue(want, v, fr.q0, fr.cnt, fr.cap, st);
    }
}

// `ccs` drops the CC depth bits (0 for the other algorithms).
__global__ void unpack_values(const unsigned long long *state, uint32_t n, uint32_t *values, uint32_t *parents,
                              uint32_t ccs) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const unsigned long long s = state[v];
        if (values) values[v] = val_of(s) >> ccs;
        if (parents) parents[v] = par_of(s);
    }
}

// Order-independent 64-bit digest of the values: sum over reached vertices
// of a SplitMix64 hash of (vertex, value).  Lets a caller confirm a result
// with 8 bytes over the host link.
__device__ __forceinline__ unsigned long long digest_mix(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long value_term(uint32_t v, unsigned long long word, uint32_t ccs) {
    const uint32_t d = val_of(word) >> ccs;
    return d != kInf ? digest_mix((static_cast<unsigned long long>(v) << 32) | d) : 0ull;
}

// The sum is order-free, so the state is read two words per 16-byte load
// (the array starts 16-byte aligned) and each block adds its total with one
// atomic (one per warp queued ~10 k atomics on one address).
__global__ void value_digest(const unsigned long long *state, uint32_t n, unsigned long long *out, uint32_t ccs) {
    __shared__ unsigned long long part[32];
    unsigned long long acc = 0;
    const ulonglong2 *pairs = reinterpret_cast<const ulonglong2 *>(state);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n / 2; p += gridDim.x * blockDim.x) {
        const ulonglong2 w = pairs[p];
        acc += value_term(2 * p, w.x, ccs) + value_term(2 * p + 1, w.y, ccs);
    }
    if ((n & 1u) && blockIdx.x == 0 && threadIdx.x == 0) acc += value_term(n - 1, state[n - 1], ccs);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane_id() == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
        if (threadIdx.x == 0 && acc) atomicAdd(out, acc);
    }
}

}  // namespace cig
