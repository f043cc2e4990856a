// pr.cuh - incremental PageRank by signed residual push.
//
// Same fixed point as the reference (samples/hybrid_pr/README.md: x[v] =
// 0.15 + 0.85 * sum x[u]/outdeg(u), parallel edges counted, dangling vertices
// send nothing) and the same residual protocol as include/framework/
// pr_residual.cuh:16-188: a vertex whose |residual| exceeds epsilon is
// consumed into its rank and pushes 0.85*r/deg to its out-neighbours; a batch
// first withdraws the old contributions of every touched source over its old
// row, mutates the topology, then re-adds them over the new row.
//
// Differences: one persistent cooperative kernel runs consume and scatter
// rounds with grid barriers (no host count read per round); the rank is
// FP32 with a per-vertex Kahan compensation term (or FP64 throughout); the
// batch reports the FP64 L1 norm of the residual.
//
// FP32 residuals lose precision where many contributions pile up between two
// consumptions: a vertex with in-degree k takes up to k atomic adds per round,
// and the rounding of each (half an ulp of the running sum) adds up to about
// 6e-8 * sqrt(k) of its residual.  So in FP32 mode vertices whose in-degree
// was at least kPrHubInDeg at load keep their residual in an FP64 slot;
// everything else stays FP32.  The hub set is a bitmap (n/8 bytes) with a
// per-word prefix count (slot = prefix + rank in the word), small enough to
// stay in L2, since every scattered edge looks its destination up.
#pragma once

#include "common.cuh"
#include "expand.cuh"

namespace cig {

constexpr float kAlphaF = 0.85f;
constexpr double kAlphaD = 0.85;

constexpr uint32_t kPrHubInDeg = 256;

template <class T>
struct PrArrays {
    T *rank;
    T *res;
    const uint32_t *hub_bits;    // FP32 mode: bit v set when v has an FP64 residual slot
    const uint32_t *hub_prefix;  // slots before word w of hub_bits
    double *res_hub;
    float *comp;       // Kahan compensation of rank (FP32 mode only)
    uint32_t *queued;
    uint32_t *q0;
    uint32_t *q1;
    uint32_t *cnt;     // 3 round counters
    T *contrib;        // per queued item: alpha * r / deg (or 0)
    uint32_t *final_round;
    uint32_t cap;
};

template <class T>
__device__ __forceinline__ T pr_abs(T x) { return x < T(0) ? -x : x; }

template <class T>
__device__ __forceinline__ bool pr_finite(T x) { return isfinite(x); }

template <class T>
__device__ __forceinline__ int32_t hub_slot(const PrArrays<T> &a, uint32_t v) {
    if (sizeof(T) != 4 || !a.hub_bits) return -1;
    const uint32_t w = __ldg(a.hub_bits + (v >> 5));
    const uint32_t b = 1u << (v & 31u);
    if (!(w & b)) return -1;
    return static_cast<int32_t>(__ldg(a.hub_prefix + (v >> 5)) + __popc(w & (b - 1u)));
}

template <class T>
__device__ __forceinline__ T res_get(const PrArrays<T> &a, uint32_t v) {
    const int32_t h = hub_slot(a, v);
    return h >= 0 ? static_cast<T>(__ldcg(a.res_hub + h)) : __ldcg(a.res + v);
}

template <class T>
__device__ __forceinline__ void res_set(const PrArrays<T> &a, uint32_t v, double x) {
    const int32_t h = hub_slot(a, v);
    if (h >= 0)
        a.res_hub[h] = x;
    else
        a.res[v] = static_cast<T>(x);
}

// Threshold tests are made in the precision the residual is stored in, so
// that "crossed epsilon" (queue the vertex) and "above epsilon" (consume it)
// always agree; a residual left above epsilon but unqueued would never be
// consumed again.

// Atomic add of c; true when |res| went from <= eps to > eps.
template <class T>
__device__ __forceinline__ bool res_add_crossed(const PrArrays<T> &a, uint32_t v, T c, T eps, bool &finite) {
    const int32_t h = hub_slot(a, v);
    if (h >= 0) {
        const double old = atomicAdd(a.res_hub + h, static_cast<double>(c));
        const double nv = old + static_cast<double>(c);
        const double e = static_cast<double>(eps);
        finite = isfinite(nv);
        return fabs(old) <= e && fabs(nv) > e;
    }
    const T old = atomicAdd(a.res + v, c);
    const T nv = old + c;
    finite = pr_finite(nv);
    return pr_abs(old) <= eps && pr_abs(nv) > eps;
}

// Consume: if |res| > eps, return true with `taken` = the whole residual
// (FP64 slots keep their full value) and clear it.
template <class T>
__device__ __forceinline__ bool res_take(const PrArrays<T> &a, uint32_t v, T eps, double &taken, bool &finite) {
    const int32_t h = hub_slot(a, v);
    if (h >= 0) {
        const double r = __ldcg(a.res_hub + h);
        finite = isfinite(r);
        if (!(fabs(r) > static_cast<double>(eps))) return false;
        taken = r;
        a.res_hub[h] = 0.0;
        return true;
    }
    const T r = __ldcg(a.res + v);
    finite = pr_finite(r);
    if (!(pr_abs(r) > eps)) return false;
    taken = static_cast<double>(r);
    a.res[v] = T(0);
    return true;
}

template <class T>
__device__ __forceinline__ T rank_value(const PrArrays<T> &a, uint32_t v) {
    if (sizeof(T) == 4)
        return static_cast<T>(static_cast<double>(__ldcg(a.rank + v)) - static_cast<double>(__ldcg(a.comp + v)));
    return __ldcg(a.rank + v);
}

template <class T>
__device__ __forceinline__ void rank_add(const PrArrays<T> &a, uint32_t v, T r) {
    if (sizeof(T) == 4) {
        // Kahan summation: comp holds the negated low-order bits lost so far.
        const float y = static_cast<float>(r) - __ldcg(a.comp + v);
        const float s = static_cast<float>(__ldcg(a.rank + v));
        const float t = __fadd_rn(s, y);
        a.comp[v] = __fsub_rn(__fsub_rn(t, s), y);
        a.rank[v] = static_cast<T>(t);
    } else {
        a.rank[v] = __ldcg(a.rank + v) + r;
    }
}

// Frontier::Add (pr_residual.cuh:16-31): add to the residual and queue the
// vertex once when its magnitude crosses epsilon.
template <class T>
struct PrPushOp {
    PrArrays<T> a;
    uint32_t *queued;
    const T *contrib;
    T eps;
    uint32_t *q_out;
    uint32_t *q_cnt;
    uint32_t cap;
    Status *st;

    __device__ __forceinline__ bool edge(bool valid, uint32_t, uint32_t item, uint32_t y) const {
        bool want = false;
        if (valid) {
            bool finite = true;
            if (res_add_crossed(a, y, contrib[item], eps, finite) && __ldcg(queued + y) == 0u)
                want = atomicCAS(queued + y, 0u, 1u) == 0u;
            if (!finite) set_error(st, kErrNonFinite, y);
        }
        warp_enqueue(want, y, q_out, q_cnt, cap, st);
        return valid;
    }
};

template <class T>
__global__ void pr_init(PrArrays<T> a, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        a.rank[v] = T(0);
        res_set(a, v, 0.15);
        if (a.comp) a.comp[v] = 0.f;
        a.queued[v] = 1u;
        a.q0[v] = v;
    }
}

constexpr int kTpbPr = 256;

// Persistent converge loop (Runtime::Converge, pr_residual.cuh:171-187):
// each round consumes the queued residuals (Consume, :54-71), then scatters
// them (Scatter, :74-100); the queue of round r is q[r&1] with cnt[r%3].
// On exit `final_round` holds the round whose queue is still pending.
template <class T>
__global__ void __launch_bounds__(kTpbPr) pr_converge(AdjView fwd, PrArrays<T> a, T eps, uint32_t max_rounds,
                                                      uint32_t *seg_hot, Status *st) {
    __shared__ ExpandSmem<kTpbPr> sm;
    ExpandCounters cnt;
    uint32_t r = 0;
    for (;; ++r) {
        const uint32_t n_in = ld_volatile(a.cnt + (r % 3));
        if (n_in == 0 || r >= max_rounds) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) a.cnt[(r + 2) % 3] = 0;
        const uint32_t *in = (r & 1) ? a.q1 : a.q0;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_in; i += gridDim.x * blockDim.x) {
            const uint32_t v = __ldcg(in + i);
            a.queued[v] = 0u;
            T c = T(0);
            double r64 = 0.0;
            bool finite = true;
            if (res_take(a, v, eps, r64, finite)) {
                // An FP64 residual enters an FP32 rank as two compensated adds
                // (its float part and the rest), so nothing of it is lost.
                const T hi = static_cast<T>(r64);
                rank_add(a, v, hi);
                if (sizeof(T) == 4) {
                    const T lo = static_cast<T>(r64 - static_cast<double>(hi));
                    if (lo != T(0)) rank_add(a, v, lo);
                }
                const uint32_t deg = rd_live(fwd.desc[v]);  // out-degree: live entries only
                if (deg) c = static_cast<T>(kAlphaD * r64 / static_cast<double>(deg));
            }
            if (!finite) set_error(st, kErrNonFinite, v);
            a.contrib[i] = c;
        }
        if (!grid_barrier(st)) break;
        PrPushOp<T> op{a, a.queued, a.contrib, eps, (r & 1) ? a.q0 : a.q1, a.cnt + ((r + 1) % 3), a.cap, st};
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpbPr) {
            const uint32_t i = base + spread_rank<kTpbPr>() * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t v = 0, deg = 0;
            uint64_t off = 0;
            if (has) {
                v = __ldcg(in + i);
                const RowDesc d = fwd.desc[v];
                deg = d.len;
                off = d.off;
                has = deg > 0 && __ldcg(a.contrib + i) != T(0);
                if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), deg);
            }
            expand_rows<kTpbPr>(fwd, has, v, i, off, deg, op, sm, cnt);
        }
        if (!grid_barrier(st)) break;
    }
    flush_counters(st, cnt, kCntPr);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.final_round = r;
        atomicAdd(&st->counters[kCntPrRounds], static_cast<unsigned long long>(r));
    }
}

// Move the pending queue of round `final_round` to (q0, cnt[0]) so that the
// next batch's amendments append to it (Runtime::BeginBatch, :140-156).
template <class T>
__global__ void pr_normalize_frontier(PrArrays<T> a) {
    const uint32_t r = *a.final_round;
    const uint32_t n = ld_volatile(a.cnt + (r % 3));
    const uint32_t *src = (r & 1) ? a.q1 : a.q0;
    if (src != a.q0)
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a.q0[i] = src[i];
}

template <class T>
__global__ void pr_set_counts(PrArrays<T> a) {
    const uint32_t r = *a.final_round;
    const uint32_t n = a.cnt[r % 3];
    a.cnt[0] = n;
    a.cnt[1] = 0;
    a.cnt[2] = 0;
    *a.final_round = 0;
}

// Unique touched sources of a batch (deletion and addition sources).
__global__ void collect_touched(const uint32_t *du, uint32_t nd, const uint32_t *au, uint32_t na, uint32_t n,
                                uint32_t *stamp, uint32_t epoch, uint32_t *list, uint32_t *count, uint32_t cap,
                                Status *st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = nd + na;
    bool want = false;
    uint32_t u = 0;
    if (i < total) {
        u = i < nd ? du[i] : au[i - nd];
        if (u < n && __ldcg(stamp + u) != epoch) want = atomicExch(stamp + u, epoch) != epoch;
    }
    if (__any_sync(kFull, i < total)) warp_enqueue(want, u, list, count, cap, st);
}

// contrib[i] = sign * alpha * rank[s] / deg(s) for every touched source
// (CombineValueBufferAmend, samples/hybrid_pr/hybrid_pr.cu:77-83).
template <class T>
__global__ void pr_amend_contrib(const RowDesc *desc, PrArrays<T> a, const uint32_t *list, const uint32_t *count,
                                 T sign, T *contrib) {
    const uint32_t n = *count;
    const T alpha = sizeof(T) == 4 ? T(kAlphaF) : T(kAlphaD);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = list[i];
        const uint32_t deg = rd_live(desc[s]);
        contrib[i] = deg ? sign * alpha * rank_value(a, s) / static_cast<T>(deg) : T(0);
    }
}

template <class T>
__global__ void __launch_bounds__(kTpbPr) pr_amend_scatter(AdjView fwd, PrArrays<T> a, const uint32_t *list,
                                                           const uint32_t *count, const T *contrib, T eps,
                                                           Status *st) {
    __shared__ ExpandSmem<kTpbPr> sm;
    ExpandCounters cnt;
    const uint32_t n = *count;
    PrPushOp<T> op{a, a.queued, contrib, eps, a.q0, a.cnt, a.cap, st};
    for (uint32_t base = 0; base < n; base += gridDim.x * kTpbPr) {
        const uint32_t i = base + spread_rank<kTpbPr>() * gridDim.x + blockIdx.x;
        bool has = i < n;
        uint32_t s = 0, deg = 0;
        uint64_t off = 0;
        if (has) {
            s = list[i];
            const RowDesc d = fwd.desc[s];
            deg = d.len;
            off = d.off;
            has = deg > 0 && contrib[i] != T(0);
        }
        expand_rows<kTpbPr>(fwd, has, s, i, off, deg, op, sm, cnt);
    }
    flush_counters(st, cnt, kCntPr);
}

// FP32 mode: a batch's amend (-old contributions over the old rows, +new
// over the new rows) accumulates per vertex in FP64 and the net change is
// rounded into the FP32 residual once (pr_amend_fold).  Added straight into
// FP32 residuals, the two large, mostly cancelling contributions of a hub
// source leave a rounding residue of ~1e-7 of the contribution behind, which
// then converges into the ranks as a real error.
template <class T>
__global__ void pr_amend_contrib64(const RowDesc *desc, PrArrays<T> a, const uint32_t *list, const uint32_t *count,
                                   double sign, double *contrib) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = list[i];
        const uint32_t deg = rd_live(desc[s]);
        contrib[i] = deg ? sign * kAlphaD * static_cast<double>(rank_value(a, s)) / static_cast<double>(deg) : 0.0;
    }
}

struct PrAmendOp {
    double *acc;
    const double *contrib;
    __device__ __forceinline__ bool edge(bool valid, uint32_t, uint32_t item, uint32_t y) const {
        if (valid) atomicAdd(acc + y, contrib[item]);
        return valid;
    }
};

template <class T>
__global__ void __launch_bounds__(kTpbPr) pr_amend_scatter64(AdjView fwd, const uint32_t *list, const uint32_t *count,
                                                             const double *contrib, double *acc, Status *st) {
    __shared__ ExpandSmem<kTpbPr> sm;
    ExpandCounters cnt;
    const uint32_t n = *count;
    const PrAmendOp op{acc, contrib};
    for (uint32_t base = 0; base < n; base += gridDim.x * kTpbPr) {
        const uint32_t i = base + spread_rank<kTpbPr>() * gridDim.x + blockIdx.x;
        bool has = i < n;
        uint32_t s = 0, deg = 0;
        uint64_t off = 0;
        if (has) {
            s = list[i];
            const RowDesc d = fwd.desc[s];
            deg = d.len;
            off = d.off;
            has = deg > 0 && contrib[i] != 0.0;
        }
        expand_rows<kTpbPr>(fwd, has, s, i, off, deg, op, sm, cnt);
    }
    flush_counters(st, cnt, kCntPr);
}

// Round the accumulated amend into the residuals and queue the vertices
// whose residual crossed epsilon (Frontier::Add, pr_residual.cuh:16-31).
template <class T>
__global__ void pr_amend_fold(PrArrays<T> a, double *acc, uint32_t n, T eps, Status *st) {
    const uint32_t rounded = (n + 31u) & ~31u;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < rounded; v += gridDim.x * blockDim.x) {
        bool want = false;
        if (v < n) {
            const double d = acc[v];
            if (d != 0.0) {
                acc[v] = 0.0;
                // one thread per vertex: a plain add, crossing tested as in res_add_crossed
                const int32_t h = hub_slot(a, v);
                bool crossed, finite;
                if (h >= 0) {
                    const double old = a.res_hub[h], nv = old + d, e = static_cast<double>(eps);
                    a.res_hub[h] = nv;
                    finite = isfinite(nv);
                    crossed = fabs(old) <= e && fabs(nv) > e;
                } else {
                    const T old = a.res[v];
                    const T nv = static_cast<T>(static_cast<double>(old) + d);
                    a.res[v] = nv;
                    finite = pr_finite(nv);
                    crossed = pr_abs(old) <= eps && pr_abs(nv) > eps;
                }
                if (!finite) set_error(st, kErrNonFinite, v);
                if (crossed && a.queued[v] == 0u) {
                    a.queued[v] = 1u;
                    want = true;
                }
            }
        }
        warp_enqueue(want, v, a.q0, a.cnt, a.cap, st);
    }
}

// FP64 L1 norm of the residual.
template <class T>
__global__ void pr_residual_l1(PrArrays<T> a, uint32_t n, double *out) {
    double acc = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int32_t h = hub_slot(a, v);
        acc += fabs(h >= 0 ? a.res_hub[h] : static_cast<double>(a.res[v]));
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane_id() == 0 && acc != 0.0) atomicAdd(out, acc);
}

template <class T>
__global__ void pr_export(PrArrays<T> a, uint32_t n, float *rank, float *res, double *rank64, double *res64) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const T x = rank_value(a, v);
        if (rank) rank[v] = static_cast<float>(x);
        if (res) res[v] = static_cast<float>(res_get(a, v));
        if (rank64) rank64[v] = static_cast<double>(x);
        if (res64) res64[v] = static_cast<double>(res_get(a, v));
    }
}

}  // namespace cig
