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
#pragma once

#include "common.cuh"
#include "expand.cuh"

namespace cig {

constexpr float kAlphaF = 0.85f;
constexpr double kAlphaD = 0.85;

template <class T>
struct PrArrays {
    T *rank;
    T *res;
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
    T *res;
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
            const T c = contrib[item];
            const T old = atomicAdd(res + y, c);
            const T nv = old + c;
            if (!pr_finite(nv)) set_error(st, kErrNonFinite, y);
            if (pr_abs(old) <= eps && pr_abs(nv) > eps && __ldcg(queued + y) == 0u)
                want = atomicCAS(queued + y, 0u, 1u) == 0u;
        }
        warp_enqueue(want, y, q_out, q_cnt, cap, st);
        return valid;
    }
};

template <class T>
__global__ void pr_init(PrArrays<T> a, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        a.rank[v] = T(0);
        a.res[v] = T(0.15);
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
    const T alpha = sizeof(T) == 4 ? T(kAlphaF) : T(kAlphaD);
    uint32_t r = 0;
    for (;; ++r) {
        const uint32_t n_in = ld_volatile(a.cnt + (r % 3));
        if (n_in == 0 || r >= max_rounds) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) a.cnt[(r + 2) % 3] = 0;
        const uint32_t *in = (r & 1) ? a.q1 : a.q0;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_in; i += gridDim.x * blockDim.x) {
            const uint32_t v = __ldcg(in + i);
            a.queued[v] = 0u;
            const T rv = __ldcg(a.res + v);
            T c = T(0);
            if (!pr_finite(rv)) set_error(st, kErrNonFinite, v);
            if (pr_abs(rv) > eps) {
                rank_add(a, v, rv);
                a.res[v] = T(0);
                const uint32_t deg = rd_live(fwd.desc[v]);  // out-degree: live entries only
                if (deg) c = alpha * rv / static_cast<T>(deg);
            }
            a.contrib[i] = c;
        }
        if (!grid_barrier(st)) break;
        PrPushOp<T> op{a.res, a.queued, a.contrib, eps, (r & 1) ? a.q0 : a.q1, a.cnt + ((r + 1) % 3), a.cap, st};
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpbPr) {
            const uint32_t i = base + threadIdx.x * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t v = 0, deg = 0;
            uint64_t off = 0;
            if (has) {
                v = __ldcg(in + i);
                const RowDesc d = fwd.desc[v];
                deg = d.len;
                off = d.off;
                has = deg > 0 && __ldcg(a.contrib + i) != T(0);
                if (has && seg_hot) atomicAdd(seg_hot + (off >> kSegShift), 1u);
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
    PrPushOp<T> op{a.res, a.queued, contrib, eps, a.q0, a.cnt, a.cap, st};
    for (uint32_t base = 0; base < n; base += gridDim.x * kTpbPr) {
        const uint32_t i = base + threadIdx.x * gridDim.x + blockIdx.x;
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

// FP64 L1 norm of the residual.
template <class T>
__global__ void pr_residual_l1(const T *res, uint32_t n, double *out) {
    double acc = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        acc += fabs(static_cast<double>(res[v]));
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane_id() == 0 && acc != 0.0) atomicAdd(out, acc);
}

template <class T>
__global__ void pr_export(PrArrays<T> a, uint32_t n, float *rank, float *res, double *rank64, double *res64) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const T x = rank_value(a, v);
        if (rank) rank[v] = static_cast<float>(x);
        if (res) res[v] = static_cast<float>(__ldcg(a.res + v));
        if (rank64) rank64[v] = static_cast<double>(x);
        if (res64) res64[v] = static_cast<double>(__ldcg(a.res + v));
    }
}

}  // namespace cig
