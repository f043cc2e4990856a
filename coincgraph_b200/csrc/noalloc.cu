// noalloc.cu - BFS depths over a device CSR without any allocation.
//
// Some callers cannot call cudaMalloc where they need a traversal: a plugin
// or embedded runtime whose device memory belongs to a host framework with
// its own pooling allocator (a raw cudaMalloc there bypasses the pool's
// accounting and fails once the pool holds the memory), or a latency-bound
// loop that must not take the device-wide synchronisation that cudaFree
// implies.  cig_bfs_csr_noalloc serves them: the caller passes the graph
// (device CSR) and the output array; every piece of scratch (frontier
// queues, per-round de-duplication stamps, counters, the grid barrier and the
// error word) lives in one file-scope __device__ array of fixed size, so the
// call performs no cudaMalloc, cudaFree or allocating library call.  The call
// is blocking: it reads the device error word back and synchronises the
// caller's stream before it returns.
//
// Limits and sharing: at most kNoAllocMaxVertices vertices (about 3 MiB of
// scratch, held by every GPU that loads the library until the process
// exits); larger graphs are rejected with CIG_ERR_ARG.  The first call on a
// device looks up the array's device address with that device current
// (set-up), so it should come before any stream capture.  All calls on a
// device share the same array and see what the last call left in it; each
// call clears everything that must start at zero before its kernels read it.
// Two calls whose work overlaps on one GPU (two host threads, or two streams)
// race on the shared array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cig.h"
#include "common.cuh"
#include "expand.cuh"

namespace {

constexpr uint32_t kNoAllocMaxVertices = CIG_NOALLOC_MAX_VERTICES;
constexpr int kTpbNa = 256;

struct NoAllocScratch {
    cig::Status st;          // error word, counters, grid barrier
    uint32_t cnt[3];         // rotating round counters of the frontier
    uint32_t q0[kNoAllocMaxVertices + 1];
    uint32_t q1[kNoAllocMaxVertices + 1];
    uint32_t stamp[kNoAllocMaxVertices];  // last round that queued a vertex
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Relax x -> y with depth(x) + 1; queue y once per round when it improves.
struct BfsDepthOp {
    uint32_t *depth;
    uint32_t *stamp;
    uint32_t tag;
    uint32_t *q_out;
    uint32_t *q_cnt;
    uint32_t cap;
    cig::Status *st;

    __device__ __forceinline__ bool edge(bool valid, uint32_t, uint32_t dx, uint32_t y) const {
        bool want = false, improved = false;
        if (valid) {
            const uint32_t nd = dx + 1u;
            if (nd < __ldcg(depth + y)) {
                improved = nd < atomicMin(depth + y, nd);
                if (improved && __ldcg(stamp + y) != tag) want = atomicExch(stamp + y, tag) != tag;
            }
        }
        cig::warp_enqueue(want, y, q_out, q_cnt, cap, st);
        return improved;
    }
};

__global__ void noalloc_bfs_init(uint32_t *depth, uint32_t n, uint32_t source, NoAllocScratch *s) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        depth[v] = (v == source) ? 0u : cig::kInf;
        s->stamp[v] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s->q0[0] = source;
        s->cnt[0] = 1u;
        s->cnt[1] = 0u;
        s->cnt[2] = 0u;
    }
}

// Persistent cooperative closure (same round structure as push_closure).
__global__ void __launch_bounds__(kTpbNa) noalloc_bfs_closure(const uint64_t *xadj, const uint32_t *adj, uint32_t n,
                                                              uint32_t *depth, NoAllocScratch *s) {
    __shared__ cig::ExpandSmem<kTpbNa> sm;
    cig::ExpandCounters cnt;
    const cig::AdjView view{nullptr, const_cast<uint32_t *>(adj), nullptr, nullptr, nullptr};
    for (uint32_t r = 0;; ++r) {
        const uint32_t n_in = cig::ld_volatile(s->cnt + (r % 3));
        if (n_in == 0) break;
        if (r > n + 1) {
            if (blockIdx.x == 0 && threadIdx.x == 0) cig::set_error(&s->st, cig::kErrRounds, r);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) s->cnt[(r + 2) % 3] = 0;
        const uint32_t *in = (r & 1) ? s->q1 : s->q0;
        BfsDepthOp op{depth, s->stamp, r + 1u, (r & 1) ? s->q0 : s->q1, s->cnt + ((r + 1) % 3), n + 1, &s->st};
        for (uint32_t base = 0; base < n_in; base += gridDim.x * kTpbNa) {
            const uint32_t i = base + threadIdx.x * gridDim.x + blockIdx.x;
            bool has = i < n_in;
            uint32_t x = 0, dx = 0, deg = 0;
            uint64_t off = 0;
            if (has) {
                x = __ldcg(in + i);
                dx = __ldcg(depth + x);
                off = xadj[x];
                deg = static_cast<uint32_t>(xadj[x + 1] - off);
                has = deg > 0;
            }
            cig::expand_rows<kTpbNa>(view, has, x, dx, off, deg, op, sm, cnt);
        }
        if (!cig::grid_barrier(&s->st)) break;
    }
}

// Device address of the scratch array, looked up once per device.
std::mutex g_setup_mutex;
NoAllocScratch *g_scratch_ptr[128] = {};

}  // namespace

// Records the message returned by cig_last_error(NULL) (engine.cu).
void cig_set_unbound_error(const std::string &message);

namespace {
int fail(int code, const std::string &msg) {
    cig_set_unbound_error(msg);
    return code;
}
}  // namespace

extern "C" int cig_bfs_csr_noalloc(const uint64_t *xadj, const uint32_t *adj, uint32_t n, uint32_t source,
                                   uint32_t *depth, void *stream_handle) {
    if (n == 0 || n > kNoAllocMaxVertices)
        return fail(CIG_ERR_ARG, "vertex count must be in [1, " + std::to_string(kNoAllocMaxVertices) + "]");
    if (!xadj || !adj || !depth || source >= n)
        return fail(CIG_ERR_ARG, "null CSR/output pointer or source out of range");
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) return fail(CIG_ERR_DEVICE, "no current CUDA device");
    NoAllocScratch *s = nullptr;
    {
        // Set-up on the first call on this device (with it current).
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(CIG_ERR_DEVICE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_ptr[dev] = static_cast<NoAllocScratch *>(p);
        }
        s = g_scratch_ptr[dev];
    }
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_bfs_closure, kTpbNa, 0) != cudaSuccess ||
        per_sm < 1)
        return fail(CIG_ERR_DEVICE, "cannot size the cooperative launch");
    const int blocks = sms * (per_sm < 2 ? per_sm : 2);
    // Clear the error word, counters and barrier state left by the last call.
    e = cudaMemsetAsync(&s->st, 0, sizeof(cig::Status), stream);
    if (e != cudaSuccess) return fail(CIG_ERR_DEVICE, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    noalloc_bfs_init<<<sms * 4, 256, 0, stream>>>(depth, n, source, s);
    void *args[] = {const_cast<uint64_t **>(&xadj), const_cast<uint32_t **>(&adj), &n, &depth, &s};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(noalloc_bfs_closure), dim3(blocks), dim3(kTpbNa),
                                    args, 0, stream);
    if (e != cudaSuccess) return fail(CIG_ERR_DEVICE, std::string("launch: ") + cudaGetErrorString(e));
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, &s->st.err, sizeof(err), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(CIG_ERR_DEVICE, std::string("BFS: ") + cudaGetErrorString(e));
    if (err) return fail(CIG_ERR_LIMIT, "device reported error flags " + std::to_string(err));
    return CIG_OK;
}
