// static_bfs.cu -- BFS levels over a caller-owned device CSR without any allocation.
//
// For callers that cannot allocate device memory themselves: processes whose device memory is
// owned by another allocator or a fixed arena (a runtime embedding this library through
// cgo/JNI, for instance, whose memory manager has already claimed the device), and real-time
// loops that must not enter the driver's allocator. They pass the graph and the output in
// device memory they already hold; every working buffer of the traversal (two frontier
// queues, counters, the grid barrier) lives in the file-scope array g_bfs_scratch below,
// which each device that loads the library keeps until exit.
//
// The device code names g_bfs_scratch directly; host code only ever uses the device address
// cudaGetSymbolAddress returns for it (the symbol itself is a host-side stand-in). That
// address is looked up once per device and context: a call after the device's context was
// torn down and recreated (cudaDeviceReset) looks it up again.
#include "ctx.cuh"

#include <cuda.h>
#include <mutex>

namespace scout {

constexpr int64_t STATIC_BFS_MAX_VERTICES = 1 << 20;   // 1,048,576 vertices
constexpr int STATIC_HDR_INTS = 64;                     // barrier + counters, zeroed per call
constexpr int STATIC_BFS_THREADS = 256;

// Layout: [0, 64) header (GridBar at 0, queue counters at 8..10), then two queues of
// STATIC_BFS_MAX_VERTICES int32 each: 8 MB + 256 B in all.
static __device__ __align__(256) int32_t g_bfs_scratch[STATIC_HDR_INTS + 2 * STATIC_BFS_MAX_VERTICES];

__global__ void __launch_bounds__(STATIC_BFS_THREADS)
k_static_bfs(const int64_t* __restrict__ off, const int32_t* __restrict__ adj, int32_t n, int32_t source,
             int32_t* level) {
    GridBar* bar = (GridBar*)g_bfs_scratch;
    int* qc = g_bfs_scratch + 8;                 // rotating queue counters qc[0..2]
    int32_t* q[2] = {g_bfs_scratch + STATIC_HDR_INTS, g_bfs_scratch + STATIC_HDR_INTS + STATIC_BFS_MAX_VERTICES};
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    for (int64_t v = tid; v < n; v += T) level[v] = v == source ? 0 : -1;
    if (leader) {
        q[0][0] = source;
        qc[0] = 1;
    }
    if (!grid_sync(bar, 90)) return;
    int cur = 0, depth = 0;
    while (true) {
        const int cnt = ld_volatile(qc + cur);   // the queue index cur % 2 holds this frontier
        if (cnt == 0) break;
        const int nxt = (cur + 1) % 3, zer = (cur + 2) % 3;
        if (leader) qc[zer] = 0;
        int32_t* qin = q[depth & 1];
        int32_t* qout = q[(depth + 1) & 1];
        for (int i = gwarp_id(); i < cnt; i += gwarp_count()) {
            int32_t x = qin[i];
            long long s = off[x], e = off[x + 1];
            for (long long b0 = s; b0 < e; b0 += WARP) {
                long long k = b0 + lane_id();
                bool found = false;
                int32_t w = 0;
                if (k < e) {
                    w = adj[k];
                    found = atomicCAS(level + w, -1, depth + 1) == -1;
                }
                int at = warp_append(found, qc + nxt);
                if (found) qout[at] = w;
            }
        }
        if (!grid_sync(bar, 91)) return;
        cur = nxt;
        depth++;
    }
}

static std::mutex g_setup_mu;
static int32_t* g_scratch_dev[64];   // device address of g_bfs_scratch, per device ordinal
static CUcontext g_scratch_ctx[64];  // the context that address belongs to
static bool g_scratch_ready[64];

// The calling thread's current context, through the driver entry point the runtime exposes
// (no link-time dependency on the driver library); null when it cannot be queried.
static CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (Fn)p;
        else
            cudaGetLastError();
        looked = true;
    }
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

}  // namespace scout

using namespace scout;

extern "C" int scout_bfs_levels_noalloc(const int64_t* d_off, const int32_t* d_adj, int64_t n, int32_t source,
                                        int32_t* d_level, void* stream) {
    if (!d_off || !d_adj || !d_level) return host_fail(SCOUT_E_INVALID, "null device pointer");
    if (n < 1 || n > STATIC_BFS_MAX_VERTICES)
        return host_fail(SCOUT_E_CAPACITY, "scout_bfs_levels_noalloc handles at most " +
                                               std::to_string(STATIC_BFS_MAX_VERTICES) + " vertices (got " +
                                               std::to_string(n) + ")");
    if (source < 0 || source >= n) return host_fail(SCOUT_E_INVALID, "source out of range");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return cuda_fail(nullptr, e, "cudaGetDevice");
    int32_t* scratch = nullptr;
    {
        // One-time set-up per device (and per context of it), with that device current: the
        // device address of the static array, looked up by the first call on a device.
        std::lock_guard<std::mutex> g(g_setup_mu);
        const CUcontext cur = current_context();
        if (!g_scratch_ready[dev] || g_scratch_ctx[dev] != cur) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_bfs_scratch);
            if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetSymbolAddress(g_bfs_scratch)");
            g_scratch_dev[dev] = (int32_t*)p;
            g_scratch_ctx[dev] = current_context();
            g_scratch_ready[dev] = true;
        }
        scratch = g_scratch_dev[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    // The array keeps the previous call's contents: the barrier and counters restart at zero.
    e = cudaMemsetAsync(scratch, 0, STATIC_HDR_INTS * sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "clearing the static scratch header");
    int sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_static_bfs, STATIC_BFS_THREADS, 0);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "occupancy query");
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    int32_t nn = (int32_t)n;
    void* args[] = {(void*)&d_off, (void*)&d_adj, (void*)&nn, (void*)&source, (void*)&d_level};
    e = cudaLaunchCooperativeKernel((const void*)k_static_bfs, dim3((unsigned)(per_sm * sms)), dim3(STATIC_BFS_THREADS),
                                    args, 0, s);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "k_static_bfs launch");
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "k_static_bfs");
    GridBar bar;
    e = cudaMemcpy(&bar, scratch, sizeof(GridBar), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "reading the static scratch header");
    if (bar.err) return host_fail(SCOUT_E_TIMEOUT, "k_static_bfs: a grid barrier timed out");
    return SCOUT_OK;
}
