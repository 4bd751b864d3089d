// common.cuh -- shared device infrastructure of the sm_100a engine.
//
//   Row        per-vertex row descriptor in HBM: (start, len) into the element pool; rows
//              are kept sorted ascending so adjacency tests are binary searches.
//   GridBar    bounded grid-wide barrier for the persistent cooperative kernels: every wait
//              is limited by %globaltimer; a timeout sets a sticky error flag that makes all
//              blocks leave, and the host reads it back as SCOUT_E_TIMEOUT.
//   Counters   small device block of per-batch counters (copied back once per batch).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace scout {

constexpr int WARP = 32;
constexpr uint32_t UNREACHED_U = 0xFFFFFFFFu;   // level -1 seen as unsigned: +infinity

struct __align__(16) Row {
    long long start;   // element index in the pool
    int len;           // degree
    int cap;           // reserved elements at start (>= len)
};

// Device-resident graph handle passed by value to kernels.
struct DGraph {
    const Row* row;
    const int32_t* pool;
    int32_t n;
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & (WARP - 1); }

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename T>
__device__ __forceinline__ T ld_volatile(const T* p) { return *(const volatile T*)p; }

// Inclusive warp scan of 64-bit values.
__device__ __forceinline__ long long warp_incl_scan(long long x) {
#pragma unroll
    for (int o = 1; o < WARP; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane_id() >= o) x += y;
    }
    return x;
}
__device__ __forceinline__ int warp_incl_scan_i(int x) {
#pragma unroll
    for (int o = 1; o < WARP; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane_id() >= o) x += y;
    }
    return x;
}

// Warp-aggregated append: every lane with `pred` gets a distinct slot of `q` through one
// atomicAdd per warp. Returns the slot (or -1); slots beyond cap are not written and the
// caller sees the overflow in the counter.
__device__ __forceinline__ int warp_append(bool pred, int* counter) {
    unsigned m = __ballot_sync(__activemask(), pred);
    if (!m) return -1;
    int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(__activemask(), base, leader);
    if (!pred) return -1;
    return base + __popc(m & ((1u << lane_id()) - 1));
}

// Binary search helpers over sorted int32 spans.
__device__ __forceinline__ long long lower_bound_i32(const int32_t* a, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ long long upper_bound_i32(const int32_t* a, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Adjacency test on sorted rows: binary search in the shorter of the two rows.
__device__ __forceinline__ bool dg_adjacent(const DGraph& g, int32_t u, int32_t v) {
    Row ru = g.row[u], rv = g.row[v];
    if (rv.len < ru.len) { Row t = ru; ru = rv; rv = t; int32_t s = u; u = v; v = s; }
    const int32_t* a = g.pool + ru.start;
    long long k = lower_bound_i32(a, ru.len, v);
    return k < ru.len && a[k] == v;
}

// ---------------------------------------------------------------------------------------
// Bounded grid barrier (cooperative launch guarantees co-residency of all blocks).
// `count` only grows within a launch: the k-th barrier is complete once it reaches k * blocks,
// so the last block's own arrival releases the others (no reset and no second counter to bump).
// Every block passes the same sequence of barriers, so a block arriving at barrier k sees
// old in [(k - 1) * blocks, k * blocks). The host zeroes the block before each launch.
// ---------------------------------------------------------------------------------------
struct GridBar {
    unsigned int count;
    unsigned int gen;   // unused; kept for the layout the host reads back
    int err;            // 0 ok, 1 barrier timeout, 2 capacity overflow inside a kernel
    int where;          // tag of the barrier that timed out
};

constexpr uint64_t GRID_WAIT_LIMIT_NS = 4000000000ull;   // 4 s

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(GridBar* b, int tag = 0) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
        __threadfence();
        const unsigned old = atomicAdd(&b->count, 1u);
        const unsigned target = (old / nb + 1) * nb;
        if (old + 1 != target) {
            uint64_t t0 = 0;
            while ((int)(ld_acquire_gpu(&b->count) - target) < 0) {
                if (ld_volatile(&b->err)) break;
                const uint64_t t = globaltimer_ns();
                if (t0 == 0) {
                    t0 = t;
                } else if (t - t0 > GRID_WAIT_LIMIT_NS) {
                    if (atomicCAS(&b->err, 0, 1) == 0) b->where = tag;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ld_volatile(&b->err) == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void grid_fail(GridBar* b, int code) { atomicCAS(&b->err, 0, code); }

// Phase timestamp written by one thread right after a grid barrier (profiling aid).
__device__ __forceinline__ void phase_mark(unsigned long long* slot) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *slot = globaltimer_ns();
}

// Global warp index / count for grid-stride warp loops.
__device__ __forceinline__ int gwarp_id() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) / WARP); }
__device__ __forceinline__ int gwarp_count() { return (int)((gridDim.x * blockDim.x) / WARP); }

}  // namespace scout
