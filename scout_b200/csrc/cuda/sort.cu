// sort.cu -- stable LSD radix sort of 64-bit keys and an exclusive int64 scan.
//
// The batch merge groups half-edits by (vertex, op, neighbour) with one sort. Small sorts run
// in one CTA entirely in shared memory (one launch); larger ones take, per 8-bit digit, tile
// histograms, a three-kernel scan of the digit-major histogram, and a stable scatter that
// ranks equal digits inside a warp with __match_any_sync.
#include "ctx.cuh"

#include <algorithm>

namespace scout {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int SORT_RADIX = 256;
// 2 * 10240 keys * 8 B + 33 * 256 * 4 B of tables = 197,632 B of dynamic shared memory,
// under the 220 KB opt-in requested below.
constexpr int SMALL_SORT_MAX = 10240;
constexpr int SMALL_SORT_THREADS = 1024;

__global__ void k_sort_hist(const unsigned long long* __restrict__ keys, int64_t n, int shift,
                            unsigned int* __restrict__ hist, int nblocks) {
    __shared__ unsigned int h[SORT_RADIX];
    for (int i = threadIdx.x; i < SORT_RADIX; i += blockDim.x) h[i] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * SORT_TILE;
    for (int k = 0; k < SORT_ITEMS; k++) {
        int64_t i = base + (int64_t)k * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & (SORT_RADIX - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < SORT_RADIX; d += blockDim.x) hist[(int64_t)d * nblocks + blockIdx.x] = h[d];
}


// Stable scatter of one tile: chunks of 256 keys, warp ranks via __match_any_sync, cross-warp
// offsets from a per-warp digit table.
__global__ void k_sort_scatter(const unsigned long long* __restrict__ keys, unsigned long long* __restrict__ out,
                               int64_t n, int shift, const unsigned int* __restrict__ hist, int nblocks) {
    constexpr int NW = SORT_THREADS / WARP;
    __shared__ unsigned int base[SORT_RADIX];
    __shared__ unsigned int wh[NW][SORT_RADIX];
    __shared__ unsigned int tot[SORT_RADIX];
    const int t = threadIdx.x, w = t / WARP, l = t % WARP;
    base[t] = hist[(int64_t)t * nblocks + blockIdx.x];
    int64_t tile = (int64_t)blockIdx.x * SORT_TILE;
    const unsigned lt = (1u << l) - 1;
    for (int k = 0; k < SORT_ITEMS; k++) {
        int64_t i = tile + (int64_t)k * SORT_THREADS + t;
        bool valid = i < n;
        unsigned long long key = valid ? keys[i] : 0ull;
        unsigned d = valid ? (unsigned)(key >> shift) & (SORT_RADIX - 1) : SORT_RADIX;   // invalid: own class
        for (int j = 0; j < NW; j++) wh[j][t] = 0;
        __syncthreads();
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned rank = __popc(peers & lt);
        if (valid && rank == 0) wh[w][d] = __popc(peers);
        __syncthreads();
        {   // thread t owns digit t: exclusive prefix over warps
            unsigned run = 0;
            for (int j = 0; j < NW; j++) {
                unsigned c = wh[j][t];
                wh[j][t] = run;
                run += c;
            }
            tot[t] = run;
        }
        __syncthreads();
        if (valid) out[base[d] + wh[w][d] + rank] = key;
        __syncthreads();
        base[t] += tot[t];
        __syncthreads();
    }
}

// Whole sort of n <= SMALL_SORT_MAX keys in one CTA (dynamic shared memory: 2 * n keys).
__global__ void k_sort_small(unsigned long long* __restrict__ keys, int n, int bits) {
    // Dynamic shared layout: a[n], b[n] (ping-pong keys), then a [NW + 1][256] table of
    // per-warp digit offsets with the chunk totals in its last row.
    extern __shared__ unsigned long long sm[];
    constexpr int NW = SMALL_SORT_THREADS / WARP;
    __shared__ unsigned int cnt[SORT_RADIX];
    unsigned long long* a = sm;
    unsigned long long* b = sm + n;
    unsigned int* wtab = (unsigned int*)(sm + 2 * (size_t)n);
    const int t = threadIdx.x, w = t / WARP, l = t % WARP;
    for (int i = t; i < n; i += blockDim.x) a[i] = keys[i];
    __syncthreads();
    for (int shift = 0; shift < bits; shift += 8) {
        if (t < SORT_RADIX) cnt[t] = 0;
        __syncthreads();
        for (int i = t; i < n; i += blockDim.x) atomicAdd(&cnt[(unsigned)(a[i] >> shift) & 255u], 1u);
        __syncthreads();
        if (t == 0) {
            unsigned run = 0;
            for (int d = 0; d < SORT_RADIX; d++) { unsigned c = cnt[d]; cnt[d] = run; run += c; }
        }
        __syncthreads();
        for (int c0 = 0; c0 < n; c0 += blockDim.x) {
            int i = c0 + t;
            bool valid = i < n;
            unsigned long long key = valid ? a[i] : 0ull;
            unsigned d = valid ? (unsigned)(key >> shift) & 255u : 256u;
            for (int j = t; j < NW * SORT_RADIX; j += blockDim.x) wtab[j] = 0;
            __syncthreads();
            unsigned peers = __match_any_sync(0xffffffffu, d);
            unsigned rank = __popc(peers & ((1u << l) - 1));
            if (valid && rank == 0) wtab[w * SORT_RADIX + d] = __popc(peers);
            __syncthreads();
            if (t < SORT_RADIX) {
                unsigned run = 0;
                for (int j = 0; j < NW; j++) {
                    unsigned c = wtab[j * SORT_RADIX + t];
                    wtab[j * SORT_RADIX + t] = run;
                    run += c;
                }
                wtab[NW * SORT_RADIX + t] = run;   // chunk total of digit t
            }
            __syncthreads();
            if (valid) b[cnt[d] + wtab[w * SORT_RADIX + d] + rank] = key;
            __syncthreads();
            if (t < SORT_RADIX) cnt[t] += wtab[NW * SORT_RADIX + t];
            __syncthreads();
        }
        unsigned long long* s = a; a = b; b = s;
    }
    for (int i = t; i < n; i += blockDim.x) keys[i] = a[i];
}

// ---------------------------------------------------------------------------------------
// Exclusive scans: tile sums, one-block scan of the sums, tile scans with offsets.
// ---------------------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_excl_scan(long long x, long long* total) {
    __shared__ long long ws[SCAN_THREADS / WARP];
    long long inc = warp_incl_scan(x);
    int w = threadIdx.x / WARP;
    if ((int)lane_id() == WARP - 1) ws[w] = inc;
    __syncthreads();
    if (threadIdx.x < WARP) {
        long long v = threadIdx.x < SCAN_THREADS / WARP ? ws[threadIdx.x] : 0;
        long long vi = warp_incl_scan(v);
        if (threadIdx.x < SCAN_THREADS / WARP) ws[threadIdx.x] = vi - v;
        if (threadIdx.x == SCAN_THREADS / WARP - 1 && total) *total = vi;
    }
    __syncthreads();
    long long r = ws[w] + inc - x;
    __syncthreads();
    return r;
}

template <typename T>
__global__ void k_scan_tiles(const T* __restrict__ a, int64_t n, int64_t* __restrict__ sums) {
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) s += (long long)a[base + k];
    __shared__ long long tot;
    block_excl_scan(s, &tot);
    __syncthreads();
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(int64_t* __restrict__ sums, int64_t nb, int64_t* __restrict__ d_total) {
    __shared__ long long part[1024];
    int t = threadIdx.x, T = blockDim.x;
    int64_t per = (nb + T - 1) / T;
    int64_t lo = (int64_t)t * per, hi = lo + per < nb ? lo + per : nb;
    long long s = 0;
    for (int64_t i = lo; i < hi; i++) s += sums[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {
        long long y = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += y;
        __syncthreads();
    }
    long long run = part[t] - s;
    for (int64_t i = lo; i < hi; i++) {
        long long x = sums[i];
        sums[i] = run;
        run += x;
    }
    if (t == T - 1 && d_total) *d_total = part[T - 1];
}

template <typename T>
__global__ void k_scan_apply(T* __restrict__ a, int64_t n, const int64_t* __restrict__ sums) {
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    long long v[SCAN_ITEMS];
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = base + k < n ? (long long)a[base + k] : 0;
        s += v[k];
    }
    long long ex = block_excl_scan(s, nullptr) + sums[blockIdx.x];
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) a[base + k] = (T)ex;
        ex += v[k];
    }
}

template <typename T>
static int scan_any(scout_ctx* c, T* data, int64_t n, int64_t* d_total) {
    if (n <= 0) {
        if (d_total) SCOUT_CU(c, cudaMemsetAsync(d_total, 0, sizeof(int64_t), c->s_main));
        return SCOUT_OK;
    }
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    SCOUT_RC(dev_grow(c, &c->d_scan_tmp, &c->cap_scan, nb + 1, "scan partials"));
    k_scan_tiles<T><<<(unsigned)nb, SCAN_THREADS, 0, c->s_main>>>(data, n, c->d_scan_tmp);
    k_scan_sums<<<1, 1024, 0, c->s_main>>>(c->d_scan_tmp, nb, d_total);
    k_scan_apply<T><<<(unsigned)nb, SCAN_THREADS, 0, c->s_main>>>(data, n, c->d_scan_tmp);
    SCOUT_LAUNCH(c, "scan");
    c->nlaunch += 3;
    return SCOUT_OK;
}

int scan_i64(scout_ctx* c, int64_t* data, int64_t n, int64_t* d_total) { return scan_any(c, data, n, d_total); }

// Sizes the radix histogram and the scan partials for sorts of up to nkeys keys and scans
// of up to nkeys entries, so later calls allocate nothing.
int sort_reserve(scout_ctx* c, int64_t nkeys) {
    const int64_t nblocks = (nkeys + SORT_TILE - 1) / SORT_TILE;
    SCOUT_RC(dev_grow(c, &c->d_sort_hist, &c->cap_hist, nblocks * SORT_RADIX, "sort histogram"));
    const int64_t scan_n = std::max<int64_t>(nblocks * SORT_RADIX, nkeys + 1);
    SCOUT_RC(dev_grow(c, &c->d_scan_tmp, &c->cap_scan, (scan_n + SCAN_TILE - 1) / SCAN_TILE + 1, "scan partials"));
    return SCOUT_OK;
}

int sort_keys(scout_ctx* c, unsigned long long* keys, unsigned long long* alt, int64_t n, int bits,
              unsigned long long** sorted_out) {
    *sorted_out = keys;
    if (n <= 1) return SCOUT_OK;
    if (n <= SMALL_SORT_MAX) {
        constexpr int NW = SMALL_SORT_THREADS / WARP;
        size_t smem = 2 * (size_t)n * sizeof(unsigned long long) + (size_t)(NW + 1) * SORT_RADIX * sizeof(unsigned);
        static bool attr_set = false;
        if (!attr_set) {
            SCOUT_CU(c, cudaFuncSetAttribute(k_sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            attr_set = true;
        }
        k_sort_small<<<1, SMALL_SORT_THREADS, smem, c->s_main>>>(keys, (int)n, bits);
        SCOUT_LAUNCH(c, "k_sort_small");
        c->nlaunch += 1;
        return SCOUT_OK;
    }
    int nblocks = (int)((n + SORT_TILE - 1) / SORT_TILE);
    SCOUT_RC(dev_grow(c, &c->d_sort_hist, &c->cap_hist, (int64_t)nblocks * SORT_RADIX, "sort histogram"));
    unsigned long long* src = keys;
    unsigned long long* dst = alt;
    for (int shift = 0; shift < bits; shift += 8) {
        k_sort_hist<<<nblocks, SORT_THREADS, 0, c->s_main>>>(src, n, shift, c->d_sort_hist, nblocks);
        SCOUT_RC(scan_any(c, c->d_sort_hist, (int64_t)nblocks * SORT_RADIX, nullptr));
        k_sort_scatter<<<nblocks, SORT_THREADS, 0, c->s_main>>>(src, dst, n, shift, c->d_sort_hist, nblocks);
        SCOUT_LAUNCH(c, "radix pass");
        c->nlaunch += 2;
        unsigned long long* s = src; src = dst; dst = s;
    }
    *sorted_out = src;
    return SCOUT_OK;
}

}  // namespace scout
