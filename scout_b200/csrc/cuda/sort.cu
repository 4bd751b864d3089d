// sort.cu -- stable LSD radix sort of 64-bit keys and an exclusive int64 scan.
//
// The batch merge groups half-edits by (vertex, op, neighbour) with one sort. Small sorts run
// in one CTA entirely in shared memory (one launch). Larger ones follow the one-sweep scheme
// (Adinets and Merrill, "Onesweep: a faster least significant digit radix sort for GPUs",
// 2022): one kernel histograms every 8-bit digit of every pass at once and turns the
// histograms into global digit offsets; then each pass is ONE kernel whose blocks take tiles in
// order from an atomic counter, rank their keys stably (each warp ranks its own contiguous 512
// keys with __match_any_sync), publish their digit counts and obtain the counts of all earlier
// tiles by a decoupled look-back, and write the tile out through shared memory so that runs of
// equal digits land contiguously. 1 + passes launches instead of five per pass.
#include "ctx.cuh"

#include <algorithm>
#include <atomic>

namespace scout {

constexpr int SORT_RADIX = 256;
// 2 * 10240 keys * 8 B + 33 * 256 * 4 B of tables = 197,632 B of dynamic shared memory,
// under the 220 KB opt-in requested below.
constexpr int SMALL_SORT_MAX = 10240;
constexpr int SMALL_SORT_THREADS = 1024;

// ---- one-sweep radix sort -------------------------------------------------------------------
constexpr int OS_THREADS = 256;
constexpr int OS_WARPS = OS_THREADS / WARP;
constexpr int OS_STEPS = 16;                        // 32-key steps per warp (large sorts)
constexpr int OS_TILE = OS_THREADS * OS_STEPS;      // 4096 keys per tile
constexpr int OS_STEPS_SMALL = 4;                   // mid-size sorts: 1024-key tiles fill more SMs
constexpr int OS_TILE_SMALL = OS_THREADS * OS_STEPS_SMALL;
constexpr int OS_MAX_PASSES = 8;
// control block in the sort buffer (32-bit words): [pass][256] histograms, then global digit
// offsets; the done counter; the per-pass tile counters; the look-back entries (64-bit) follow
constexpr int OS_DONE = OS_MAX_PASSES * SORT_RADIX;
constexpr int OS_TILECTR = OS_DONE + 1;
constexpr int OS_CTRL_WORDS = 4096;
constexpr unsigned long long OS_AGG = 1ull << 32, OS_INC = 2ull << 32;
constexpr uint64_t OS_WAIT_LIMIT_NS = 2000000000ull;   // 2 s

// Every digit of every pass at once; the last block to finish turns the histograms into
// exclusive global offsets and resets the tile counters.
__global__ void __launch_bounds__(OS_THREADS) k_os_hist(const unsigned long long* __restrict__ keys, int64_t n,
                                                        int passes, unsigned int* __restrict__ ctl) {
    __shared__ unsigned int h[OS_MAX_PASSES][SORT_RADIX];
    __shared__ bool last;
    for (int i = threadIdx.x; i < OS_MAX_PASSES * SORT_RADIX; i += OS_THREADS) (&h[0][0])[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)OS_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * OS_THREADS) {
        const unsigned long long k = keys[i];
        for (int p = 0; p < passes; p++) atomicAdd(&h[p][(unsigned)(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; p++)
        if (h[p][threadIdx.x]) atomicAdd(&ctl[p * SORT_RADIX + threadIdx.x], h[p][threadIdx.x]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ctl[OS_DONE], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int p = 0; p < passes; p++) {   // thread d: exclusive prefix of digit d in pass p
        __shared__ unsigned int col[SORT_RADIX];
        col[threadIdx.x] = ld_volatile(&ctl[p * SORT_RADIX + threadIdx.x]);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned run = 0;
            for (int d = 0; d < SORT_RADIX; d++) { const unsigned c = col[d]; col[d] = run; run += c; }
        }
        __syncthreads();
        ctl[p * SORT_RADIX + threadIdx.x] = col[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x < OS_MAX_PASSES) ctl[OS_TILECTR + threadIdx.x] = 0;
    if (threadIdx.x == 0) ctl[OS_DONE] = 0;
}

// One pass: stable scatter of every tile of STEPS * 256 keys by the digit at `shift`. stamp
// tags this pass's look-back entries (entries of earlier passes read as empty).
template <int STEPS>
__global__ void __launch_bounds__(OS_THREADS) k_os_pass(const unsigned long long* __restrict__ src,
                                                        unsigned long long* __restrict__ dst, int64_t n, int pass,
                                                        unsigned int* __restrict__ ctl,
                                                        unsigned long long* __restrict__ lb, unsigned stamp,
                                                        int* __restrict__ err) {
    constexpr int TILE = OS_THREADS * STEPS;
    __shared__ unsigned long long sk[TILE];
    __shared__ unsigned int wh[OS_WARPS][SORT_RADIX];   // per-warp digit counts, then prefixes
    __shared__ unsigned int tot[SORT_RADIX], toff[SORT_RADIX];
    __shared__ long long gbase[SORT_RADIX];
    __shared__ int s_tile;
    const int t = threadIdx.x, w = t / WARP, l = (int)lane_id();
    const int shift = 8 * pass;
    if (t == 0) s_tile = (int)atomicAdd(&ctl[OS_TILECTR + pass], 1u);
    for (int j = 0; j < OS_WARPS; j++) wh[j][t] = 0;
    __syncthreads();
    const int tile = s_tile;
    const int64_t t0 = (int64_t)tile * TILE;
    // each warp ranks its contiguous 512 keys, 32 at a time, in order (stable)
    unsigned long long key[STEPS];
    unsigned short lr[STEPS];
    const unsigned lt = (1u << l) - 1;
    const int64_t wbase = t0 + (int64_t)w * (STEPS * WARP);
#pragma unroll
    for (int s = 0; s < STEPS; s++) {
        const int64_t i = wbase + s * WARP + l;
        const bool valid = i < n;
        key[s] = valid ? src[i] : ~0ull;
        const unsigned d = valid ? (unsigned)(key[s] >> shift) & 255u : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        unsigned c = 0;
        if (valid && l == leader) c = wh[w][d];
        c = __shfl_sync(0xffffffffu, c, leader);
        lr[s] = (unsigned short)(c + __popc(peers & lt));
        __syncwarp();
        if (valid && l == leader) wh[w][d] = c + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {   // thread t owns digit t: prefix over warps (warp order is key order), tile total
        unsigned run = 0;
        for (int j = 0; j < OS_WARPS; j++) { const unsigned c = wh[j][t]; wh[j][t] = run; run += c; }
        tot[t] = run;
    }
    // publish this tile's count, then look back over the earlier tiles
    const unsigned long long tag = (unsigned long long)stamp << 34;
    unsigned long long* mine = lb + (int64_t)tile * SORT_RADIX + t;
    if (tile == 0) {
        atomicExch(mine, tag | OS_INC | tot[t]);
        gbase[t] = ctl[pass * SORT_RADIX + t];
    } else {
        atomicExch(mine, tag | OS_AGG | tot[t]);
        unsigned long long excl = 0;
        int j = tile - 1;
        const uint64_t start = globaltimer_ns();
        while (j >= 0) {
            const unsigned long long v = ld_volatile(lb + (int64_t)j * SORT_RADIX + t);
            if ((v >> 34) == (unsigned long long)stamp && (v & (3ull << 32))) {
                excl += v & 0xffffffffull;
                if (v & OS_INC) break;
                j--;
                continue;
            }
            if (globaltimer_ns() - start > OS_WAIT_LIMIT_NS) { atomicExch(err, 1); break; }
            __nanosleep(32);
        }
        atomicExch(mine, tag | OS_INC | (excl + tot[t]));
        gbase[t] = (long long)ctl[pass * SORT_RADIX + t] + (long long)excl;
    }
    // tile-local digit offsets (exclusive scan of tot)
    {
        __shared__ unsigned int ws[OS_WARPS];
        unsigned x = tot[t], inc = x;
#pragma unroll
        for (int o = 1; o < WARP; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
            if (l >= o) inc += y;
        }
        if (l == WARP - 1) ws[w] = inc;
        __syncthreads();
        unsigned wb = 0;
        for (int j = 0; j < w; j++) wb += ws[j];
        toff[t] = wb + inc - x;
    }
    __syncthreads();
    // stage the tile in digit order, then write it out: equal digits are contiguous runs
#pragma unroll
    for (int s = 0; s < STEPS; s++) {
        const int64_t i = wbase + s * WARP + l;
        if (i < n) {
            const unsigned d = (unsigned)(key[s] >> shift) & 255u;
            sk[toff[d] + wh[w][d] + lr[s]] = key[s];
        }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)TILE, n - t0);
    for (int j = t; j < cnt; j += OS_THREADS) {
        const unsigned long long k = sk[j];
        const unsigned d = (unsigned)(k >> shift) & 255u;
        const long long pos = gbase[d] + (j - (int)toff[d]);
        if (pos >= 0 && pos < n) dst[pos] = k;
        else atomicExch(err, 2);
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

// Single-pass exclusive scan (decoupled look-back, after Merrill and Garland, "Single-pass
// parallel prefix scan with decoupled look-back", 2016). Tiles of SCAN_TILE entries take
// tickets in order from a counter; a tile publishes its aggregate, its first warp walks back
// over the earlier tiles 32 at a time (adding aggregates up to the nearest published inclusive
// prefix) and publishes its own prefix, then the block writes its exclusive prefixes. One launch for any
// length. State in st (64-bit words): [0] the ticket counter, then per tile a status word
// (LB_TAG | stamp << 2 | flag; flag 1 aggregate, 2 inclusive prefix), the aggregate and the
// prefix. The stamp is unique per call, so no state is cleared between calls. A wait past
// LB_WAIT_LIMIT_NS flags err = 4 (the host fails the batch) and the tile goes on.
constexpr unsigned long long LB_TAG = 0xA5ull << 56;
constexpr uint64_t LB_WAIT_LIMIT_NS = 1000000000ull;   // 1 s

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_lb(T* __restrict__ a, int64_t n, int64_t* __restrict__ d_total,
                                                          unsigned long long* __restrict__ st, unsigned stamp,
                                                          int* __restrict__ err) {
    __shared__ int s_tile;
    __shared__ long long s_tot, s_prefix;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd((unsigned*)st, 1u);
    __syncthreads();
    const int tile = s_tile;
    const int64_t base = (int64_t)tile * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    long long v[SCAN_ITEMS];
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = base + k < n ? (long long)a[base + k] : 0;
        sum += v[k];
    }
    const long long ex = block_excl_scan(sum, &s_tot);
    if (threadIdx.x < WARP) {   // warp 0: publish, look back 32 tiles per step, publish the prefix
        const long long tot = s_tot;
        const unsigned long long want = LB_TAG | ((unsigned long long)stamp << 2);
        unsigned long long* me = st + 1 + 3 * (int64_t)tile;
        const int lane = (int)threadIdx.x;
        long long prefix = 0;
        if (tile > 0) {
            if (lane == 0) {
                me[1] = (unsigned long long)tot;
                __threadfence();
                *(volatile unsigned long long*)me = want | 1ull;
            }
            const uint64_t t0 = globaltimer_ns();
            for (long long end = tile - 1;; end -= WARP) {
                const long long j = end - lane;   // lane 0 looks at the nearest tile
                unsigned long long w = want | 2ull;   // tiles before the first: a prefix of 0
                bool ok = true;
                if (j >= 0) {
                    const unsigned long long* pj = st + 1 + 3 * j;
                    w = ld_volatile(pj);
                    for (unsigned it = 1; (w & ~3ull) != want || (w & 3ull) == 0; it++) {
                        if ((it & 63) == 0 && globaltimer_ns() - t0 > LB_WAIT_LIMIT_NS) { ok = false; break; }
                        w = ld_volatile(pj);
                    }
                }
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicCAS(err, 0, 4);
                    break;
                }
                __threadfence();
                const bool pre = (w & 3ull) == 2;
                long long v = 0;
                if (j >= 0) v = (long long)ld_volatile(st + 1 + 3 * j + (pre ? 2 : 1));
                const unsigned pm = __ballot_sync(0xffffffffu, pre);
                const int f = pm ? __ffs(pm) - 1 : WARP;   // nearest tile with an inclusive prefix
                if (lane > f) v = 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                prefix += v;
                if (pm) break;
            }
        }
        if (lane == 0) {
            me[2] = (unsigned long long)(prefix + tot);
            __threadfence();
            *(volatile unsigned long long*)me = want | 2ull;
            s_prefix = prefix;
            if (d_total && (int64_t)(tile + 1) * SCAN_TILE >= n) *d_total = prefix + tot;
        }
    }
    __syncthreads();
    long long run = s_prefix + ex;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) a[base + k] = (T)run;
        run += v[k];
    }
}

static unsigned next_stamp();

template <typename T>
static int scan_any(scout_ctx* c, T* data, int64_t n, int64_t* d_total) {
    if (n <= 0) {
        if (d_total) SCOUT_CU(c, cudaMemsetAsync(d_total, 0, sizeof(int64_t), c->s_main));
        return SCOUT_OK;
    }
    const int64_t nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    SCOUT_RC(dev_grow(c, &c->d_scan_tmp, &c->cap_scan, std::max<int64_t>(64, 1 + 3 * nt), "scan look-back"));
    SCOUT_CU(c, cudaMemsetAsync(c->d_scan_tmp, 0, sizeof(int64_t), c->s_main));   // tile tickets
    k_scan_lb<T><<<(unsigned)nt, SCAN_THREADS, 0, c->s_main>>>(data, n, d_total, (unsigned long long*)c->d_scan_tmp,
                                                                next_stamp(), &c->d_ctr->sort_err);
    SCOUT_LAUNCH(c, "k_scan_lb");
    c->nlaunch += 1;
    return SCOUT_OK;
}

int scan_i64(scout_ctx* c, int64_t* data, int64_t n, int64_t* d_total) { return scan_any(c, data, n, d_total); }

// Sizes the radix histogram and the scan partials for sorts of up to nkeys keys and scans
// of up to nkeys entries, so later calls allocate nothing.
// Look-back stamps are unique across the process (contexts share freed device memory).
static unsigned next_stamp() {
    static std::atomic<unsigned> counter{0};
    unsigned s = 0;
    while (s == 0) s = (counter.fetch_add(1) + 1) & ((1u << 30) - 1);
    return s;
}

int sort_reserve(scout_ctx* c, int64_t nkeys) {
    const int64_t ntiles = (nkeys + OS_TILE_SMALL - 1) / OS_TILE_SMALL;   // the most tiles a sort can have
    unsigned int* before = c->d_sort_hist;
    SCOUT_RC(dev_grow(c, &c->d_sort_hist, &c->cap_hist, OS_CTRL_WORDS + 2 * SORT_RADIX * ntiles, "sort look-back"));
    if (c->d_sort_hist != before)   // fresh memory: no stale look-back entry may match a stamp
        SCOUT_CU(c, cudaMemsetAsync(c->d_sort_hist, 0, (size_t)c->cap_hist * 4, c->s_main));
    const int64_t scan_n = nkeys + 1;
    SCOUT_RC(dev_grow(c, &c->d_scan_tmp, &c->cap_scan, std::max<int64_t>(64, 1 + 3 * ((scan_n + SCAN_TILE - 1) / SCAN_TILE)),
                      "scan look-back"));
    return SCOUT_OK;
}

int sort_keys(scout_ctx* c, unsigned long long* keys, unsigned long long* alt, int64_t n, int bits,
              unsigned long long** sorted_out) {
    *sorted_out = keys;
    if (n <= 1) return SCOUT_OK;
    if (n <= SMALL_SORT_MAX) {
        constexpr int NW = SMALL_SORT_THREADS / WARP;
        size_t smem = 2 * (size_t)n * sizeof(unsigned long long) + (size_t)(NW + 1) * SORT_RADIX * sizeof(unsigned);
        static std::atomic<unsigned long long> attr_done{0};   // per-device setting, once per device
        const unsigned long long bit = 1ull << (c->device & 63);
        if (!(attr_done.load() & bit)) {
            SCOUT_CU(c, cudaFuncSetAttribute(k_sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
            attr_done.fetch_or(bit);
        }
        k_sort_small<<<1, SMALL_SORT_THREADS, smem, c->s_main>>>(keys, (int)n, bits);
        SCOUT_LAUNCH(c, "k_sort_small");
        c->nlaunch += 1;
        return SCOUT_OK;
    }
    const int passes = (bits + 7) / 8;
    if (passes > OS_MAX_PASSES) return c->fail(SCOUT_E_INVALID, "sort keys wider than 64 bits");
    // large tiles once they give every SM two of them, else small tiles
    const bool small_tiles = (n + OS_TILE - 1) / OS_TILE < 2 * (int64_t)c->sm_count;
    const int tile = small_tiles ? OS_TILE_SMALL : OS_TILE;
    const int64_t ntiles = (n + tile - 1) / tile;
    SCOUT_RC(sort_reserve(c, n));
    unsigned int* ctl = c->d_sort_hist;
    unsigned long long* lb = (unsigned long long*)(ctl + OS_CTRL_WORDS);
    SCOUT_CU(c, cudaMemsetAsync(ctl, 0, (size_t)(OS_DONE + 1) * 4, c->s_main));
    // a block per 1024 keys (at most four per SM): the digit histograms of skewed keys (hub
    // vertices) collide in shared memory, so fewer keys per block means shorter atomic queues
    const int hb = (int)std::min<int64_t>((n + 1023) / 1024, 4 * (int64_t)c->sm_count);
    k_os_hist<<<hb, OS_THREADS, 0, c->s_main>>>(keys, n, passes, ctl);
    SCOUT_LAUNCH(c, "k_os_hist");
    c->nlaunch += 1;
    unsigned long long* src = keys;
    unsigned long long* dst = alt;
    for (int p = 0; p < passes; p++) {
        const unsigned stamp = next_stamp();
        if (small_tiles)
            k_os_pass<OS_STEPS_SMALL><<<(unsigned)ntiles, OS_THREADS, 0, c->s_main>>>(src, dst, n, p, ctl, lb, stamp,
                                                                                    &c->d_ctr->sort_err);
        else
            k_os_pass<OS_STEPS><<<(unsigned)ntiles, OS_THREADS, 0, c->s_main>>>(src, dst, n, p, ctl, lb, stamp,
                                                                              &c->d_ctr->sort_err);
        SCOUT_LAUNCH(c, "k_os_pass");
        c->nlaunch += 1;
        unsigned long long* s = src; src = dst; dst = s;
    }
    *sorted_out = src;
    return SCOUT_OK;
}

}  // namespace scout
