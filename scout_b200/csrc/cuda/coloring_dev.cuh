// coloring_dev.cuh -- device code of the coloring repair kernel (k_coloring): its parameters, helpers and
// body, shared by coloring.cu (the kernel and its host launcher) and union.cu (the one persistent
// kernel that runs several problems' repairs of a round).
#pragma once

#include "ctx.cuh"

namespace scout {

constexpr int COL_THREADS = 256;
constexpr int COL_WIN = 1024;            // colours per bitmap window
constexpr int COL_WORDS = COL_WIN / 32;
constexpr int COL_BIG = 4096;            // rows longer than this are processed by a whole block
constexpr int32_t UNMARKED = -2;

struct ColParams {
    DGraph g;
    int32_t* color;
    int32_t* marker;     // proposal of round vertices, UNMARKED elsewhere (persistent)
    const unsigned long long* hkeys;
    int B;
    int32_t* list[2];    // round vertex lists (n each)
    int32_t* prop;       // proposal per list index
    int32_t* touched;
    int32_t* st_round;   // dedupe of the initial marking (epoch)
    int32_t* st_touch;
    int32_t epoch;
    DevCounters* ctr;
    GridBar* bar;
};

struct WarpSync {
    __device__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
    __device__ void operator()() const { __syncthreads(); }
};

// Smallest colour absent from the neighbours of x, scanned by `lanes` threads of a group whose
// shared bitmap is `bm` (COL_WORDS words). `sync` synchronises the group.
template <typename Sync>
static __device__ int smallest_free(const ColParams& p, int32_t x, int tid, int lanes, unsigned* bm, Sync sync,
                             int* s_res, long long& bytes) {
    Row r = p.g.row[x];
    const int32_t* rw = p.g.pool + r.start;
    for (int base = 0;; base += COL_WIN) {
        for (int k = tid; k < COL_WORDS; k += lanes) bm[k] = 0;
        sync();
        for (long long i = tid; i < r.len; i += lanes) {
            int c = ld_volatile(p.color + rw[i]);
            if (c >= base && c < base + COL_WIN) atomicOr(&bm[(c - base) >> 5], 1u << ((c - base) & 31));
        }
        bytes += 8LL * ((r.len + lanes - 1 - tid) / lanes);
        sync();
        if (tid == 0) *s_res = -1;
        sync();
        for (int k = tid; k < COL_WORDS; k += lanes) {
            unsigned free_bits = ~bm[k];
            if (free_bits) atomicMin((unsigned*)s_res, (unsigned)(k * 32 + __ffs(free_bits) - 1));
        }
        sync();
        int res = *s_res;
        sync();
        if (res >= 0) return base + res;
    }
}

__device__ __forceinline__ void coloring_body(const ColParams& p) {
    __shared__ unsigned s_bm[COL_THREADS / WARP][COL_WORDS];
    __shared__ int s_res[COL_THREADS / WARP];
    __shared__ unsigned s_bbm[COL_WORDS];
    __shared__ int s_bres;
    __shared__ int s_flag;
    const int W = gwarp_count(), wid = gwarp_id(), wl = threadIdx.x / WARP;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    long long bytes = 0;
    int rounds = 0;

    // ---- marking: higher endpoint of every same-colour inserted edge (pre-batch colours) ----
    const int nh = ld_volatile(&p.ctr->n_half);
    for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += T) {
        int64_t k = b + lane_id();
        bool mark = false, conflict = false;
        int32_t loser = 0;
        if (k < nh) {
            unsigned long long key = p.hkeys[k];
            int op = (int)((key >> p.B) & 1ull);
            int32_t x = (int32_t)(key >> (p.B + 1));
            int32_t y = (int32_t)(key & ((1ull << p.B) - 1));
            if (op == 0 && x < y && ld_volatile(p.color + x) == ld_volatile(p.color + y)) {
                conflict = true;
                loser = y;
                mark = atomicExch(&p.st_round[y], p.epoch) != p.epoch;
            }
        }
        unsigned mc = __ballot_sync(0xffffffffu, conflict);
        if (lane_id() == 0 && mc) atomicAdd(&p.ctr->conflicts, __popc(mc));
        int at = warp_append(mark, &p.ctr->list_count[0]);
        if (mark) p.list[0][at] = loser;
    }
    if (!grid_sync(p.bar, 10)) return;

    int cur = 0;
    while (true) {
        const int cnt = ld_volatile(&p.ctr->list_count[cur]);
        if (cnt == 0) break;
        const int nxt = cur ^ 1;
        // ---- propose ----
        if (leader) p.ctr->list_count[nxt] = 0;   // nobody reads it until the detect phase
        for (int i = wid; i < cnt; i += W) {   // rows up to COL_BIG: one warp
            int32_t x = p.list[cur][i];
            if (p.g.row[x].len > COL_BIG) continue;
            int c = smallest_free(p, x, (int)lane_id(), WARP, s_bm[wl], WarpSync(), &s_res[wl], bytes);
            if (lane_id() == 0) { p.prop[i] = c; p.marker[x] = c; }
        }
        for (int i = blockIdx.x; i < cnt; i += gridDim.x) {   // longer rows: one block
            int32_t x = p.list[cur][i];
            if (p.g.row[x].len <= COL_BIG) continue;
            int c = smallest_free(p, x, threadIdx.x, COL_THREADS, s_bbm, BlockSync(), &s_bres, bytes);
            if (threadIdx.x == 0) { p.prop[i] = c; p.marker[x] = c; }
            __syncthreads();
        }
        if (!grid_sync(p.bar, 11)) return;
        // ---- detect: a lower-id round neighbour proposed the same colour ----
        for (int i = wid; i < cnt; i += W) {
            int32_t x = p.list[cur][i];
            Row r = p.g.row[x];
            if (r.len > COL_BIG) continue;
            const int32_t* rw = p.g.pool + r.start;
            int c = p.prop[i];
            bool lose = false;
            for (int b0 = 0; b0 < r.len && !lose; b0 += WARP) {
                int k = b0 + (int)lane_id();
                bool l2 = false;
                if (k < r.len) {
                    int32_t w = rw[k];
                    l2 = w < x && ld_volatile(p.marker + w) == c;
                }
                lose = __any_sync(0xffffffffu, l2);
                if (k < r.len) bytes += 8;
            }
            int at = warp_append(lane_id() == 0 && lose, &p.ctr->list_count[nxt]);
            if (lane_id() == 0 && lose) p.list[nxt][at] = x;
        }
        for (int i = blockIdx.x; i < cnt; i += gridDim.x) {
            int32_t x = p.list[cur][i];
            Row r = p.g.row[x];
            if (r.len <= COL_BIG) continue;
            const int32_t* rw = p.g.pool + r.start;
            int c = p.prop[i];
            if (threadIdx.x == 0) s_flag = 0;
            __syncthreads();
            for (long long k = threadIdx.x; k < r.len; k += COL_THREADS) {
                int32_t w = rw[k];
                if (w < x && ld_volatile(p.marker + w) == c) s_flag = 1;
            }
            bytes += 8LL * ((r.len + COL_THREADS - 1 - threadIdx.x) / COL_THREADS);
            __syncthreads();
            if (threadIdx.x == 0 && s_flag) p.list[nxt][atomicAdd(&p.ctr->list_count[nxt], 1)] = x;
            __syncthreads();
        }
        if (!grid_sync(p.bar, 12)) return;
        // ---- apply all proposals, clear markers, record touched vertices ----
        for (int64_t b = tid - (tid & (WARP - 1)); b < cnt; b += T) {
            int64_t i = b + lane_id();
            bool nt = false;
            int32_t x = 0;
            if (i < cnt) {
                x = p.list[cur][i];
                p.color[x] = p.prop[i];
                p.marker[x] = UNMARKED;
                nt = atomicExch(&p.st_touch[x], p.epoch) != p.epoch;
                bytes += 16;
            }
            int at = warp_append(nt, &p.ctr->changed);
            if (nt) p.touched[at] = x;
        }
        rounds++;
        if (!grid_sync(p.bar, 13)) return;
        cur = nxt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
    if (leader) {
        p.ctr->rounds = rounds;
        p.ctr->affected = p.ctr->changed;
    }
}
// host: the kernel parameters of the context's current batch (coloring.cu)
int coloring_params(scout_ctx* c, ColParams* out);

}  // namespace scout
