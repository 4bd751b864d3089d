// seed.cu -- initial solutions computed on the device from the resident graph.
//
// The reference seeds its streams with offline host tools: greedy MIS in vertex-id order
// (tools/compute_initial_mis.py:32-43), greedy smallest-free colouring in vertex-id order
// (tools/greedy_color.cpp:37-52), BFS levels (tools/bfs_ground_truth.cu:39-151) and min-id
// component labels (tools/excc_src/excc_v1.cu:520-531). scout_seed computes the same solutions
// on the GPU: BFS and CC by the engine's own full traversal and recompute, the two greedy
// rules by one persistent kernel of rounds. A vertex decides once every lower-id neighbour has
// decided (rows are sorted, so those neighbours are a prefix of its row):
//   MIS       in iff no lower-id neighbour is in
//   colouring the smallest colour no lower-id neighbour has
// Decisions only go from undecided to final, so reading neighbours that decide during the same
// round cannot change any outcome: the result is the sequential greedy one whatever the timing.
// The number of rounds is the longest chain of vertices each waiting on a lower-id neighbour.
#include "ctx.cuh"

#include <cstring>

namespace scout {

constexpr int SEED_THREADS = 256;
constexpr int32_t UNDECIDED = -1;

struct SeedParams {
    DGraph g;
    int32_t* out;       // MIS: 1 in / 0 out; colouring: colour; UNDECIDED while open
    int mode;           // 0 MIS, 1 colouring
    int32_t* wl[2];     // open vertices of the current and the next round (n each)
    DevCounters* ctr;   // list_count[0..1]: sizes of wl, rounds
    GridBar* bar;
};

// The row prefix of neighbours below v (rows ascending).
__device__ __forceinline__ int lower_prefix(const int32_t* r, int len, int32_t v) {
    return (int)lower_bound_i32(r, len, v);
}

__global__ void __launch_bounds__(SEED_THREADS) k_seed_greedy(SeedParams p) {
    const int64_t n = p.g.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    for (int64_t v = tid; v < n; v += T) {
        p.out[v] = UNDECIDED;
        p.wl[0][v] = (int32_t)v;
    }
    if (leader) { p.ctr->list_count[0] = (int)n; p.ctr->list_count[1] = 0; }
    if (!grid_sync(p.bar, 50)) return;
    int cur = 0, rounds = 0;
    long long bytes = 0;
    while (true) {
        const int cnt = ld_volatile(&p.ctr->list_count[cur]);
        if (cnt == 0) break;
        const int nxt = cur ^ 1;
        for (int64_t b = tid - (tid & (WARP - 1)); b < cnt; b += T) {
            const int64_t i = b + lane_id();
            bool open = false;
            int32_t v = 0;
            if (i < cnt) {
                v = p.wl[cur][i];
                const Row r = p.g.row[v];
                const int32_t* row = p.g.pool + r.start;
                const int k = lower_prefix(row, r.len, v);
                bytes += 16 + 4LL * k * 2;
                if (p.mode == 0) {
                    bool any_in = false, all_done = true;
                    for (int j = 0; j < k && !any_in; j++) {
                        const int32_t s = ld_volatile(p.out + row[j]);
                        any_in = s == 1;
                        all_done &= s != UNDECIDED;
                    }
                    if (any_in) p.out[v] = 0;
                    else if (all_done) p.out[v] = 1;
                    else open = true;
                } else {
                    bool all_done = true;
                    for (int j = 0; j < k && all_done; j++) all_done = ld_volatile(p.out + row[j]) != UNDECIDED;
                    if (!all_done) {
                        open = true;
                    } else {
                        int32_t colour = 0;
                        for (int32_t base = 0;; base += 64) {   // smallest colour absent below
                            unsigned long long used = 0;
                            for (int j = 0; j < k; j++) {
                                const int32_t c = ld_volatile(p.out + row[j]) - base;
                                if (c >= 0 && c < 64) used |= 1ull << c;
                            }
                            if (~used) { colour = base + __ffsll((long long)~used) - 1; break; }
                        }
                        p.out[v] = colour;
                    }
                }
            }
            const int at = warp_append(open, &p.ctr->list_count[nxt]);
            if (open) p.wl[nxt][at] = v;
        }
        rounds++;
        if (!grid_sync(p.bar, 51)) return;
        if (leader) p.ctr->list_count[cur] = 0;
        if (!grid_sync(p.bar, 52)) return;
        cur = nxt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
    if (leader) p.ctr->rounds = rounds;
}

}  // namespace scout

using namespace scout;

extern "C" int scout_recompute_bfs(scout_ctx*, int32_t, scout_batch_stats*);
extern "C" int scout_recompute_cc(scout_ctx*, scout_batch_stats*);

extern "C" {

int scout_seed(scout_ctx* c, int problem, int32_t source, scout_batch_stats* st) {
    if (!c) return SCOUT_E_INVALID;
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    if (problem < SCOUT_MIS || problem > SCOUT_CC) return c->fail(SCOUT_E_INVALID, "unknown problem");
    cudaSetDevice(c->device);
    scout_batch_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    int32_t** slot = problem == SCOUT_MIS ? &c->mis : problem == SCOUT_COLORING ? &c->color
                     : problem == SCOUT_BFS ? &c->level : &c->label;
    if (!*slot) {
        SCOUT_RC(dev_alloc(c, (void**)slot, (size_t)c->n * 4, "solution state"));
        // a fresh state: BFS unreached everywhere, CC every vertex its own label (the full
        // traversal and recompute overwrite every entry)
        SCOUT_CU(c, cudaMemsetAsync(*slot, problem == SCOUT_BFS ? 0xff : 0, (size_t)c->n * 4, c->s_main));
    }
    if (problem == SCOUT_BFS) {
        if (source < 0 || source >= c->n) return c->fail(SCOUT_E_INVALID, "source out of range");
        return scout_recompute_bfs(c, source, st);
    }
    if (problem == SCOUT_CC) return scout_recompute_cc(c, st);
    SCOUT_RC(lists_ensure(c));
    SCOUT_RC(batch_begin(c));
    SeedParams p;
    p.g = dgraph(c);
    p.out = *slot;
    p.mode = problem == SCOUT_MIS ? 0 : 1;
    p.wl[0] = c->d_list[0];
    p.wl[1] = c->d_list[1];
    p.ctr = c->d_ctr;
    p.bar = c->d_bar;
    c->last_problem = problem;
    SCOUT_CU(c, cudaEventRecord(c->ev_t[1], c->s_main));
    void* args[] = {&p};
    SCOUT_RC(coop_launch(c, (const void*)k_seed_greedy, SEED_THREADS, args, 0));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[2], c->s_main));
    SCOUT_RC(counters_fetch(c));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev_t[1], c->ev_t[2]);
    st->ms_repair = ms;
    st->rounds = c->h_ctr->rounds;
    st->hbm_bytes = c->h_ctr->hbm_bytes;
    st->changed = c->n;
    c->last_changed = 0;   // nothing to commit: download the state
    return SCOUT_OK;
}

}  // extern "C"
