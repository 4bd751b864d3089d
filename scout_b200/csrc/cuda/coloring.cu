// coloring.cu -- dynamic colouring repair (LCL, 1-hop), the reference's round rule on device.
//
// Rule (scout_coloring.cu:243-277, 46-100): an inserted edge whose endpoints share a colour
// (pre-batch colours) marks its higher endpoint. Then rounds: every marked vertex proposes the
// smallest colour c >= 0 absent from its neighbours' pre-round colours; a vertex loses if a
// lower-id neighbour in the same round proposed the same colour; all proposals are applied;
// losers form the next round. Deletions never need repair. The reference caps a round at
// 200,000 vertices / 20M adjacency entries and drops the rest (scout_coloring.cu:180-188);
// here every marked vertex is processed, so the outcome equals the reference's wherever the
// reference did not truncate, and is a proper colouring always.
//
// One cooperative launch per batch; per round three phases separated by the bounded grid
// barrier: propose (warp per row up to 4096 entries, whole block per longer row, colours
// gathered into a shared-memory bitmap of 1024-colour windows), detect, apply.
#include "ctx.cuh"
#include "coloring_dev.cuh"

namespace scout {

__global__ void __launch_bounds__(COL_THREADS) k_coloring(ColParams p) { coloring_body(p); }


__global__ void k_fill_marker(int32_t* __restrict__ m, int64_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        m[v] = UNMARKED;
}

int coloring_ensure(scout_ctx* c) {
    if (!c->d_misc || c->cap_misc < c->n) {   // per-vertex proposal markers, UNMARKED at rest
        if (c->d_misc) dev_free(c, c->d_misc, (size_t)c->cap_misc * 4);
        c->d_misc = nullptr;
        c->cap_misc = 0;
        SCOUT_RC(dev_alloc(c, &c->d_misc, (size_t)c->n * 4, "colour markers"));
        c->cap_misc = c->n;
        k_fill_marker<<<blocks_for(c->n, 256), 256, 0, c->s_main>>>((int32_t*)c->d_misc, c->n);
        SCOUT_LAUNCH(c, "k_fill_marker");
    }
    return SCOUT_OK;
}

// The kernel's parameters for the context's current batch (buffers ensured first).
int coloring_params(scout_ctx* c, ColParams* out) {
    SCOUT_RC(lists_ensure(c));
    SCOUT_RC(coloring_ensure(c));
    ColParams& p = *out;
    p.g = dgraph(c);
    p.color = c->color;
    p.marker = (int32_t*)c->d_misc;
    p.hkeys = c->d_hkeys;
    p.B = c->key_bits;
    p.list[0] = c->d_list[1];
    p.list[1] = (int32_t*)c->d_qbuf[0];
    p.prop = (int32_t*)c->d_qbuf[1];
    p.touched = c->d_list[0];
    p.st_round = c->stamp_a;
    p.st_touch = c->stamp_b;
    p.epoch = (int32_t)c->epoch;
    p.ctr = c->d_ctr;
    p.bar = c->d_bar;
    return SCOUT_OK;
}

int coloring_repair(scout_ctx* c, scout_batch_stats* st) {
    (void)st;
    ColParams p;
    SCOUT_RC(coloring_params(c, &p));
    void* args[] = {&p};
    return coop_launch(c, (const void*)k_coloring, COL_THREADS, args, 0);
}

}  // namespace scout
