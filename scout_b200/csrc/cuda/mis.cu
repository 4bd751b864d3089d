// mis.cu -- dynamic maximal independent set repair (LCL, 2-hop), deterministic id priority.
//
// Trigger rule of the reference (process_clusters_csr_kernel, scout_mis.cu:290-362): an
// inserted edge with both endpoints in the set drops max(u,v); a deleted edge may free its
// non-member endpoint. The reference re-admits only the first qualifying vertex of the
// dropped vertex's packed 2-hop ball, in a racy cluster order, and checks deletions against
// 2-hop balls, so its set is neither deterministic nor always maximal. Here the repair region
// is the same 2-hop neighbourhood, and every vertex that may have lost its last set neighbour
// (the dropped vertices, their neighbours, the endpoints of deleted edges) is re-admitted in
// ascending vertex-id order: the parallel rounds below (a candidate joins once no lower-id
// undecided candidate neighbour and no member neighbour remains) give exactly the sequential
// greedy result, so the set is independent and maximal after every batch.
#include "ctx.cuh"
#include "mis_dev.cuh"

namespace scout {

__global__ void __launch_bounds__(MIS_THREADS) k_mis(MisParams p) { mis_body(p); }


// The kernel's parameters for the context's current batch (buffers ensured first).
int mis_params(scout_ctx* c, MisParams* out) {
    SCOUT_RC(lists_ensure(c));
    MisParams& p = *out;
    p.g = dgraph(c);
    p.mis = c->mis;
    p.hkeys = c->d_hkeys;
    p.B = c->key_bits;
    p.list[0] = c->d_list[1];
    p.list[1] = (int32_t*)c->d_qbuf[0];
    p.removed = (int32_t*)c->d_qbuf[1];
    p.touched = c->d_list[0];
    p.st_cand = c->stamp_a;
    p.st_done = c->stamp_c;
    p.st_touch = c->stamp_b;
    p.epoch = (int32_t)c->epoch;
    p.ctr = c->d_ctr;
    p.bar = c->d_bar;
    return SCOUT_OK;
}

int mis_repair(scout_ctx* c, scout_batch_stats* st) {
    (void)st;
    MisParams p;
    SCOUT_RC(mis_params(c, &p));
    void* args[] = {&p};
    return coop_launch(c, (const void*)k_mis, MIS_THREADS, args, 0);
}

}  // namespace scout
