// bfs.cu -- exact batch-dynamic BFS levels on the device (one persistent kernel per batch).
//
// Replaces the reference's per-edit host loop (processBatch, scout_bfs.cu:436-515), its
// relax rounds (gpu_relax_round 177-272, relax_frontier_kernel 56-71), deletion cascade
// (gpu_deletion_round 325-415, deletion_compute/apply 73-105) and full traversal
// (gpu_full_bfs 274-323). The reference defers cascades past 200 touched vertices and can
// leave stale levels until one catch-up traversal at the end of the stream; here every
// batch ends with the exact BFS levels of the current graph:
//   A  invalidate: a vertex at level l > 0 stays valid while some neighbour at level l - 1
//      is valid; children (level l + 1) of every invalidated vertex are rechecked, so the
//      fixpoint is exactly the set of vertices that lost every shortest-path parent.
//   B  invalidated vertices restart at +inf and are seeded from their valid neighbours;
//      inserted edges seed their endpoints (levels only ever decrease from here).
//   C  relax rounds: atomicMin of level + 1 over the rows of every decreased vertex.
// All three phases run in one cooperative launch separated by a bounded grid barrier; rows
// longer than one queue item (2^chunk_log2 entries, 256 by default) are split into items so a
// hub spreads over warps.
//
// Two full traversals from the source replace the repair when the scheduler picks one
// (mode 1: top-down with a queue frontier; mode 2: direction-optimizing, the frontier kept
// as the level array itself and scanned bottom-up while it is large). Both write the new
// levels into a side array; a last pass stores and lists only the levels that changed, so
// the commit copies back the same entries whichever variant ran.
#include "ctx.cuh"
#include "bfs_dev.cuh"

namespace scout {

// At least four blocks per SM: the register budget this grants (64 per thread) holds the
// kernel without spills (the unconstrained build spilled to local memory at 40 registers).
__global__ void __launch_bounds__(BFS_THREADS, 4) k_bfs(BfsParams p) { bfs_body(p); }


// The kernel's parameters for the context's current batch (buffers ensured first).
int bfs_params(scout_ctx* c, int mode, const int* mode_dev, BfsParams* out) {
    SCOUT_RC(lists_ensure(c));
    if (!c->bfs_lv) SCOUT_RC(dev_alloc(c, (void**)&c->bfs_lv, (size_t)c->n * 4, "BFS traversal levels"));
    BfsParams& p = *out;
    p.g = dgraph(c);
    p.level = c->level;
    p.source = c->source;
    p.hkeys = c->d_hkeys;
    p.B = c->key_bits;
    for (int i = 0; i < 3; i++) p.q[i] = (unsigned long long*)c->d_qbuf[i];
    p.qcap = c->qcap;
    p.inval = c->d_list[1];
    p.touched = c->d_list[0];
    p.st_inval = c->stamp_a;
    p.st_touch = c->stamp_b;
    p.st_q = (uint32_t*)c->stamp_c;
    p.found = c->stamp_d;
    p.epoch = (int32_t)c->epoch;
    p.qtag0 = c->qtag;
    p.ctr = c->d_ctr;
    p.bar = c->d_bar;
    p.mode = mode;
    p.mode_dev = mode_dev;
    p.lv_new = c->bfs_lv;
    p.nnz_pre = c->nnz;
    p.sources = c->d_sources;
    p.nsrc = c->nsrc;
    p.chunk_log2 = c->tune_chunk_log2;
    p.max_share = c->tune_share > 0 ? c->tune_share : (1 << 20);
    p.chunk = 1 << p.chunk_log2;
    return SCOUT_OK;
}

static int bfs_launch(scout_ctx* c, int mode, const int* mode_dev, scout_batch_stats* st) {
    (void)st;
    BfsParams p;
    SCOUT_RC(bfs_params(c, mode, mode_dev, &p));
    void* args[] = {&p};
    return coop_launch(c, (const void*)k_bfs, BFS_THREADS, args, 0);
}

int bfs_repair(scout_ctx* c, int mode, const int* mode_dev, scout_batch_stats* st) {
    return bfs_launch(c, mode, mode_dev, st);
}
int bfs_recompute(scout_ctx* c, int32_t source, scout_batch_stats* st) {
    c->source = source;
    return bfs_launch(c, BFS_MODE_DIRECTION_OPT, nullptr, st);
}

}  // namespace scout
