// fetch_host.cpp -- fetch pipeline: rows of the hybrid graph (mmap'd base + scratchpad)
// are read by OpenMP workers into host staging in chunks bounded by cumulative degree
// (core/chunking.h:20-32) and handed to scout_stage_rows, alternating the two copy slots so
// the next chunk is read while the previous one is in flight (scout_cc.cu:160-215).
#include "host.hpp"

#include <algorithm>
#include <vector>

namespace scout {

static int stage_range(HGraph& g, scout_ctx* ctx, const int32_t* ids, int64_t k, int64_t slab_elems) {
    std::vector<int64_t> deg((size_t)k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < k; i++) deg[i] = g.degree(ids[i]);
    std::vector<int64_t> off;
    std::vector<int32_t> elems;
    int slot = 0;
    int64_t i = 0;
    while (i < k) {
        int64_t j = i, sum = 0;
        while (j < k && (j == i || sum + deg[j] <= slab_elems)) sum += deg[j++];
        off.assign((size_t)(j - i + 1), 0);
        for (int64_t t = i; t < j; t++) off[t - i + 1] = off[t - i] + deg[t];
        elems.resize((size_t)sum);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t t = i; t < j; t++) g.neighbors_write(ids[t], elems.data() + off[t - i]);
        int rc = scout_stage_rows(ctx, slot, ids + i, off.data(), elems.data(), j - i, sum);
        if (rc != SCOUT_OK) return rc;
        slot ^= 1;
        i = j;
    }
    return SCOUT_OK;
}

}  // namespace scout

using namespace scout;

extern "C" {

int scout_fetch_all(scout_hgraph* h, scout_ctx* ctx, int64_t slab_elems) {
    if (!h || !ctx) return host_fail(SCOUT_E_INVALID, "null argument");
    if (slab_elems <= 0) slab_elems = 1 << 24;
    const int64_t n = h->g.nodes();
    int64_t nnz = 0;
#pragma omp parallel for reduction(+ : nnz)
    for (int64_t v = 0; v < n; v++) nnz += h->g.degree((int32_t)v);
    int rc = scout_graph_reserve(ctx, n, nnz);
    if (rc != SCOUT_OK) return rc;
    std::vector<int32_t> ids((size_t)n);
    for (int64_t v = 0; v < n; v++) ids[v] = (int32_t)v;
    rc = stage_range(h->g, ctx, ids.data(), n, slab_elems);
    if (rc != SCOUT_OK) return rc;
    return scout_graph_seal(ctx);
}

int scout_fetch_rows(scout_hgraph* h, scout_ctx* ctx, const int32_t* ids, int64_t k) {
    if (!h || !ctx || (k > 0 && !ids)) return host_fail(SCOUT_E_INVALID, "null argument");
    for (int64_t i = 0; i < k; i++)
        if (ids[i] < 0 || ids[i] >= h->g.nodes()) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    int rc = stage_range(h->g, ctx, ids, k, 1 << 24);
    if (rc != SCOUT_OK) return rc;
    return scout_graph_seal(ctx);
}

}  // extern "C"
