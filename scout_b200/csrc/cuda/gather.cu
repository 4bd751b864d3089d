// gather.cu -- the fetch of batch K+1 while batch K repairs: the next batch's edits are copied
// to the device, and in the tiered store its cold rows are gathered into HBM, on a copy stream.
//
// The reference fetches the affected neighbourhoods of every batch from its mmap into pinned
// staging and copies them to the device (scout_mis.cu:500-627, scout_bfs.cu:199-229), and only
// its MIS engine prepares batch K+1 while batch K runs on the GPU (scout_mis.cu:855-912). Here
// the graph lives in HBM except for the tiered store's cold rows, which sit in mapped
// page-locked host memory and are read in place. scout_prefetch(next edits) makes the next
// scout_repair call, once its own merge is queued, copy the hinted edits to the device on a
// copy stream (a later scout_repair that declares them, scout_sched.prefetched, skips its own
// upload) and, in the tiered store, gather the rows of their endpoints that are still cold
// into free HBM, while its repair runs:
//   k_gather_plan   one thread per endpoint: a cold row seen for the first time in this gather
//                   (a stamp per vertex) takes space in the free HBM region by an atomic bump
//                   (lengths rounded up to 4 entries, so every copy starts 16-byte aligned);
//                   space beyond the region is not taken and the row stays cold
//   k_gather_copy   one warp per gathered row: the row is copied over the host link with
//                   coalesced loads, then, after a fence, its descriptor's start is switched
//                   to the HBM copy (len unchanged)
// A repair kernel running meanwhile reads either descriptor version of a gathered row: both
// hold the same entries (the host copy is only reclaimed by a later host-pool compaction on
// the main stream, and no merge runs until the gather has finished). The next batch's merge
// waits for the gather; the host then advances the HBM tail past the space the gather used.
#include "ctx.cuh"

#include <cstring>

namespace scout {

struct GatherCtr {
    int count;            // rows gathered
    int pad;
    unsigned long long bump;   // entries requested from the region (may exceed it)
    unsigned long long used;   // end of the last region slot actually taken
    unsigned long long bytes;  // bytes copied over the host link
};

constexpr int GATHER_THREADS = 256;

__global__ void k_gather_plan(const Row* __restrict__ row, int32_t n, const scout_edge* __restrict__ e, int64_t m,
                              long long hbm_cap, int32_t* __restrict__ stamp, int32_t tag, long long base,
                              long long room, int32_t* __restrict__ list, long long* __restrict__ dst,
                              GatherCtr* __restrict__ gc) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x - lane_id(); b < 2 * m;
         b += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = b + lane_id();
        bool take = false;
        int32_t x = -1;
        long long at = 0;
        int len = 0;
        if (i < 2 * m) {
            const scout_edge ed = e[i >> 1];
            x = (i & 1) ? ed.v : ed.u;
            if (x >= 0 && x < n) {   // the hint is not validated on the host
                const Row r = row[x];
                len = r.len;
                const bool cold = !(r.start >= 0 && r.start < hbm_cap) && len > 0;
                if (cold && atomicExch(stamp + x, tag) != tag) {
                    const long long need = ((long long)len + 3) & ~3LL;
                    at = (long long)atomicAdd(&gc->bump, (unsigned long long)need);
                    take = at + need <= room;
                    if (take) atomicMax(&gc->used, (unsigned long long)(at + need));
                }
            }
        }
        const int slot = warp_append(take, &gc->count);
        if (take) {
            list[slot] = x;
            dst[slot] = base + at;
        }
    }
}

__global__ void __launch_bounds__(GATHER_THREADS) k_gather_copy(Row* __restrict__ row, int32_t* __restrict__ pool,
                                                                const int32_t* __restrict__ list,
                                                                const long long* __restrict__ dst,
                                                                GatherCtr* __restrict__ gc) {
    const int cnt = ld_volatile(&gc->count);
    long long moved = 0;
    for (int k = gwarp_id(); k < cnt; k += gwarp_count()) {
        const int32_t x = list[k];
        const Row r = row[x];
        const int32_t* s = pool + r.start;
        int32_t* d = pool + dst[k];
        // four loads in flight per lane before their stores (reads cross the host link)
        constexpr int U = 4;
        for (int j0 = 0; j0 < r.len; j0 += U * WARP) {
            int32_t v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * WARP + (int)lane_id();
                v[u] = j < r.len ? s[j] : 0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * WARP + (int)lane_id();
                if (j < r.len) d[j] = v[u];
            }
        }
        moved += r.len;
        __syncwarp();
        __threadfence();   // the entries are visible before the descriptor points at them
        if (lane_id() == 0) {
            row[x].start = dst[k];
            row[x].cap = r.len;
        }
    }
    if (lane_id() == 0 && moved) atomicAdd(&gc->bytes, (unsigned long long)moved * 4);
}

// After the current batch's merge has been queued on the main stream: the hinted next batch's
// edits are copied to the device on the copy stream (ev_pf marks the end), and in the tiered
// store its endpoints' cold rows are then gathered into HBM from `base` (ev_gather0 /
// ev_gather1 bracket the copy and the gather). Both overlap the current batch's repair.
int prefetch_launch(scout_ctx* c, long long base) {
    c->gather_active = false;
    if (!c->pf_pending || c->pf_m == 0) { c->pf_pending = false; return SCOUT_OK; }
    c->pf_pending = false;
    const int64_t m = c->pf_m;
    SCOUT_RC(gather_reserve(c, m));
    cudaStream_t s = c->s_copy[1];
    // two slots: the merge just queued may read the latest one (when this batch was the
    // previous hint), so the new copy goes to the other, once the work queued so far is done
    const int slot = 1 - c->pf_slot;
    scout_edge* dst = c->d_pf_edits[slot];
    SCOUT_CU(c, cudaEventRecord(c->ev_copy[0], c->s_main));
    SCOUT_CU(c, cudaStreamWaitEvent(s, c->ev_copy[0], 0));
    if (c->tiered) SCOUT_CU(c, cudaEventRecord(c->ev_gather0, s));
    SCOUT_CU(c, cudaMemcpyAsync(dst, c->pf_host, (size_t)m * sizeof(scout_edge), cudaMemcpyHostToDevice, s));
    SCOUT_CU(c, cudaEventRecord(c->ev_pf, s));
    c->pf_slot = slot;
    c->pf_ready = true;
    c->pf_ready_m = m;
    const long long room = (long long)c->pool_cap - base - 4096;
    if (!c->tiered || room <= 0) return SCOUT_OK;
    SCOUT_CU(c, cudaMemsetAsync(c->d_gctr, 0, sizeof(GatherCtr), s));
    c->gather_tag = c->gather_tag + 1 == 0 ? 1 : c->gather_tag + 1;
    k_gather_plan<<<blocks_for(2 * m, GATHER_THREADS, c->sm_count), GATHER_THREADS, 0, s>>>(
        c->row, (int32_t)c->n, dst, m, (long long)c->pool_cap, c->gather_stamp, (int32_t)c->gather_tag, base, room,
        c->d_gather_list, c->d_gather_dst, (GatherCtr*)c->d_gctr);
    // one block per SM: the copy is bound by the host link, and the repair's persistent kernel
    // (up to four 256-thread blocks per SM) must still fit beside it to run concurrently
    k_gather_copy<<<c->sm_count, GATHER_THREADS, 0, s>>>(c->row, c->pool, c->d_gather_list, c->d_gather_dst,
                                                         (GatherCtr*)c->d_gctr);
    SCOUT_LAUNCH(c, "gather");
    c->nlaunch += 2;
    SCOUT_CU(c, cudaMemcpyAsync(c->h_gctr, c->d_gctr, sizeof(GatherCtr), cudaMemcpyDeviceToHost, s));
    SCOUT_CU(c, cudaEventRecord(c->ev_gather1, s));
    c->gather_base = base;
    c->gather_active = true;
    return SCOUT_OK;
}

// Buffers a prefetch of batches of up to max_edits edits needs, allocated now: the device copy
// of the hinted edits, and in the tiered store the gather's stamps, counters and lists.
int gather_reserve(scout_ctx* c, int64_t max_edits) {
    if (max_edits <= 0) return SCOUT_OK;
    for (int i = 0; i < 2; i++)
        SCOUT_RC(dev_grow(c, &c->d_pf_edits[i], &c->cap_pf_edits[i], max_edits, "prefetched edits"));
    if (!c->tiered) return SCOUT_OK;
    if (!c->gather_stamp) {
        SCOUT_RC(dev_alloc(c, (void**)&c->gather_stamp, (size_t)c->n * 4, "gather stamps"));
        SCOUT_CU(c, cudaMemsetAsync(c->gather_stamp, 0, (size_t)c->n * 4, c->s_main));
    }
    if (!c->d_gctr) {
        SCOUT_RC(dev_alloc(c, (void**)&c->d_gctr, sizeof(GatherCtr), "gather counters"));
        SCOUT_CU(c, cudaMallocHost((void**)&c->h_gctr, sizeof(GatherCtr)));
    }
    SCOUT_RC(dev_grow(c, &c->d_gather_list, &c->cap_gather_list, 2 * max_edits, "gather list"));
    SCOUT_RC(dev_grow(c, &c->d_gather_dst, &c->cap_gather_dst, 2 * max_edits, "gather destinations"));
    return SCOUT_OK;
}

// Before a batch's merge: the main stream waits for a gather in flight and the HBM tail moves
// past the space it used. Returns the gather's duration and bytes through the outputs.
int gather_finish(scout_ctx* c, double* ms, int64_t* rows, int64_t* bytes) {
    if (ms) *ms = 0;
    if (rows) *rows = 0;
    if (bytes) *bytes = 0;
    if (!c->gather_active) return SCOUT_OK;
    c->gather_active = false;
    SCOUT_CU(c, cudaEventSynchronize(c->ev_gather1));
    SCOUT_CU(c, cudaStreamWaitEvent(c->s_main, c->ev_gather1, 0));
    const GatherCtr* g = (const GatherCtr*)c->h_gctr;
    const long long end = c->gather_base + (long long)g->used;
    if (end > c->tail) c->tail = end;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, c->ev_gather0, c->ev_gather1) != cudaSuccess) { cudaGetLastError(); t = 0.f; }
    if (ms) *ms = t;
    if (rows) *rows = g->count;
    if (bytes) *bytes = (int64_t)g->bytes;
    c->gathered_rows += g->count;
    c->gathered_bytes += (int64_t)g->bytes;
    return SCOUT_OK;
}

}  // namespace scout

using namespace scout;

extern "C" int scout_prefetch(scout_ctx* c, const scout_edge* next, int64_t m) {
    if (!c || m < 0 || (m > 0 && !next)) return c ? c->fail(SCOUT_E_INVALID, "bad arguments") : SCOUT_E_INVALID;
    c->pf_pending = false;
    c->pf_m = 0;
    // the copy stream may still read the previous hint's edits (from the staging buffer
    // overwritten below) or gather its rows; a copy already made stays usable
    if (c->gather_active) SCOUT_CU(c, cudaEventSynchronize(c->ev_gather1));
    if (c->pf_ready) SCOUT_CU(c, cudaEventSynchronize(c->ev_pf));
    if (m == 0) return SCOUT_OK;
    cudaPointerAttributes at;
    const bool pinned = cudaPointerGetAttributes(&at, next) == cudaSuccess && at.type == cudaMemoryTypeHost;
    if (!pinned) cudaGetLastError();
    if (pinned) {
        c->pf_host = next;   // read in place by the copy: unchanged until the repair that uses it
    } else {
        SCOUT_RC(pin_grow(c, &c->h_pf_edits, &c->cap_h_pf_edits, m * (int64_t)sizeof(scout_edge)));
        stage_copy(c->h_pf_edits, next, (size_t)m * sizeof(scout_edge));
        c->pf_host = (const scout_edge*)c->h_pf_edits;
    }
    c->pf_m = m;
    c->pf_pending = true;
    return SCOUT_OK;
}
