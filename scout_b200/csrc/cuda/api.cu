// api.cu -- the C ABI of scout_gpu.h: context, graph store, state, repair dispatch, commit.
#include "ctx.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>

namespace scout {

int host_fail(int code, const std::string& msg);   // graph_host.cpp (thread-local message)
const char* host_last_error();

int cuda_fail(scout_ctx* c, cudaError_t e, const char* where) {
    std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
    if (c) c->err = msg;
    else host_fail(SCOUT_E_CUDA, msg);
    return SCOUT_E_CUDA;
}

int dev_alloc(scout_ctx* c, void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (bytes == 0) bytes = 256;
    if (c->held + bytes > c->budget)
        return c->fail(SCOUT_E_CAPACITY, std::string("HBM budget exceeded allocating ") + what + " (" +
                                             std::to_string(bytes) + " B, held " + std::to_string(c->held) +
                                             " of " + std::to_string(c->budget) + ")");
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return c->fail(e == cudaErrorMemoryAllocation ? SCOUT_E_CAPACITY : SCOUT_E_CUDA,
                       std::string("cudaMalloc failed for ") + what + ": " + cudaGetErrorString(e));
    }
    c->held += bytes;
    return SCOUT_OK;
}

void dev_free(scout_ctx* c, void* p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    if (bytes == 0) bytes = 256;
    c->held -= std::min<uint64_t>(c->held, bytes);
}

int pin_grow(scout_ctx* c, void** p, int64_t* cap, int64_t need) {
    if (*p && *cap >= need) return SCOUT_OK;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    int64_t nc = need + need / 4 + 4096;
    SCOUT_CU(c, cudaMallocHost(p, (size_t)nc));
    *cap = nc;
    return SCOUT_OK;
}

int coop_launch(scout_ctx* c, const void* fn, int threads, void** args, size_t smem) {
    int per_sm = 0;
    SCOUT_CU(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) return c->fail(SCOUT_E_CUDA, "persistent kernel does not fit on an SM");
    per_sm = std::min(per_sm, c->tune_blocks_per_sm > 0 ? c->tune_blocks_per_sm : 4);
    dim3 grid((unsigned)(per_sm * c->sm_count)), block((unsigned)threads);
    // the grid barrier's arrival counter starts every launch at zero (its error flag persists
    // until the batch's counters are read)
    SCOUT_CU(c, cudaMemsetAsync(&c->d_bar->count, 0, sizeof(unsigned int), c->s_main));
    SCOUT_CU(c, cudaLaunchCooperativeKernel(fn, grid, block, args, smem, c->s_main));
    c->nlaunch += 1;
    return SCOUT_OK;
}

static void release(scout_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->s_main) cudaStreamSynchronize(c->s_main);
    for (int i = 0; i < 2; i++) if (c->s_copy[i]) cudaStreamSynchronize(c->s_copy[i]);
    sched_release(c);
    if (c->host_pool) { cudaFreeHost(c->host_pool); c->host_pool = nullptr; }
    void* devs[] = {c->row, c->pool, c->spare, c->level, c->color, c->label, c->mis, c->stamp_a, c->stamp_b, c->stamp_c, c->stamp_d,
                    c->aux_v, c->aux_w, c->ws, c->d_qbuf[0], c->d_qbuf[1], c->d_qbuf[2], c->d_list[0], c->d_list[1],
                    c->d_commit, c->d_sort_hist, c->d_scan_tmp, c->d_slices, c->d_coff, c->d_misc, c->d_cc, c->bfs_lv, c->d_sources, c->d_ctr, c->d_bar, c->d_flags, c->d_stage_ids[0],
                    c->d_stage_ids[1], c->d_stage_off[0], c->d_stage_off[1]};
    for (void* p : devs) if (p) cudaFree(p);
    void* hosts[] = {c->h_ctr, c->h_bar, c->h_pin_edits, c->h_pin_commit, c->h_slab[0], c->h_slab[1],
                     c->h_slab_off[0], c->h_slab_off[1], c->h_slab_ids[0], c->h_slab_ids[1]};
    for (void* p : hosts) if (p) cudaFreeHost(p);
    for (int i = 0; i < 8; i++) if (c->ev_t[i]) cudaEventDestroy(c->ev_t[i]);
    if (c->ev_gather0) cudaEventDestroy(c->ev_gather0);
    if (c->ev_gather1) cudaEventDestroy(c->ev_gather1);
    if (c->ev_pf) cudaEventDestroy(c->ev_pf);
    if (c->ev_union) cudaEventDestroy(c->ev_union);
    void* gdev[] = {c->gather_stamp, c->d_gctr, c->d_pf_edits[0], c->d_pf_edits[1], c->d_gather_list, c->d_gather_dst};
    for (void* p : gdev) if (p) cudaFree(p);
    if (c->h_gctr) cudaFreeHost(c->h_gctr);
    if (c->h_pf_edits) cudaFreeHost(c->h_pf_edits);
    for (int i = 0; i < 2; i++) {
        if (c->ev_copy[i]) cudaEventDestroy(c->ev_copy[i]);
        if (c->s_copy[i]) cudaStreamDestroy(c->s_copy[i]);
    }
    if (c->s_main) cudaStreamDestroy(c->s_main);
    delete c;
}

static int32_t** state_slot(scout_ctx* c, int problem) {
    switch (problem) {
    case SCOUT_MIS: return &c->mis;
    case SCOUT_COLORING: return &c->color;
    case SCOUT_BFS: return &c->level;
    case SCOUT_CC: return &c->label;
    default: return nullptr;
    }
}

__global__ void k_label_min(const int32_t* __restrict__ lab, int32_t* __restrict__ mn, int64_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        atomicMin(&mn[lab[v]], (int32_t)v);
}
__global__ void k_label_apply(int32_t* __restrict__ lab, const int32_t* __restrict__ mn, int64_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        lab[v] = mn[lab[v]];
}
__global__ void k_fill_i32(int32_t* __restrict__ a, int64_t n, int32_t x) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        a[v] = x;
}

// (id, value) pairs of the touched list for the commit.
__global__ void k_commit_gather(const int32_t* __restrict__ list, const DevCounters* __restrict__ ctr,
                                const int32_t* __restrict__ val, int32_t* __restrict__ out) {
    const int cnt = ctr->changed;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        int32_t v = list[i];
        out[2 * i] = v;
        out[2 * i + 1] = val[v];
    }
}

static double ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { cudaGetLastError(); return 0.0; }
    return (double)ms;
}

}  // namespace scout

using namespace scout;

extern "C" {

const char* scout_last_error(const scout_ctx* c) { return c ? c->err.c_str() : host_last_error(); }

int scout_device_count(int* out) {
    if (!out) return SCOUT_E_INVALID;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { cudaGetLastError(); n = 0; }
    *out = n;
    return SCOUT_OK;
}

int scout_ctx_create(int device, uint64_t budget, scout_ctx** out) {
    if (!out) return host_fail(SCOUT_E_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return host_fail(SCOUT_E_NODEV, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return host_fail(SCOUT_E_INVALID, "device id out of range");
    auto* c = new scout_ctx();
    c->device = device;
    // gpu_warmup_and_device_setup (cli_setup.h:54-58)
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaFree(0);
    cudaDeviceProp prop;
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) { release(c); return cuda_fail(nullptr, e, "device setup"); }
    std::strncpy(c->name, prop.name, sizeof(c->name) - 1);
    c->sm_count = prop.multiProcessorCount;
    if (!prop.cooperativeLaunch) { release(c); return host_fail(SCOUT_E_NODEV, "device lacks cooperative launch"); }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = budget ? budget : (uint64_t)(0.9 * (double)fr);
    bool ok = cudaStreamCreateWithFlags(&c->s_main, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; i < 2 && ok; i++) {
        ok = cudaStreamCreateWithFlags(&c->s_copy[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->ev_copy[i], cudaEventDisableTiming) == cudaSuccess;
    }
    for (int i = 0; i < 8 && ok; i++) ok = cudaEventCreate(&c->ev_t[i]) == cudaSuccess;
    ok = ok && cudaEventCreate(&c->ev_gather0) == cudaSuccess && cudaEventCreate(&c->ev_gather1) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_pf, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_union, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaMallocHost((void**)&c->h_ctr, sizeof(DevCounters)) == cudaSuccess &&
         cudaMallocHost((void**)&c->h_bar, sizeof(GridBar)) == cudaSuccess;
    if (!ok) { cudaError_t le = cudaGetLastError(); release(c); return cuda_fail(nullptr, le, "context streams"); }
    int rc = dev_alloc(c, (void**)&c->d_ctr, sizeof(DevCounters), "counters");
    if (rc == SCOUT_OK) rc = dev_alloc(c, (void**)&c->d_bar, sizeof(GridBar), "grid barrier");
    if (rc == SCOUT_OK) rc = dev_alloc(c, (void**)&c->d_flags, 64, "error flags");
    if (rc != SCOUT_OK) { std::string m = c->err; release(c); return host_fail(rc, m); }
    cudaMemset(c->d_ctr, 0, sizeof(DevCounters));
    cudaMemset(c->d_bar, 0, sizeof(GridBar));
    cudaMemset(c->d_flags, 0, 64);
    std::memset(c->h_ctr, 0, sizeof(DevCounters));   // scout_sched_last before any repair reads it
    std::memset(c->h_bar, 0, sizeof(GridBar));
    *out = c;
    return SCOUT_OK;
}

int scout_ctx_destroy(scout_ctx* c) { release(c); return SCOUT_OK; }

int scout_ctx_info(scout_ctx* c, char* name, int cap, uint64_t* held) {
    if (!c) return SCOUT_E_INVALID;
    if (name && cap > 0) { std::strncpy(name, c->name, (size_t)cap - 1); name[cap - 1] = 0; }
    if (held) *held = c->held;
    return SCOUT_OK;
}

// ---- state -------------------------------------------------------------------------------
int scout_state_upload(scout_ctx* c, int problem, const int32_t* sol, int64_t n) {
    if (!c || !sol) return SCOUT_E_INVALID;
    int32_t** slot = state_slot(c, problem);
    if (!slot) return c->fail(SCOUT_E_INVALID, "unknown problem");
    if (!c->reserved || n != c->n) return c->fail(SCOUT_E_STATE, "state size does not match the graph");
    if (problem == SCOUT_CC)
        for (int64_t v = 0; v < n; v++)
            if (sol[v] < 0 || sol[v] >= n) return c->fail(SCOUT_E_INVALID, "component labels must lie in [0, n)");
    cudaSetDevice(c->device);
    if (!*slot) SCOUT_RC(dev_alloc(c, (void**)slot, (size_t)n * 4, "solution state"));
    SCOUT_CU(c, cudaMemcpyAsync(*slot, sol, (size_t)n * 4, cudaMemcpyHostToDevice, c->s_main));
    if (problem == SCOUT_CC) {   // min-vertex-id labels
        SCOUT_RC(graph_ensure_scratch(c));
        k_fill_i32<<<blocks_for(n, 256), 256, 0, c->s_main>>>(c->aux_v, n, INT32_MAX);
        k_label_min<<<blocks_for(n, 256), 256, 0, c->s_main>>>(*slot, c->aux_v, n);
        k_label_apply<<<blocks_for(n, 256), 256, 0, c->s_main>>>(*slot, c->aux_v, n);
        SCOUT_LAUNCH(c, "label canonicalisation");
    }
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    return SCOUT_OK;
}

int scout_state_download(scout_ctx* c, int problem, int32_t* out, int64_t n) {
    if (!c || !out) return SCOUT_E_INVALID;
    int32_t** slot = state_slot(c, problem);
    if (!slot) return c->fail(SCOUT_E_INVALID, "unknown problem");
    if (!*slot || n != c->n) return c->fail(SCOUT_E_STATE, "no state uploaded for this problem");
    cudaSetDevice(c->device);
    SCOUT_CU(c, cudaMemcpyAsync(out, *slot, (size_t)n * 4, cudaMemcpyDeviceToHost, c->s_main));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    return SCOUT_OK;
}

int scout_set_source(scout_ctx* c, int32_t s) {
    if (!c) return SCOUT_E_INVALID;
    if (s < 0 || (c->reserved && s >= c->n)) return c->fail(SCOUT_E_INVALID, "source out of range");
    c->source = s;
    return SCOUT_OK;
}

}  // extern "C"

// ---- repair ------------------------------------------------------------------------------
namespace scout {

// Repair variant a plain (non-learned) schedule asks for: BFS 0 incremental, 1 top-down
// traversal, 2 direction-optimizing traversal; CC 0 incremental, 1 recompute of every class
// (2, recompute of the touched classes, is the scheduler's).
static int plain_variant(int problem, const scout_sched& sd) {
    if (sd.mode != SCOUT_MODE_RECOMPUTE) return 0;
    if (problem == SCOUT_BFS) return sd.frontier == SCOUT_FRONTIER_QUEUE ? BFS_MODE_TOP_DOWN : BFS_MODE_DIRECTION_OPT;
    if (problem == SCOUT_CC) return 1;
    return 0;
}

static int run_repair(scout_ctx* c, int problem, const scout_sched& sd, int variant, const int* mode_dev,
                      scout_batch_stats* st) {
    switch (problem) {
    case SCOUT_BFS: return bfs_repair(c, variant, mode_dev, st);
    case SCOUT_CC: return cc_repair(c, &sd, variant, mode_dev, st);
    case SCOUT_COLORING: return coloring_repair(c, st);
    case SCOUT_MIS: return mis_repair(c, st);
    }
    return c->fail(SCOUT_E_INVALID, "unknown problem");
}

// The pool tails after a batch's merge (where its rewritten rows went).
static void advance_tails(scout_ctx* c, const DevCounters& h) {
    if (c->batch_dest == 1) c->host_tail += h.new_elems;
    else c->tail += h.new_elems;
    if (c->batch_dest == 2) c->host_tail += h.new_elems_host;
}

// Batch statistics from the counters of the last repair run (already fetched).
static void fill_stats(scout_ctx* c, scout_batch_stats* st, int64_t launch0) {
    const DevCounters& h = *c->h_ctr;
    st->edits = h.n_ins + h.n_del;
    st->insertions = h.n_ins;
    st->deletions = h.n_del;
    st->noop = h.noop;
    st->conflicts = h.conflicts;
    st->affected = h.affected;
    st->changed = h.changed;
    st->rounds = h.rounds;
    st->recomputes += h.recomputes;
    st->splits = h.splits;
    st->searches = h.searches;
    st->ins_effective = c->last_problem == SCOUT_COLORING ? h.conflicts : h.ins_eff;
    st->del_effective = c->last_problem == SCOUT_CC ? h.splits : h.del_eff;
    st->hbm_bytes = h.hbm_bytes;
    st->update_bytes = h.update_bytes;
    st->d2h_bytes += sizeof(DevCounters);
    st->ms_compact = ev_ms(c->ev_t[6], c->ev_t[7]);
    st->ms_h2d = ev_ms(c->ev_t[7], c->ev_t[3]);
    st->ms_update = ev_ms(c->ev_t[3], c->ev_t[1]);
    st->compactions = c->compactions;
    st->launches = c->nlaunch - launch0;
    for (int i = 0; i < 4; i++) {
        unsigned long long a = h.phase_ns[i], b = h.phase_ns[i + 1];
        st->phase_ms[i] = (a && b && b >= a) ? (double)(b - a) / 1e6 : 0.0;
    }
    c->last_changed = h.changed;
}

// Common prologue of a batch: validation, counters, classification + merge of the edits.
// Tuning knobs of a call: persistent-kernel blocks per SM (1..4, 0 = as many as fit) and the
// BFS queue item size (2^8 .. 2^13 row entries, 0 = 2^8).
static int apply_tuning(scout_ctx* c, const scout_sched& sd) {
    if (sd.blocks_per_sm < 0 || sd.blocks_per_sm > 4) return c->fail(SCOUT_E_INVALID, "blocks_per_sm must be 0..4");
    if (sd.chunk_log2 != 0 && (sd.chunk_log2 < 8 || sd.chunk_log2 > 13))
        return c->fail(SCOUT_E_INVALID, "chunk_log2 must be 0 or 8..13");
    const int lpv = sd.lanes_per_vertex;
    if (!(lpv == 0 || lpv == 32 || lpv == 64 || lpv == 128 || lpv == 256 || lpv == 1024))
        return c->fail(SCOUT_E_INVALID, "lanes_per_vertex must be 0, 32, 64, 128, 256 or 1024");
    if (sd.frontier < SCOUT_FRONTIER_AUTO || sd.frontier > SCOUT_FRONTIER_BITMAP)
        return c->fail(SCOUT_E_INVALID, "unknown frontier mode");
    c->tune_blocks_per_sm = sd.blocks_per_sm;
    // defaults: the autotuner's choice on a B200 (R-MAT scale 22 stream): 256-entry queue items,
    // at most two warps sharing one
    c->tune_chunk_log2 = sd.chunk_log2 ? sd.chunk_log2 : 8;
    c->tune_share = (lpv ? lpv : 64) / 32;
    return SCOUT_OK;
}

static int batch_prologue(scout_ctx* c, int problem, const scout_edge* edits, const uint8_t* ops, int64_t m,
                          scout_batch_stats* st) {
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    int32_t** slot = state_slot(c, problem);
    if (!slot) return c->fail(SCOUT_E_INVALID, "unknown problem");
    if (!*slot) return c->fail(SCOUT_E_STATE, "no state uploaded for this problem");
    cudaSetDevice(c->device);
    std::memset(st, 0, sizeof(*st));
    // the gather of this batch's cold rows, hinted by scout_prefetch and run during the previous
    // repair, completes before the merge
    SCOUT_RC(gather_finish(c, &st->ms_gather, &st->gather_rows, &st->gather_bytes));
    c->last_problem = problem;
    SCOUT_RC(batch_begin(c));
    SCOUT_RC(lists_ensure(c));
    c->epoch++;
    SCOUT_CU(c, cudaEventRecord(c->ev_t[0], c->s_main));
    SCOUT_RC(graph_update(c, edits, ops, m, st));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[1], c->s_main));
    return SCOUT_OK;
}

// (id, value) pairs of the last repair's touched entries, gathered on the device and copied
// into the context's page-locked buffer (*pairs points there until the next call).
int commit_gather(scout_ctx* c, int problem, const int32_t** pairs, int64_t* count) {
    int32_t** slot = state_slot(c, problem);
    if (!slot || !*slot) return c->fail(SCOUT_E_STATE, "nothing to commit for this problem");
    if (problem != c->last_problem) return c->fail(SCOUT_E_STATE, "the last repair was for another problem");
    cudaSetDevice(c->device);
    const int64_t cnt = c->last_changed;
    *pairs = nullptr;
    *count = 0;
    if (cnt > 0) {
        SCOUT_RC(pin_grow(c, &c->h_pin_commit, &c->cap_pin_commit, cnt * 8));
        k_commit_gather<<<blocks_for(cnt, 256), 256, 0, c->s_main>>>(c->d_list[0], c->d_ctr, *slot, c->d_commit);
        SCOUT_LAUNCH(c, "k_commit_gather");
        c->nlaunch += 1;
        SCOUT_CU(c, cudaMemcpyAsync(c->h_pin_commit, c->d_commit, (size_t)cnt * 8, cudaMemcpyDeviceToHost, c->s_main));
        SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
        *pairs = (const int32_t*)c->h_pin_commit;
        *count = cnt;
    }
    c->last_changed = 0;
    return SCOUT_OK;
}

__global__ void k_count_diff(const int32_t* __restrict__ a, const int32_t* __restrict__ b, int64_t n,
                             unsigned long long* __restrict__ cnt) {
    unsigned long long d = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        d += a[v] != b[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(cnt, d);
}

// One round of several union stores of distinct problems (ne <= 4, one device): every batch is
// merged on its store's stream, then ONE cooperative launch runs all the repairs (union.cu),
// then each store's counters are read into its stats (ms_repair: the shared launch). The
// repairs run their plain variants; the learned scheduler decides per launch and is not used.
int union_run(scout_ctx* const* cs, const int* problems, const scout_edge* const* edits, const uint8_t* const* ops,
              const int64_t* counts, int ne, const scout_sched* sched, scout_batch_stats* stats) {
    if (ne < 1 || ne > 4 || !cs || !problems || !edits || !counts || !stats) return host_fail(SCOUT_E_INVALID, "bad round arguments");
    for (int i = 0; i < ne; i++) {
        if (!cs[i]) return host_fail(SCOUT_E_INVALID, "null engine");
        if (cs[i]->device != cs[0]->device) return cs[i]->fail(SCOUT_E_INVALID, "the engines of a fused round share one device");
        for (int j = 0; j < i; j++)
            if (problems[j] == problems[i] || cs[j] == cs[i])
                return cs[i]->fail(SCOUT_E_INVALID, "a fused round takes one engine per problem");
        if (counts[i] < 0 || (counts[i] > 0 && !edits[i])) return cs[i]->fail(SCOUT_E_INVALID, "bad batch");
    }
    auto t0 = std::chrono::steady_clock::now();
    scout_sched sds[4];
    int variants[4];
    int64_t launch0[4];
    for (int i = 0; i < ne; i++) {
        std::memset(&sds[i], 0, sizeof(scout_sched));
        if (sched) sds[i] = *sched;
        sds[i].policy = SCOUT_SCHED_PLAIN;
        SCOUT_RC(apply_tuning(cs[i], sds[i]));
        launch0[i] = cs[i]->nlaunch;
        SCOUT_RC(batch_prologue(cs[i], problems[i], edits[i], ops ? ops[i] : nullptr, counts[i], &stats[i]));
        variants[i] = plain_variant(problems[i], sds[i]);
    }
    SCOUT_RC(union_launch(cs, problems, sds, variants, ne));
    for (int i = 0; i < ne; i++) {
        scout_ctx* c = cs[i];
        SCOUT_CU(c, cudaEventRecord(c->ev_t[2], c->s_main));
        SCOUT_RC(counters_fetch(c));
        const DevCounters& h = *c->h_ctr;
        advance_tails(c, h);
        c->nnz += h.nnz_delta;
        c->qtag += (uint32_t)h.rounds + 8;
        fill_stats(c, &stats[i], launch0[i]);
        stats[i].variant = variants[i];
    }
    const double ms = ev_ms(cs[0]->ev_t[4], cs[0]->ev_t[5]);
    const double total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < ne; i++) {
        stats[i].ms_repair = ms;
        stats[i].ms_total = total;
        cs[i]->prev_repair_ms[problems[i]] = ms;
    }
    return SCOUT_OK;
}

}  // namespace scout

extern "C" {

int scout_repair(scout_ctx* c, int problem, const scout_edge* edits, const uint8_t* ops, int64_t m,
                 const scout_sched* sched, scout_batch_stats* st) {
    if (!c || m < 0 || (m > 0 && !edits)) return c ? c->fail(SCOUT_E_INVALID, "bad arguments") : SCOUT_E_INVALID;
    auto t0 = std::chrono::steady_clock::now();
    scout_batch_stats local;
    if (!st) st = &local;
    scout_sched sd;
    std::memset(&sd, 0, sizeof(sd));
    if (sched) sd = *sched;
    SCOUT_RC(apply_tuning(c, sd));
    const int64_t launch0 = c->nlaunch;
    c->pf_use = sd.prefetched != 0;
    const int prc = batch_prologue(c, problem, edits, ops, m, st);
    c->pf_use = false;
    SCOUT_RC(prc);
    // the hinted next batch: its edits' copy (and, tiered, its cold rows' gather) during this repair
    SCOUT_RC(prefetch_launch(c, c->merge_tail));
    const int* mode_dev = nullptr;
    const int variant = plain_variant(problem, sd);
    if (sd.policy == SCOUT_SCHED_LEARNED && sched_variants(problem) > 1)
        SCOUT_RC(sched_decide(c, problem, m, true, &mode_dev));
    SCOUT_RC(run_repair(c, problem, sd, variant, mode_dev, st));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[2], c->s_main));
    SCOUT_RC(counters_fetch(c));
    const DevCounters& h = *c->h_ctr;
    advance_tails(c, h);
    c->nnz += h.nnz_delta;
    c->qtag += (uint32_t)h.rounds + 8;
    fill_stats(c, st, launch0);
    st->variant = mode_dev ? h.decision : variant;
    st->ms_repair = ev_ms(c->ev_t[1], c->ev_t[2]);
    c->prev_repair_ms[problem] = st->ms_repair;
    st->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SCOUT_OK;
}

int scout_repair_probe(scout_ctx* c, int problem, const scout_edge* edits, const uint8_t* ops, int64_t m,
                       const scout_sched* sched, double* variant_ms, float* features, scout_batch_stats* st) {
    if (!c || m < 0 || (m > 0 && !edits) || !variant_ms)
        return c ? c->fail(SCOUT_E_INVALID, "bad arguments") : SCOUT_E_INVALID;
    const int nv = sched_variants(problem);
    if (nv < 2) return c->fail(SCOUT_E_INVALID, "the probe applies to BFS and CC only");
    auto t0 = std::chrono::steady_clock::now();
    scout_batch_stats local;
    if (!st) st = &local;
    scout_sched sd;
    std::memset(&sd, 0, sizeof(sd));
    if (sched) sd = *sched;
    SCOUT_RC(apply_tuning(c, sd));
    const int64_t launch0 = c->nlaunch;
    SCOUT_RC(batch_prologue(c, problem, edits, ops, m, st));
    const int* unused = nullptr;
    SCOUT_RC(sched_decide(c, problem, m, false, &unused));
    const int64_t n = c->n;
    if (!c->probe_buf) SCOUT_RC(dev_alloc(c, (void**)&c->probe_buf, (size_t)(2 * n + 64) * 4, "probe buffers"));
    if (!c->d_ctr_snap) SCOUT_RC(dev_alloc(c, (void**)&c->d_ctr_snap, sizeof(DevCounters), "probe counters"));
    int32_t* state = *state_slot(c, problem);
    int32_t* pre = c->probe_buf;
    int32_t* ref = c->probe_buf + n;
    unsigned long long* d_diff = (unsigned long long*)(c->probe_buf + 2 * n);
    SCOUT_CU(c, cudaMemcpyAsync(c->d_ctr_snap, c->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToDevice, c->s_main));
    SCOUT_CU(c, cudaMemcpyAsync(pre, state, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->s_main));
    // variant 0 (the incremental repair) runs last, so the batch ends in its state and its
    // touched list is the one the commit reads
    int order[3];
    for (int i = 0; i < nv; i++) order[i] = (i + 1) % nv;
    double best = 1e300;
    for (int i = 0; i < nv; i++) {
        const int v = order[i];
        if (i > 0) {
            SCOUT_CU(c, cudaMemcpyAsync(c->d_ctr, c->d_ctr_snap, sizeof(DevCounters), cudaMemcpyDeviceToDevice,
                                        c->s_main));
            SCOUT_CU(c, cudaMemcpyAsync(state, pre, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->s_main));
            SCOUT_CU(c, cudaMemsetAsync(c->d_bar, 0, sizeof(GridBar), c->s_main));
            c->epoch++;
        }
        SCOUT_CU(c, cudaEventRecord(c->ev_t[4], c->s_main));
        SCOUT_RC(run_repair(c, problem, sd, v, nullptr, st));
        SCOUT_CU(c, cudaEventRecord(c->ev_t[5], c->s_main));
        SCOUT_RC(counters_fetch(c));
        variant_ms[v] = ev_ms(c->ev_t[4], c->ev_t[5]);
        best = std::min(best, variant_ms[v]);
        c->qtag += (uint32_t)c->h_ctr->rounds + 8;
        if (i == 0) {
            SCOUT_CU(c, cudaMemcpyAsync(ref, state, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->s_main));
        } else {
            SCOUT_CU(c, cudaMemsetAsync(d_diff, 0, 8, c->s_main));
            k_count_diff<<<blocks_for(n, 256), 256, 0, c->s_main>>>(state, ref, n, d_diff);
            SCOUT_LAUNCH(c, "k_count_diff");
            unsigned long long diff = 0;
            SCOUT_CU(c, cudaMemcpyAsync(&diff, d_diff, 8, cudaMemcpyDeviceToHost, c->s_main));
            SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
            if (diff)
                return c->fail(SCOUT_E_STATE, "repair variants disagree on " + std::to_string(diff) + " vertices");
        }
    }
    for (int v = nv; v < 3; v++) variant_ms[v] = -1.0;
    const DevCounters& h = *c->h_ctr;
    advance_tails(c, h);
    c->nnz += h.nnz_delta;
    fill_stats(c, st, launch0);
    st->variant = 0;
    st->ms_repair = variant_ms[0];
    if (features) for (int i = 0; i < 24; i++) features[i] = h.feat[i];
    c->prev_repair_ms[problem] = best;
    st->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SCOUT_OK;
}

int scout_repair_mis(scout_ctx* c, const scout_edge* e, const uint8_t* o, int64_t m, const scout_sched* s, scout_batch_stats* st) { return scout_repair(c, SCOUT_MIS, e, o, m, s, st); }
int scout_repair_coloring(scout_ctx* c, const scout_edge* e, const uint8_t* o, int64_t m, const scout_sched* s, scout_batch_stats* st) { return scout_repair(c, SCOUT_COLORING, e, o, m, s, st); }
int scout_repair_bfs(scout_ctx* c, const scout_edge* e, const uint8_t* o, int64_t m, const scout_sched* s, scout_batch_stats* st) { return scout_repair(c, SCOUT_BFS, e, o, m, s, st); }
int scout_repair_cc(scout_ctx* c, const scout_edge* e, const uint8_t* o, int64_t m, const scout_sched* s, scout_batch_stats* st) { return scout_repair(c, SCOUT_CC, e, o, m, s, st); }

int scout_commit(scout_ctx* c, int problem, int32_t* mirror, int64_t n, int64_t* changed) {
    if (!c || !mirror) return SCOUT_E_INVALID;
    if (n != c->n) return c->fail(SCOUT_E_STATE, "nothing to commit for this problem");
    const int32_t* p = nullptr;
    int64_t cnt = 0;
    SCOUT_RC(commit_gather(c, problem, &p, &cnt));
    int64_t diff = 0;
    for (int64_t i = 0; i < cnt; i++) {
        int32_t v = p[2 * i], x = p[2 * i + 1];
        if (v < 0 || v >= n) continue;
        if (mirror[v] != x) { mirror[v] = x; diff++; }
    }
    if (changed) *changed = diff;
    return SCOUT_OK;
}

int scout_recompute_bfs(scout_ctx* c, int32_t source, scout_batch_stats* st) {
    if (!c) return SCOUT_E_INVALID;
    if (!c->sealed || !c->level) return c->fail(SCOUT_E_STATE, "graph or BFS state missing");
    if (source < 0 || source >= c->n) return c->fail(SCOUT_E_INVALID, "source out of range");
    cudaSetDevice(c->device);
    scout_batch_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    c->source = source;
    c->last_problem = SCOUT_BFS;
    SCOUT_RC(batch_begin(c));
    SCOUT_RC(lists_ensure(c));
    c->epoch++;
    SCOUT_CU(c, cudaEventRecord(c->ev_t[1], c->s_main));
    SCOUT_RC(bfs_recompute(c, source, st));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[2], c->s_main));
    SCOUT_RC(counters_fetch(c));
    c->qtag += (uint32_t)c->h_ctr->rounds + 8;
    st->rounds = c->h_ctr->rounds;
    st->recomputes = 1;
    st->hbm_bytes = c->h_ctr->hbm_bytes;
    st->changed = c->h_ctr->changed;
    c->last_changed = c->h_ctr->changed;
    st->ms_repair = ev_ms(c->ev_t[1], c->ev_t[2]);
    return SCOUT_OK;
}

int scout_recompute_cc(scout_ctx* c, scout_batch_stats* st) {
    if (!c) return SCOUT_E_INVALID;
    if (!c->sealed || !c->label) return c->fail(SCOUT_E_STATE, "graph or CC state missing");
    cudaSetDevice(c->device);
    scout_batch_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    c->last_problem = SCOUT_CC;
    SCOUT_RC(batch_begin(c));
    SCOUT_RC(lists_ensure(c));
    c->epoch++;
    SCOUT_CU(c, cudaEventRecord(c->ev_t[1], c->s_main));
    SCOUT_RC(cc_recompute(c, st));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[2], c->s_main));
    SCOUT_RC(counters_fetch(c));
    c->qtag += (uint32_t)c->h_ctr->rounds + 8;
    st->rounds = c->h_ctr->rounds;
    st->recomputes = 1;
    st->hbm_bytes = c->h_ctr->hbm_bytes;
    st->changed = c->h_ctr->changed;
    c->last_changed = c->h_ctr->changed;
    st->ms_repair = ev_ms(c->ev_t[1], c->ev_t[2]);
    return SCOUT_OK;
}

int scout_reserve(scout_ctx* c, int64_t max_edits) {
    if (!c || max_edits < 0) return c ? c->fail(SCOUT_E_INVALID, "bad arguments") : SCOUT_E_INVALID;
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    cudaSetDevice(c->device);
    SCOUT_RC(graph_reserve_batch(c, max_edits));
    SCOUT_RC(gather_reserve(c, max_edits));
    if (c->level && !c->bfs_lv) SCOUT_RC(dev_alloc(c, (void**)&c->bfs_lv, (size_t)c->n * 4, "BFS traversal levels"));
    if (c->label) SCOUT_RC(cc_ensure(c));
    if (c->color) SCOUT_RC(coloring_ensure(c));
    SCOUT_RC(pin_grow(c, &c->h_pin_commit, &c->cap_pin_commit, c->n * 8));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    return SCOUT_OK;
}

int scout_sync(scout_ctx* c, int64_t timeout_us) {
    if (!c) return SCOUT_E_INVALID;
    cudaSetDevice(c->device);
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t ss[3] = {c->s_main, c->s_copy[0], c->s_copy[1]};
    for (cudaStream_t s : ss) {
        while (true) {
            cudaError_t e = cudaStreamQuery(s);
            if (e == cudaSuccess) break;
            if (e != cudaErrorNotReady) return cuda_fail(c, e, "scout_sync");
            if (timeout_us > 0 &&
                std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count() > timeout_us)
                return c->fail(SCOUT_E_TIMEOUT, "scout_sync timed out");
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
    return SCOUT_OK;
}

int scout_host_alloc(uint64_t bytes, void** out) {
    if (!out) return host_fail(SCOUT_E_INVALID, "scout_host_alloc: null output");
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, (size_t)std::max<uint64_t>(bytes, 1), cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return host_fail(SCOUT_E_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
    }
    return SCOUT_OK;
}

int scout_host_free(void* p) {
    if (!p) return SCOUT_OK;
    cudaError_t e = cudaFreeHost(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return host_fail(SCOUT_E_CUDA, std::string("cudaFreeHost: ") + cudaGetErrorString(e));
    }
    return SCOUT_OK;
}

}  // extern "C"
