// ctx.cuh -- the engine context (struct scout_ctx) and host-side helpers shared by the
// .cu translation units.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../../include/scout_gpu.h"
#include "common.cuh"

// Per-batch device counters, copied back once per batch.
struct DevCounters {
    // update phase
    int n_ins;          // edits classified as insertions
    int n_del;          // edits classified as deletions
    int n_half;         // applied half-edits (2 per applied edit)
    int n_aff;          // vertices whose row changed
    int n_small, n_large;     // rows of the short-row merge / long rows compacted in place
    int n_slices, n_pad;      // merge slices
    long long new_elems;      // elements written to the pool this batch (HBM part when split)
    long long new_elems_host; // tiered store, split batch: elements written to the host pool
    long long nnz_delta;      // inserted minus deleted entries
    long long update_bytes;   // algorithmic bytes of the row merge
    // repair
    int q_count[4];           // rotating queue counters
    int list_count[4];        // auxiliary list counters
    int rounds;
    int changed;
    int affected;
    int conflicts;
    int noop;
    int recomputes;
    int splits;
    int searches;
    int overflow;             // a device list hit its capacity (results invalid)
    int pad;                  // CC: an edge joins two labels (inconsistent uploaded labelling)
    int ins_eff;              // BFS: insertions that lowered a level; CC: insertions that merged classes
    int del_eff;              // BFS: deletions of shortest-path tree edges
    long long hbm_bytes;      // algorithmic bytes of the repair
    long long aux64[4];
    unsigned long long phase_ns[8];   // %globaltimer marks written by the repair kernels
    // scheduler: feature accumulators, the 24 features, the model's 4 outputs, its decision
    int sched_hist[16];       // affected rows by floor(log2(1 + new degree))
    int sched_del_hit;        // deletion half-edits meeting the problem's structural test
    int sched_del;            // deletion half-edits
    int decision;             // repair variant the kernels run (read on the device)
    int sort_err;             // 1: a sort look-back wait timed out, 2: a sort position out of range,
                              // 3: a bulk copy into shared memory (row merge) did not complete,
                              // 4: a scan look-back wait timed out
    int sched_flags;          // 1 features computed, 2 model applied
    float feat[24];
    float pred[4];
};

struct scout_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t s_main = nullptr;
    cudaStream_t s_copy[2] = {nullptr, nullptr};
    cudaEvent_t ev_copy[2] = {nullptr, nullptr};
    cudaEvent_t ev_t[8] = {nullptr};
    uint64_t budget = 0;
    uint64_t held = 0;
    std::string err;
    char name[256] = {0};

    // ---- graph store ----
    int64_t n = 0;
    int64_t nnz = 0;           // live entries (host view, exact after each batch)
    scout::Row* row = nullptr;
    int32_t* pool = nullptr;
    int64_t pool_cap = 0;
    int64_t tail = 0;          // first free pool element (host view)
    int32_t* spare = nullptr;  // previous pool, next compaction target
    int64_t spare_cap = 0;
    // tiered store (device budget smaller than the graph): cold rows live in mapped page-locked
    // host memory and are read in place by the kernels; a row is HBM-resident iff
    // 0 <= start < pool_cap, otherwise start is its element offset from `pool` into host_pool
    bool tiered = false;
    int32_t* host_pool = nullptr;   // host pointer (also the device pointer: unified addressing)
    int64_t host_cap = 0;
    int64_t host_tail = 0;
    int64_t evictions = 0;          // rows moved from HBM to the host pool by compactions
    int64_t evicted_entries = 0;
    int batch_dest = 0;             // where this batch's rewritten rows go: 0 HBM tail, 1 host
                                    // tail, 2 split (rows from HBM to HBM, host rows to host)
    int64_t host_batches = 0;       // batches whose rows were rewritten into the host pool
    int64_t compactions = 0;
    long long merge_tail = 0;       // HBM tail once the current batch's merge is done
    // gather of the next batch's cold rows (tiered store; scout_prefetch, gather.cu)
    bool pf_pending = false;        // a hint waits for the next repair's merge
    int64_t pf_m = 0;
    const scout_edge* pf_host = nullptr;   // where the hinted edits are read from (page-locked)
    void* h_pf_edits = nullptr;  int64_t cap_h_pf_edits = 0;   // pinned copy of pageable hinted edits
    scout_edge* d_pf_edits[2] = {nullptr, nullptr};  int64_t cap_pf_edits[2] = {0, 0};
    int pf_slot = 0;                // slot of the latest copy of hinted edits
    bool pf_ready = false;          // that slot holds (once ev_pf completes) a batch not yet used
    int64_t pf_ready_m = 0;
    bool pf_use = false;            // this call's edits are the hinted batch (scout_sched.prefetched)
    cudaEvent_t ev_pf = nullptr;    // the hinted edits' copy is done (copy stream)
    cudaEvent_t ev_union = nullptr; // fused repair rounds: this store's merge / the repair is done
    int32_t* gather_stamp = nullptr;   // n: last gather that took the vertex's row
    uint32_t gather_tag = 0;
    void* d_gctr = nullptr;
    void* h_gctr = nullptr;            // pinned
    int32_t* d_gather_list = nullptr;  int64_t cap_gather_list = 0;
    long long* d_gather_dst = nullptr; int64_t cap_gather_dst = 0;
    cudaEvent_t ev_gather0 = nullptr, ev_gather1 = nullptr;   // start / end of the gather (copy stream)
    long long gather_base = 0;
    bool gather_active = false;
    int64_t gathered_rows = 0, gathered_bytes = 0;
    bool reserved = false;
    bool sealed = false;
    int32_t* d_tmp_rows = nullptr;   // staging target for rows of one slot
    int64_t staged_rows = 0;

    // ---- per-problem state ----
    int32_t* level = nullptr;
    int32_t* color = nullptr;
    int32_t* label = nullptr;
    int32_t* mis = nullptr;
    int32_t source = 0;
    int32_t* d_sources = nullptr;   // BFS roots of a union of graphs (nsrc > 0), else `source`
    int nsrc = 0;
    int last_problem = -1;

    // ---- persistent per-vertex scratch (stamped with a batch epoch; never cleared) ----
    int32_t* stamp_a = nullptr;   // e.g. invalid / queued marks
    int32_t* stamp_b = nullptr;
    int32_t* stamp_c = nullptr;
    int32_t* stamp_d = nullptr;
    int32_t* aux_v = nullptr;     // per-vertex int scratch (marker / uf parent)
    int32_t* aux_w = nullptr;
    uint32_t epoch = 0;

    // ---- per-batch workspace: one allocation, carved per batch size (grow-only) ----
    void* ws = nullptr;
    int64_t ws_bytes = 0;
    int64_t ws_m = 0;               // edits the workspace is carved for
    scout_edge* d_edits = nullptr;
    uint8_t* d_ops = nullptr;
    uint8_t* d_eflag = nullptr;
    unsigned long long* d_keys = nullptr;       // half-edit keys (2m)
    unsigned long long* d_keys_alt = nullptr;   // radix ping-pong (2m)
    unsigned long long* d_hkeys = nullptr;      // sorted half-edits of the current batch
    long long* d_mdp = nullptr;     // matched-deletion prefix, aligned with keys (2m)
    int32_t* d_aff = nullptr;       // affected vertex ids (2m)
    int64_t* d_aff_seg = nullptr;   // [3 * 2m]: segment begin, first deletion, end
    int64_t* d_aff_len = nullptr;   // new length, then exclusive offsets (2m + 1)
    int64_t* d_aff_len2 = nullptr;  // tiered split batches: lengths / offsets of the host rows (2m + 1)
    int32_t* d_aff_small = nullptr; // affected rows merged by the short-row merge (2m)
    int32_t* d_aff_long = nullptr;  // long affected rows compacted in place (2m)
    int64_t* d_small_off = nullptr; // short-row lengths, then their exclusive scan (2m + 1)
    scout::Row* d_old_row = nullptr;   // descriptors of the affected rows before the batch (2m)
    int64_t* d_slices = nullptr;  int64_t cap_slices = 0;   // merge items (row << 32 | slice)
    int64_t* d_coff = nullptr;      // compaction offsets (n + 1)
    int key_bits = 0;

    // ---- per-vertex work lists (n-sized, allocated on first repair) ----
    void* d_qbuf[3] = {nullptr, nullptr, nullptr};   // queues (uint64 items), qcap each
    int64_t qcap = 0;
    int32_t* d_list[2] = {nullptr, nullptr};         // touched / invalid lists, n each
    int32_t* d_commit = nullptr;                     // (id, value) pairs for the commit (2n)
    uint32_t qtag = 1;                               // per-round dedupe tags, never reused
    unsigned int* d_sort_hist = nullptr; int64_t cap_hist = 0;   // one-sweep control + look-back
    int64_t* d_scan_tmp = nullptr;  int64_t cap_scan = 0;
    void* d_misc = nullptr;         int64_t cap_misc = 0;   // colouring proposal markers
    int32_t* d_cc = nullptr;        // component scratch (7 n int32)
    int32_t* bfs_lv = nullptr;      // levels of a full BFS traversal before the diff (n int32)

    // ---- scheduler ----
    void* model[4] = {nullptr, nullptr, nullptr, nullptr};   // bf16 cost model per problem
    double prev_repair_ms[4] = {0, 0, 0, 0};                  // last batch's repair time per problem
    int32_t* probe_buf = nullptr;   // probe: pre-repair state, first variant's result, mismatch counter
    DevCounters* d_ctr_snap = nullptr;

    DevCounters* d_ctr = nullptr;
    DevCounters* h_ctr = nullptr;   // pinned
    scout::GridBar* d_bar = nullptr;
    scout::GridBar* h_bar = nullptr; // pinned
    int* d_flags = nullptr;          // staging / seal error flags (int[16])

    // ---- pinned staging ----
    void* h_pin_edits = nullptr;  int64_t cap_pin_edits = 0;
    void* h_pin_commit = nullptr; int64_t cap_pin_commit = 0;
    void* h_slab[2] = {nullptr, nullptr}; int64_t cap_slab = 0;   // int32 elements
    int64_t* h_slab_off[2] = {nullptr, nullptr}; int32_t* h_slab_ids[2] = {nullptr, nullptr};
    int64_t cap_slab_rows = 0;
    int32_t* d_stage_ids[2] = {nullptr, nullptr};
    int64_t* d_stage_off[2] = {nullptr, nullptr};
    int64_t cap_stage_rows = 0;

    // ---- last batch bookkeeping ----
    int64_t last_changed = 0;
    int64_t last_half = 0;
    int64_t last_aff = 0;
    int32_t coop_blocks = 0;   // resident blocks of the persistent kernels
    // tuning knobs of the current call (scout_sched.blocks_per_sm / chunk_log2)
    int tune_blocks_per_sm = 0;   // 0: as many as fit, at most 4
    int tune_chunk_log2 = 10;     // BFS queue item = 2^chunk_log2 row entries
    int tune_share = 0;           // most warps sharing one BFS queue item (0: as many as useful)
    int64_t nlaunch = 0;       // kernels launched (running count)

    int fail(int code, const std::string& msg) { err = msg; return code; }
};

namespace scout {

// Allocation against the context's HBM budget.
int dev_alloc(scout_ctx* c, void** p, size_t bytes, const char* what);
void dev_free(scout_ctx* c, void* p, size_t bytes);
template <typename T>
int dev_grow(scout_ctx* c, T** p, int64_t* cap, int64_t need, const char* what) {
    if (*cap >= need && *p) return SCOUT_OK;
    int64_t nc = need + need / 4 + 1024;
    if (*p) dev_free(c, *p, (size_t)*cap * sizeof(T));
    *p = nullptr;
    *cap = 0;
    int rc = dev_alloc(c, (void**)p, (size_t)nc * sizeof(T), what);
    if (rc != SCOUT_OK) return rc;
    *cap = nc;
    return SCOUT_OK;
}
int pin_grow(scout_ctx* c, void** p, int64_t* cap_bytes, int64_t need_bytes);

int cuda_fail(scout_ctx* c, cudaError_t e, const char* where);
int host_fail(int code, const std::string& msg);   // thread-local message for calls without a context
#define SCOUT_CU(c, call)                                                  \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return ::scout::cuda_fail((c), e_, #call);  \
    } while (0)
#define SCOUT_LAUNCH(c, what)                                              \
    do {                                                                   \
        cudaError_t e_ = cudaGetLastError();                               \
        if (e_ != cudaSuccess) return ::scout::cuda_fail((c), e_, what);   \
    } while (0)
#define SCOUT_RC(x)                          \
    do {                                     \
        int rc_ = (x);                       \
        if (rc_ != SCOUT_OK) return rc_;     \
    } while (0)

inline DGraph dgraph(const scout_ctx* c) { return DGraph{c->row, c->pool, (int32_t)c->n}; }
inline int blocks_for(int64_t items, int threads, int cap = 148 * 32) {
    int64_t b = (items + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

// sort.cu
int sort_keys(scout_ctx* c, unsigned long long* keys, unsigned long long* alt, int64_t n, int bits,
              unsigned long long** sorted_out);
// scan.cu: exclusive scan of int64 values in place; *total receives the sum (device ptr or null)
int scan_i64(scout_ctx* c, int64_t* data, int64_t n, int64_t* d_total);
int sort_reserve(scout_ctx* c, int64_t nkeys);
// graph.cu: every buffer a batch of up to m edits can grow, allocated now
int graph_reserve_batch(scout_ctx* c, int64_t m);
// problem scratch allocated on first use, or ahead of time by scout_reserve
int cc_ensure(scout_ctx* c);
int coloring_ensure(scout_ctx* c);
// graph.cu
int graph_update(scout_ctx* c, const scout_edge* edits, const uint8_t* ops, int64_t m, scout_batch_stats* st);
int graph_ensure_scratch(scout_ctx* c);
int graph_compact(scout_ctx* c, int64_t min_free, bool nnz_exact = false);
int ws_ensure(scout_ctx* c, int64_t m);
int lists_ensure(scout_ctx* c);
int batch_begin(scout_ctx* c);   // zeroes the counters and the barrier for a new batch
int counters_fetch(scout_ctx* c); // copies the device counters into c->h_ctr (synchronous)
// problem kernels (their .cu files)
// BFS repair variants: 0 incremental, 1 top-down traversal, 2 direction-optimizing
// traversal; mode_dev (device int) overrides mode when the scheduler decides on the device.
constexpr int BFS_MODE_INCREMENTAL = 0, BFS_MODE_TOP_DOWN = 1, BFS_MODE_DIRECTION_OPT = 2;
int bfs_repair(scout_ctx* c, int mode, const int* mode_dev, scout_batch_stats* st);
int bfs_recompute(scout_ctx* c, int32_t source, scout_batch_stats* st);
// CC repair variants: 0 incremental, 1 recompute of every class, 2 recompute of every class
// with an unsettled deletion; mode_dev as for BFS.
int cc_repair(scout_ctx* c, const scout_sched* sched, int variant, const int* mode_dev, scout_batch_stats* st);
int cc_recompute(scout_ctx* c, scout_batch_stats* st);
int coloring_repair(scout_ctx* c, scout_batch_stats* st);
int mis_repair(scout_ctx* c, scout_batch_stats* st);
// sched.cu: features + on-device inference of the installed model; writes ctr->decision.
// Returns SCOUT_OK and sets *mode_dev to the decision's device address when the learned
// policy applies to the problem, else leaves it null (plain policy).
int sched_decide(scout_ctx* c, int problem, int64_t m, bool use_model, const int** mode_dev);
void sched_release(scout_ctx* c);
int sched_variants(int problem);   // repair variants a problem has (BFS 3, CC 2, others 1)
// api.cu: the last repair's (id, value) pairs in page-locked memory (valid until the next call)
int commit_gather(scout_ctx* c, int problem, const int32_t** pairs, int64_t* count);
// persistent launch helper
int coop_launch(scout_ctx* c, const void* fn, int threads, void** args, size_t smem);
// gather.cu: the hinted next batch's edits to the device and (tiered store) its cold rows into
// free HBM from `base` on a copy stream, after the current merge is queued; gather_finish waits
// for the gather (main stream and host) and moves the tail.
int prefetch_launch(scout_ctx* c, long long base);
// union.cu: one cooperative launch of the repairs of ne union stores of distinct problems whose
// batches are merged (queued); api.cu: the whole round (merges, launch, counters, stats)
int union_launch(scout_ctx* const* cs, const int* problems, const scout_sched* sds, const int* variants, int ne);
int union_run(scout_ctx* const* cs, const int* problems, const scout_edge* const* edits, const uint8_t* const* ops,
              const int64_t* counts, int ne, const scout_sched* sched, scout_batch_stats* stats);
// graph.cu: host copy into page-locked staging, over the host threads for large copies
void stage_copy(void* dst, const void* src, size_t bytes);
int gather_finish(scout_ctx* c, double* ms, int64_t* rows, int64_t* bytes);
int gather_reserve(scout_ctx* c, int64_t max_edits);

}  // namespace scout
