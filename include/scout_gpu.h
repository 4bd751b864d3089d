/*
 * scout_gpu.h -- device C ABI of scout-b200 (sm_100a).
 *
 * The reference keeps its kernels static inside each src/<problem>/scout_<problem>.cu and
 * drives them from main(); it has no library interface. This header is the seam the
 * host side (bin/scout_<problem>, the Python package, or a foreign caller over ctypes/cgo)
 * binds. Each entry point names the reference code it replaces (path:line inside the
 * reference project, anonymous-artifacts/SCOUT).
 *
 * Conventions
 *  - Every function returns SCOUT_OK (0) or a negative SCOUT_E* code and never exits the
 *    process (the reference calls exit(1) on any CUDA error, core/gpu_common.h:12-19).
 *    scout_last_error(ctx) returns the message of the last failure on that context
 *    (scout_last_error(NULL): last failure of scout_ctx_create on this thread).
 *  - Vertex ids are 0-indexed int32; adjacency offsets are int64.
 *  - Host buffers passed in are only read or written during the call; they may be pageable.
 *    One exception: a page-locked batch given to scout_prefetch is read by the copy that the
 *    next scout_repair call starts, so it stays unchanged until the repair that uses it.
 *  - A repair call that fails after its batch was merged (a device error, a timeout, a
 *    capacity error inside the repair) leaves that store's graph updated and its solution
 *    unrepaired: reload the store (or recompute the solution) before the next batch. A fused
 *    round (scout_multi_run_all) that fails does so for every engine of the round.
 *  - One controlling host thread per context. Contexts are independent (replicas).
 *  - No call drops work silently: a capacity overflow grows the buffer (within the HBM
 *    budget) or returns SCOUT_E_CAPACITY (the reference truncates and warns,
 *    scout_bfs.cu:186-193, 242; scout_coloring.cu:180-188).
 */
#ifndef SCOUT_GPU_H
#define SCOUT_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCOUT_OK          0
#define SCOUT_E_INVALID  (-1)  /* bad argument or id out of range            */
#define SCOUT_E_CUDA     (-2)  /* CUDA runtime error                          */
#define SCOUT_E_CAPACITY (-3)  /* buffer too small or HBM budget exceeded     */
#define SCOUT_E_TIMEOUT  (-4)  /* a bounded device-side wait expired          */
#define SCOUT_E_STATE    (-5)  /* call out of order (e.g. repair before seal) */
#define SCOUT_E_IO       (-6)  /* file could not be opened / read / written   */
#define SCOUT_E_FORMAT   (-7)  /* malformed .egr or state file                */
#define SCOUT_E_NODEV    (-8)  /* no CUDA device                              */

enum scout_problem { SCOUT_MIS = 0, SCOUT_COLORING = 1, SCOUT_BFS = 2, SCOUT_CC = 3 };

/* Per-edit operation. TOGGLE is the reference batch-file semantics: insert if (u,v) is
 * absent from the graph as it stood before this batch, delete if present
 * (core/cli_setup.h:87-103); a pair toggled twice in one batch is classified twice against
 * that same state. INSERT/DELETE carry a classification made by the caller (the MIS binary
 * classifies every batch against the base graph up front, scout_mis.cu:835-842) and are
 * applied only when consistent with the current graph (scout_mis.cu:743-749). */
enum scout_op { SCOUT_OP_TOGGLE = 0, SCOUT_OP_INSERT = 1, SCOUT_OP_DELETE = 2 };

typedef struct scout_edge { int32_t u; int32_t v; } scout_edge;

enum scout_policy   { SCOUT_SCHED_PLAIN = 0, SCOUT_SCHED_LEARNED = 1 };
enum scout_mode     { SCOUT_MODE_AUTO = 0, SCOUT_MODE_INCREMENTAL = 1, SCOUT_MODE_RECOMPUTE = 2 };
enum scout_frontier { SCOUT_FRONTIER_AUTO = 0, SCOUT_FRONTIER_QUEUE = 1, SCOUT_FRONTIER_BITMAP = 2 };

/* Scheduling knobs. A zeroed struct (or NULL) is the plain engine with the reference's
 * heuristics: CC search bound 5000, or unbounded below average degree 10
 * (scout_cc.cu:68-69, 469; core/local_repair.h:13-20). */
typedef struct scout_sched {
    int32_t policy;           /* scout_policy                                       */
    int32_t mode;             /* scout_mode: incremental repair vs full recompute    */
    int32_t frontier;         /* scout_frontier: with mode RECOMPUTE, the BFS traversal's
                                 frontier (QUEUE: top-down queue; BITMAP or AUTO:
                                 direction-optimizing, bottom-up steps over the level array) */
    int32_t lanes_per_vertex; /* BFS expansion: most lanes that share one queue item (one
                                 chunk_log2-sized slice of a row) when a round has fewer
                                 items than warps: 32, 64, 128, 256 or 1024 (1-32 warps);
                                 0 = 64 (two warps), the best measured on a B200         */
    int64_t search_bound;     /* CC local-search bound (vertices); 0 = reference rule */
    int64_t search_limit;     /* CC: a class with more deletions left to search than this is
                                 recomputed instead (0 = 32; < 0 = always search)        */
    int32_t blocks_per_sm;    /* persistent repair kernels: resident blocks per SM (1..4;
                                 0 = as many as fit, at most 4)                          */
    int32_t chunk_log2;       /* BFS queue item = 2^chunk_log2 row entries (8..13; 0 = 8,
                                 the best measured on a B200)                            */
    int32_t prefetched;       /* 1: this call's edits (same count, no ops) are the batch given
                                 to the last scout_prefetch; the device copy that the previous
                                 scout_repair started is used instead of a new upload (when
                                 there is none, or the count differs, the edits are uploaded) */
    int32_t pad0;
    int64_t reserved[1];
} scout_sched;

/* Per-batch statistics (the fields of the reference's Stats structs, scout_bfs.cu:417-424,
 * scout_cc.cu:344-352, scout_coloring.cu:160-165, plus device timings and traffic). */
typedef struct scout_batch_stats {
    int64_t edits;        /* edits accepted                                         */
    int64_t insertions;   /* classified as insertions                                */
    int64_t deletions;    /* classified as deletions                                 */
    int64_t noop;         /* edits that needed no repair                             */
    int64_t conflicts;    /* coloring: same-colour insertions; MIS: both-in-set inserts */
    int64_t affected;     /* vertices examined by the repair                         */
    int64_t changed;      /* solution entries whose value changed                    */
    int64_t rounds;       /* device repair rounds                                    */
    int64_t recomputes;   /* full on-GPU recomputes taken                            */
    int64_t splits;       /* CC: components split by a local search                  */
    int64_t searches;     /* CC: local searches run                                  */
    int64_t hbm_bytes;    /* algorithmic HBM bytes of the repair kernels              */
    int64_t h2d_bytes;    /* host-to-device bytes of the call                         */
    int64_t d2h_bytes;    /* device-to-host bytes of the call                         */
    double  ms_update;    /* device: classification + merge of the edits into HBM rows
                             (edits already in HBM)                                  */
    double  ms_repair;    /* device: repair kernels                                  */
    double  ms_commit;    /* device: changed-entry gather + copy back                */
    double  ms_total;     /* host wall time of the call                              */
    int64_t update_bytes; /* algorithmic HBM bytes of the row merge                   */
    int64_t launches;     /* kernels launched by the call                             */
    double  ms_h2d;       /* device: copy of the edits into HBM                       */
    double  phase_ms[4];  /* device: duration of the repair kernel's first four phases   */
    int64_t variant;      /* repair variant that ran (BFS: 0 incremental, 1 top-down
                             traversal, 2 direction-optimizing traversal; CC: 0
                             incremental, 1 recompute of every class; others 0)     */
    double  ms_compact;   /* device: pool compaction before the merge (0 when none ran) */
    int64_t compactions;  /* pool compactions of the context so far                   */
    int64_t ins_effective; /* BFS: insertions that lowered a level (the reference's
                              "repaired"); CC: insertions that merged two components
                              ("merged"); coloring: same-colour insertions             */
    int64_t del_effective; /* BFS: deletions of a shortest-path tree edge (the reference's
                              local + fallback); CC: deletions whose local search split
                              a component (the reference's "definitive_split")        */
    double  ms_gather;    /* device: the gather of this batch's cold rows into HBM (tiered
                             store, hinted by scout_prefetch; it ran on a copy stream
                             during the previous repair), 0 when none ran             */
    int64_t gather_rows;  /* rows that gather moved into HBM                           */
    int64_t gather_bytes; /* bytes it read over the host link                          */
} scout_batch_stats;

typedef struct scout_ctx scout_ctx;

/* ---- context ------------------------------------------------------------------------ */
/* Replaces gpu_warmup_and_device_setup (core/cli_setup.h:54-58): selects the device,
 * creates the context's streams and events. hbm_budget_bytes caps every allocation the
 * context makes (0 = 90% of the device's free memory); the reference has no such knob. */
int scout_ctx_create(int device, uint64_t hbm_budget_bytes, scout_ctx** out);
int scout_ctx_destroy(scout_ctx* ctx);
const char* scout_last_error(const scout_ctx* ctx);
int scout_device_count(int* out);
/* Device name and HBM bytes currently held by the context. */
int scout_ctx_info(scout_ctx* ctx, char* name, int name_cap, uint64_t* bytes_held);

/* ---- graph store in HBM ------------------------------------------------------------- */
/* Sizes the row table for n vertices and the element pool for nnz entries plus headroom
 * for rows rewritten by later batches (alloc_pair / alloc_and_upload, gpu_common.h:43-72). */
int scout_graph_reserve(scout_ctx* ctx, int64_t n, int64_t nnz);
/* Gather of rows from host staging into HBM: nrows rows (ids[i], elements
 * elems[offs[i] .. offs[i+1]) ) are copied to the device pool and become the current
 * adjacency of those vertices. Replaces the pack + cudaMemcpyAsync of every round
 * (scout_bfs.cu:207-229, scout_coloring.cu:177-201, scout_mis.cu:583-647) and the chunked
 * full-graph upload (scout_cc.cu:160-215). slot (0 or 1) selects the copy stream and the
 * pinned bounce slab; a slot's previous copy is waited for before its slab is reused. */
int scout_stage_rows(scout_ctx* ctx, int slot, const int32_t* ids, const int64_t* offs,
                     const int32_t* elems, int64_t nrows, int64_t nelems);
/* Ends staging: waits for both slots, sorts any row that is not ascending, and makes the
 * store ready for repairs. */
int scout_graph_seal(scout_ctx* ctx);
/* reserve + one stage of every row + seal, from a host CSR. */
int scout_graph_load_csr(scout_ctx* ctx, int64_t n, const int64_t* off, const int32_t* adj);
int scout_graph_info(scout_ctx* ctx, int64_t* n, int64_t* nnz, int64_t* pool_used,
                     int64_t* pool_cap);
/* Out-of-core load for graphs larger than the device budget (the reference keeps the base
 * graph in an mmap and fetches affected rows per round, core/FlashGraph.h:68-83,
 * scout_bfs.cu:199-229): the highest-degree rows, up to half of an HBM pool of hbm_entries
 * elements (0 = derived from the budget), are copied to HBM; every other row lives in mapped
 * page-locked host memory and is read in place by the kernels over the host link. Rows a
 * batch rewrites move to HBM; when the HBM pool cannot take a batch, its shortest rows are
 * evicted to the host pool. scout_graph_load_csr switches to this layout by itself when the
 * budget cannot hold the graph. */
int scout_graph_load_tiered(scout_ctx* ctx, int64_t n, const int64_t* off, const int32_t* adj,
                            int64_t hbm_entries);
/* HBM pool capacity and use, host pool capacity and use (0 when not tiered), entries evicted
 * from HBM so far, and batches whose rewritten rows went to the host pool. */
int scout_graph_tier_info(scout_ctx* ctx, int64_t* hbm_cap, int64_t* hbm_used, int64_t* host_cap,
                          int64_t* host_used, int64_t* evicted, int64_t* host_batches);
/* Current adjacency, rows ascending, written as CSR (off: n+1 entries). Two-call protocol:
 * with cap < nnz returns SCOUT_E_CAPACITY and stores nnz in off[n]. */
int scout_graph_download(scout_ctx* ctx, int64_t* off, int32_t* adj, int64_t cap);
/* Rewrites the pool so every row is contiguous again (the on-device half of
 * compact_flash_graph, core/flash_compactor.h:23-119). */
int scout_graph_compact(scout_ctx* ctx);
/* Toggle classification only (cli_setup.h:98 / FlashGraph.h:356-366) against the current
 * HBM adjacency: is_insertion[i] = 1 if (u,v) is absent. */
int scout_classify(scout_ctx* ctx, const scout_edge* e, int64_t m, uint8_t* is_insertion);

/* ---- solution state ----------------------------------------------------------------- */
/* Upload / download of the maintained solution (setMISFromHost / getMISToHost,
 * scout_mis.cu:480-494; the level/colour cudaMemcpy of scout_bfs.cu:562,
 * scout_coloring.cu:313). Layouts: MIS 0/1 flags, coloring colours, BFS levels (-1
 * unreached), CC component labels (any labelling; the store keeps min-vertex-id labels). */
int scout_state_upload(scout_ctx* ctx, int problem, const int32_t* sol, int64_t n);
int scout_state_download(scout_ctx* ctx, int problem, int32_t* out, int64_t n);
/* BFS source vertex (the reference fixes it to 0, scout_bfs.cu:547). */
int scout_set_source(scout_ctx* ctx, int32_t source);

/* ---- repair --------------------------------------------------------------------------- */
/* One batch: edits go to the device, are classified (ops == NULL means all TOGGLE),
 * merged into the HBM rows, and the solution is repaired on the device. Returns when the
 * batch is repaired. Replaces processBatch of each engine: scout_mis.cu:738-767 (launch +
 * collect), scout_coloring.cu:243-277, scout_bfs.cu:436-515, scout_cc.cu:392-441. */
int scout_repair(scout_ctx* ctx, int problem, const scout_edge* edits, const uint8_t* ops,
                 int64_t m, const scout_sched* sched, scout_batch_stats* stats);
int scout_repair_mis(scout_ctx* ctx, const scout_edge* edits, const uint8_t* ops, int64_t m,
                     const scout_sched* sched, scout_batch_stats* stats);
int scout_repair_coloring(scout_ctx* ctx, const scout_edge* edits, const uint8_t* ops,
                          int64_t m, const scout_sched* sched, scout_batch_stats* stats);
int scout_repair_bfs(scout_ctx* ctx, const scout_edge* edits, const uint8_t* ops, int64_t m,
                     const scout_sched* sched, scout_batch_stats* stats);
int scout_repair_cc(scout_ctx* ctx, const scout_edge* edits, const uint8_t* ops, int64_t m,
                    const scout_sched* sched, scout_batch_stats* stats);
/* Hint: the edits of the batch that will follow the next scout_repair call. That repair call,
 * once its own merge is queued, copies them to the device on a copy stream while its repair
 * runs; the following scout_repair that declares them (scout_sched.prefetched = 1) reads that
 * copy instead of uploading its edits. On a tiered store the same call also gathers the rows
 * of these edits' endpoints that are still in host memory into free HBM, so the hinted batch's
 * merge and repair find them in HBM (its stats report the gather). A page-locked `next` is
 * read in place by that copy and must stay unchanged until the repair that uses it; other
 * buffers are copied here and are free on return. The fetch of batch K+1 overlapping the
 * repair of batch K replaces the reference's per-round host fetch (scout_bfs.cu:199-229) and
 * MIS's K+1 || K channels (scout_mis.cu:855-912). A hint that is not used only costs the copy. */
int scout_prefetch(scout_ctx* ctx, const scout_edge* next, int64_t m);
/* Commit of the last repair's changed entries into a host mirror of n entries: the device
 * gathers (id, value) pairs of changed entries and copies them back; the host scatters
 * them. Replaces the gather_levels + D2H + mirror loop (scout_bfs.cu:244-262), the proposal
 * fold-back (scout_coloring.cu:215-219) and getMISToHost (scout_mis.cu:487-494). */
int scout_commit(scout_ctx* ctx, int problem, int32_t* host_mirror, int64_t n,
                 int64_t* changed_count);
/* Full on-GPU recomputes: BFS from source (gpu_full_bfs, scout_bfs.cu:274-323) and
 * min-id components (full_recompute_cc_gpu, scout_cc.cu:118-278). */
int scout_recompute_bfs(scout_ctx* ctx, int32_t source, scout_batch_stats* stats);
int scout_recompute_cc(scout_ctx* ctx, scout_batch_stats* stats);
/* ---- learned scheduler ------------------------------------------------------------------ */
/* No counterpart in the reference, which fixes its BFS/CC strategy with constants
 * (scout_bfs.cu:475-476, scout_cc.cu:68-69 and 469, core/local_repair.h:13-26). BFS and CC
 * batches can run one of several exact repair variants (scout_batch_stats.variant); with
 * sched->policy = SCOUT_SCHED_LEARNED and a model installed for the problem, a cost model
 * evaluated on the device between the merge and the repair picks the variant with the
 * lowest predicted repair time. Without a model the plain policy (incremental) runs. */
#define SCOUT_SCHED_FEATURES 24
#define SCOUT_SCHED_OUTPUTS  4
#define SCOUT_MLP_PARAMS     6020
/* Installs (params != NULL, 6020 fp32 values in the layout of scout_mlp_get_params, stored
 * as bf16 on the device) or removes (params == NULL) the model of a problem. */
int scout_sched_install(scout_ctx* ctx, int problem, const float* params, int64_t count);
/* Features (24), model outputs (4; NaN without a model) and decision of the last repair that
 * ran the scheduler. */
int scout_sched_last(scout_ctx* ctx, float* features, float* pred, int32_t* decision);
/* Training-data probe: one batch is merged once, then every repair variant of the problem
 * runs from the same pre-repair state and is timed (variant_ms[v] in ms, -1 for variants
 * the problem lacks); their results must agree vertex for vertex (SCOUT_E_STATE otherwise).
 * The batch ends in the incremental variant's state, ready for scout_commit; features
 * receives the 24 scheduler features of the batch. */
int scout_repair_probe(scout_ctx* ctx, int problem, const scout_edge* edits, const uint8_t* ops, int64_t m,
                       const scout_sched* sched, double* variant_ms, float* features,
                       scout_batch_stats* stats);

/* The cost model's own training on the device: a 24-64-64-4 ReLU perceptron with fp32
 * master parameters, trained by hand-written forward/backward kernels and Adam, minibatch
 * loop captured in a CUDA graph; bf16 copy for inference. Errors: scout_last_error(NULL). */
typedef struct scout_mlp scout_mlp;
int scout_mlp_create(int device, uint64_t seed, scout_mlp** out);
int scout_mlp_destroy(scout_mlp* m);
int scout_mlp_get_params(scout_mlp* m, float* out, int64_t count);
int scout_mlp_set_params(scout_mlp* m, const float* in, int64_t count);
/* y[n][4] = model(x[n][24]) with the fp32 parameters, or the bf16 copy when use_bf16. */
int scout_mlp_forward(scout_mlp* m, const float* x, int64_t n, int use_bf16, float* y);
/* Masked mean squared error over all n samples and its gradient (6020 values). */
int scout_mlp_loss_grad(scout_mlp* m, const float* x, const float* t, const float* mask, int64_t n,
                        float* loss, float* grad);
/* epochs of minibatch Adam (learning rate lr) over a seeded shuffle; loss_per_epoch (may be
 * NULL) receives the epoch's mean masked loss measured during the epoch. */
int scout_mlp_train(scout_mlp* m, const float* x, const float* t, const float* mask, int64_t n, int epochs,
                    int batch, float lr, uint64_t seed, float* loss_per_epoch);

/* ---- batched multi-stream engine ---------------------------------------------------------- */
/* No counterpart in the reference, which runs one update stream per process
 * (scout_bfs.cu:517-629, scout_cc.cu:443-554, scout_coloring.cu:279-371, scout_mis.cu:769-1013).
 * K independent streams of one problem, each with its own graph, live as a disjoint union in
 * one device store (stream k owns the vertex range [base_k, base_k + n_k)). A round takes at
 * most one pending batch per stream and runs their union as one batch: one merge, one
 * persistent repair kernel whose work queues hold every stream's items, one commit. Each
 * stream's solution equals the one it would have alone (stream-local vertex ids throughout). */
typedef struct scout_multi scout_multi;
int scout_multi_create(int device, int problem, uint64_t hbm_budget_bytes, scout_multi** out);
int scout_multi_destroy(scout_multi* m);
/* The engine's underlying context (scheduler model install, graph info, compaction). */
scout_ctx* scout_multi_context(scout_multi* m);
/* Adds a stream before the first round: its CSR (n vertices, off[n + 1], adj), its initial
 * solution in the problem's layout (CC labels: vertex ids of the stream), and its BFS source;
 * *stream_id receives its index. */
int scout_multi_add_stream(scout_multi* m, int64_t n, const int64_t* off, const int32_t* adj, const int32_t* init,
                           int32_t source, int32_t* stream_id);
/* Uploads the union (also done by the first round). */
int scout_multi_seal(scout_multi* m);
/* One round of k batches: batch i belongs to stream stream_ids[i] (distinct), with counts[i]
 * edits in stream-local ids and optional ops[i] (NULL array or entry: toggles). Edits whose
 * ids fall outside their stream's graph are skipped. */
int scout_multi_round(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops, const scout_sched* sched,
                      scout_batch_stats* stats);
/* scout_repair_probe of a round's union batch (training data of the scheduler for rounds). */
int scout_multi_probe(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops, const scout_sched* sched,
                      double* variant_ms, float* features, scout_batch_stats* stats);
/* Changed entries of the last round into per-stream host mirrors (mirrors[k]: n_k entries, or
 * NULL to skip stream k); *changed receives the number of entries that changed. */
/* A round of several engines of distinct problems (at most one per problem, one device)
 * repaired by ONE persistent kernel: each engine's round is assembled by scout_multi_stage
 * (the arguments of scout_multi_round), then scout_multi_run_all merges every staged round
 * into its engine's store (on its own stream) and runs one cooperative launch in which the
 * engines' repairs follow one another, each over its own store with its own counters and
 * bounded grid barrier. stats: ne entries (ms_repair is the shared launch); repairs use their
 * plain variants. Commit each engine with scout_multi_commit as after scout_multi_round. */
int scout_multi_stage(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops);
int scout_multi_run_all(int32_t ne, scout_multi* const* ms, const scout_sched* sched, scout_batch_stats* stats);
int scout_multi_commit(scout_multi* m, int32_t* const* mirrors, int64_t* changed);
/* One stream's current solution (n = the stream's vertex count). */
int scout_multi_download(scout_multi* m, int32_t stream, int32_t* out, int64_t n);
int scout_multi_streams(scout_multi* m, int32_t* count, int64_t* total_vertices);
/* scout_reserve of the union for rounds of up to max_round_edits edits (seals first). */
int scout_multi_reserve(scout_multi* m, int64_t max_round_edits);

/* Allocates, now, every buffer that batches of up to max_edits edits and the uploaded
 * problems would otherwise grow on first use (workspace, sort and scan partials, work lists,
 * the compaction target, page-locked commit buffers), so later repairs of that size call no
 * allocator. No counterpart in the reference (it sizes its buffers per run, scout_mis.cu:802-815). */
int scout_reserve(scout_ctx* ctx, int64_t max_edits);
/* Initial solution of a problem computed on the device from the current graph, replacing the
 * reference's offline seeding tools: greedy MIS in vertex-id order
 * (tools/compute_initial_mis.py:32-43), greedy smallest-free colouring in vertex-id order
 * (tools/greedy_color.cpp:37-52), BFS levels from source (tools/bfs_ground_truth.cu:39-151),
 * min-vertex-id component labels (tools/excc_src/excc_v1.cu:520-531). The state is allocated
 * if none was uploaded; read it with scout_state_download. */
int scout_seed(scout_ctx* ctx, int problem, int32_t source, scout_batch_stats* stats);
/* Waits for all work of the context, at most timeout_us (<= 0: no limit). */
int scout_sync(scout_ctx* ctx, int64_t timeout_us);

/* Page-locked host memory for edit batches and mirrors (alloc_pair's pinned half,
 * core/gpu_common.h:43-52). Edits passed to scout_repair from such memory are copied to the
 * device directly; edits in pageable memory go through the context's pinned staging buffer
 * first. */
int scout_host_alloc(uint64_t bytes, void** out);
int scout_host_free(void* p);

/* ---- allocation-free entry point ------------------------------------------------------ */
/* No counterpart in the reference. BFS levels from `source` (-1 unreached) over a CSR that
 * the caller already holds in device memory (d_off: n + 1 int64 offsets, d_adj: int32
 * neighbours), written to the caller's device buffer d_level (n int32), on the caller's
 * stream (a cudaStream_t, NULL for the default stream); returns when the levels are ready.
 * It allocates nothing: for callers that cannot call cudaMalloc (runtimes whose device
 * memory belongs to another allocator or a fixed arena, real-time loops that must stay off
 * the driver's allocator). Its working
 * buffers live in one static device array of 8 MB that every GPU loading the library keeps
 * until the process exits, which bounds n to 1,048,576 vertices; larger graphs are refused
 * with SCOUT_E_CAPACITY. The first call on a device looks up that array's device address
 * (again after the device's context is recreated). Every call waits for its stream, so it
 * cannot be used while that stream is being captured. All calls share the array: calls that overlap on
 * the GPU (two host threads, or two streams) race and must be serialised by the caller.
 * No context is involved; errors are reported through scout_last_error(NULL). */
int scout_bfs_levels_noalloc(const int64_t* d_off, const int32_t* d_adj, int64_t n, int32_t source,
                             int32_t* d_level, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SCOUT_GPU_H */
