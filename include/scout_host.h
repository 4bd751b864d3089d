/*
 * scout_host.h -- host-side C ABI of scout-b200.
 *
 * Everything the reference keeps on the host around its GPU kernels: the mmap'd .egr
 * CSR reader, the edge-update scratchpad (base adjacency minus tombstones plus
 * additions), the compactor, batch-folder and initial-state I/O, and the fetch
 * pipeline that stages rows from the mmap into pinned slabs for the device.
 * None of these entry points needs a GPU except scout_fetch_* (they call scout_gpu.h).
 *
 * All functions return 0 (SCOUT_OK) or a negative SCOUT_E* code (scout_gpu.h) and never
 * exit the process. Vertex ids are 0-indexed int32 everywhere in this ABI; the text
 * formats on disk stay 1-indexed exactly as the reference reads and writes them.
 * Citations are path:line inside the reference project (anonymous-artifacts/SCOUT).
 */
#ifndef SCOUT_HOST_H
#define SCOUT_HOST_H

#include <stdint.h>
#include "scout_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------------------
 * .egr storage-resident graph
 * ------------------------------------------------------------------------------------- */
typedef struct scout_egr scout_egr;

/* Replaces FlashGraph::open / map_file (core/FlashGraph.h:46-49, 130-192): parses the
 * narrow (int32 nindex) or wide (-1 sentinel, uint64 count, int64 nindex) header, mmaps the
 * file read-only and applies MADV_RANDOM unless madv_random == 0 (the reference's
 * SCOUT_NO_MADV_RANDOM switch, FlashGraph.h:177-179). Truncated files are rejected with
 * SCOUT_E_FORMAT instead of faulting later. */
int scout_egr_open(const char* path, int madv_random, scout_egr** out);
int scout_egr_close(scout_egr* g);
/* FlashGraph::nodes / edges / wide_nindex (FlashGraph.h:37-38, 89). */
int64_t scout_egr_nodes(const scout_egr* g);
int64_t scout_egr_edges(const scout_egr* g);
int     scout_egr_is_wide(const scout_egr* g);
/* FlashGraph::nindex_at for v in [0, n] copied out as int64 (FlashGraph.h:68-71). */
int scout_egr_offsets(const scout_egr* g, int64_t* out_n_plus_1);
/* FlashGraph::neighbors_begin (FlashGraph.h:77-79): pointer into the mapping, valid until close. */
const int32_t* scout_egr_nlist(const scout_egr* g);
/* Writes a .egr. wide != 0 writes the -1 sentinel + uint64 count + int64 nindex layout
 * (README.md:118-128; flash_compactor.h:51-59); wide == 0 requires nnz < 2^31. */
int scout_egr_write(const char* path, int64_t n, const int64_t* off, const int32_t* adj, int wide);

/* ---------------------------------------------------------------------------------------
 * Hybrid graph = base .egr + edge-update scratchpad
 * ------------------------------------------------------------------------------------- */
typedef struct scout_hgraph scout_hgraph;

/* HybridGraph::open (FlashGraph.h:345-354). */
int scout_hgraph_open(const char* egr_path, int madv_random, scout_hgraph** out);
int scout_hgraph_close(scout_hgraph* h);
int64_t scout_hgraph_nodes(const scout_hgraph* h);
/* HybridGraph::isAdjacent (FlashGraph.h:356-366): scratchpad first, then the base row.
 * Returns 1 / 0, or a negative code for out-of-range ids. */
int scout_hgraph_is_adjacent(const scout_hgraph* h, int32_t u, int32_t v);
/* HybridGraph::insertEdge / removeEdge (FlashGraph.h:373-374; DeltaOverlay 227-243). */
int scout_hgraph_insert(scout_hgraph* h, int32_t u, int32_t v);
int scout_hgraph_remove(scout_hgraph* h, int32_t u, int32_t v);
/* HybridGraph::degree (FlashGraph.h:387; DeltaOverlay::degree 267-274). */
int64_t scout_hgraph_degree(const scout_hgraph* h, int32_t v);
/* HybridGraph::neighbors_into (FlashGraph.h:376-385; DeltaOverlay 246-265): base row minus
 * tombstones, then additions in insertion order. Writes up to cap ids, returns the degree. */
int64_t scout_hgraph_neighbors(const scout_hgraph* h, int32_t v, int32_t* out, int64_t cap);
/* Number of vertices with a scratchpad entry and total scratchpad edits (delta_edge_count). */
int64_t scout_hgraph_delta_edits(const scout_hgraph* h);
/* compact_flash_graph + FlashGraph::remap + DeltaOverlay::clear (flash_compactor.h:23-119;
 * FlashGraph.h:56-66, 276-280): writes the wide .egr to <out>.tmp.<pid>, fsyncs, renames
 * atomically, fsyncs the directory, remaps and clears the scratchpad. */
int scout_hgraph_compact(scout_hgraph* h, const char* out_path);

/* ---------------------------------------------------------------------------------------
 * Fetch pipeline: mmap + scratchpad rows -> pinned staging slabs -> HBM
 * ------------------------------------------------------------------------------------- */
/* Streams every row of the hybrid graph into the context's HBM graph store through two
 * pinned slabs on two copy streams (the pattern of scout_cc.cu:160-215 and
 * chunking.h:20-32), then seals the store. The base rows are read with OpenMP workers. */
int scout_fetch_all(scout_hgraph* h, scout_ctx* ctx, int64_t slab_elems);
/* Fetches only the listed rows (the per-round fetch of scout_bfs.cu:197-205 /
 * scout_mis.cu:553-569) and stages them; used for out-of-core misses and for rows the
 * scratchpad changed. */
int scout_fetch_rows(scout_hgraph* h, scout_ctx* ctx, const int32_t* ids, int64_t k);

/* ---------------------------------------------------------------------------------------
 * Batch folders and initial-state files
 * ------------------------------------------------------------------------------------- */
/* parse_batch_file (core/cli_setup.h:87-103) without the classification step: reads
 * "u v" lines (1-indexed), keeps lines whose two leading integers parse, converts to
 * 0-indexed, drops out-of-range ids and self-loops. Two-call protocol: with cap too small
 * returns SCOUT_E_CAPACITY and stores the needed count in *m. */
int scout_parse_batch_file(const char* path, int64_t n, scout_edge* out, int64_t cap, int64_t* m);
/* read_ints_fast (core/cli_setup.h:110-131): every integer of the file in order. */
int scout_read_ints(const char* path, int64_t* out, int64_t cap, int64_t* count);
/* Initial-state decoding exactly as each reference main() does it:
 *   MIS      ids (1-indexed) -> flags, in-range only            (scout_mis.cu:820-828)
 *   coloring color[i] = vals[i] for i < min(n, count), else 0   (scout_coloring.cu:298-306)
 *   BFS      "v level" pairs (1-indexed), default -1             (scout_bfs.cu:546-555)
 *   CC       root ids per line, resolved through find_root       (scout_cc.cu:474-485)
 * sol receives n int32 values; *aux receives the initial MIS count (with repeats, as the
 * reference counts them) or the number of initially reached BFS vertices. */
int scout_load_state(const char* path, int problem, int64_t n, int32_t* sol, int64_t* aux);
/* Writes a state file in the same layout (MIS: 1-indexed ids of members, one per line). */
int scout_write_state(const char* path, int problem, int64_t n, const int32_t* sol);
/* Writes <dir>/1.mtx .. <dir>/<nbatches>.mtx, "u v" 1-indexed per line. */
int scout_write_batch_folder(const char* dir, const scout_edge* pairs, int64_t batch_size,
                             int64_t nbatches);

/* ---------------------------------------------------------------------------------------
 * Synthetic workloads (seeded; the reference's tools/ define the sampling rules)
 * ------------------------------------------------------------------------------------- */
typedef struct scout_csr scout_csr;
/* R-MAT(scale, edge_factor, a, b, c, d = 1-a-b-c), symmetrised, self-loops and duplicate
 * entries removed, rows sorted ascending. Counter-based RNG: identical output for a seed
 * on any machine and thread count. */
int scout_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                   scout_csr** out);
int scout_csr_from_arrays(int64_t n, const int64_t* off, const int32_t* adj, scout_csr** out);
int scout_csr_free(scout_csr* g);
int64_t scout_csr_nodes(const scout_csr* g);
int64_t scout_csr_nnz(const scout_csr* g);
const int64_t* scout_csr_offsets(const scout_csr* g);
const int32_t* scout_csr_adj(const scout_csr* g);

/* Update-stream kinds (rules of tools/generate_*_batches.py):
 *   SCOUT_STREAM_MIXED        existing edges uniform over directed entries + verified
 *                             non-edges with uniform endpoints (generate_mixed_batches.py:77-129)
 *   SCOUT_STREAM_PREFERENTIAL existing edges with the first endpoint proportional to degree
 *                             (generate_preferential_batches.py:56-94) + non-edges with both
 *                             endpoints proportional to degree
 *   SCOUT_STREAM_LOWDEG       deletions: a fraction lowdeg_frac with the first endpoint
 *                             proportional to 1/degree (generate_low_degree_batches.py:56-66),
 *                             the rest uniform; insertions: uniform non-edges
 * Every undirected pair appears at most once in the whole stream; the deletions and
 * insertions are pooled, shuffled, then cut into batches (generate_mixed_batches.py:131-141). */
enum { SCOUT_STREAM_MIXED = 0, SCOUT_STREAM_PREFERENTIAL = 1, SCOUT_STREAM_LOWDEG = 2 };
int scout_gen_stream(const scout_csr* g, int kind, int64_t batch_size, int64_t nbatches,
                     double insert_ratio, double lowdeg_frac, uint64_t seed, scout_edge* out);

/* Initial states (semantics of the reference's seeding tools):
 *   greedy MIS in vertex-id order            (tools/compute_initial_mis.py:32-43), flags
 *   greedy smallest-free colour, id order    (tools/greedy_color.cpp:37-52)
 *   BFS levels from source, -1 unreached      (tools/bfs_ground_truth.cu:39-151)
 *   min-vertex-id component labels            (tools/excc_src/excc_v1.cu:520-531) */
int scout_init_state(const scout_csr* g, int problem, int32_t source, int32_t* out);

#ifdef __cplusplus
}
#endif
#endif /* SCOUT_HOST_H */
