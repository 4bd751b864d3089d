// graph.cu -- the HBM graph store: row table + element pool, staging from pinned host slabs,
// toggle classification and the per-batch merge of edits into the rows.
//
// Layout. row[v] = {start, len, cap} indexes the int32 pool; every row is kept sorted
// ascending (a sorted multiset: a pair inserted twice in one batch appears twice, as the
// reference's scratchpad appends it twice, core/FlashGraph.h:227-234). A batch never
// rewrites a row in place: the merged row is appended at the pool tail and the descriptor
// switched, so kernels reading other rows are never disturbed. The host compacts the pool
// when the free space could not hold a full rewrite plus the batch.
//
// Batch merge (replaces DeltaOverlay::insertEdge / removeEdge + neighbors_into,
// core/FlashGraph.h:227-265, done on the device for every affected row at once):
//   k_classify        toggle -> insert/delete by binary search in the shorter row
//                     (HybridGraph::isAdjacent, FlashGraph.h:356-366); emits two half-edit
//                     keys (u, op, v) and (v, op, u) per applied edit
//   sort_keys         groups half-edits by vertex; inserts before deletes; neighbours sorted
//   k_seg_heads/tails affected-vertex list and its key segments
//   k_row_plan        per affected row: matched deletions (multiset cancel) -> new length
//   scan_i64          new rows' offsets in the pool
//   k_merge_small/large  merge(old row minus deletions, insertions) into the new space
#include "ctx.cuh"

#include <algorithm>
#include <cstring>

namespace scout {

constexpr int SMALL_ROW_LIMIT = 2048;   // rows up to this size are merged by one warp
constexpr int LARGE_THREADS = 512;

// ---------------------------------------------------------------------------------------
// Staging
// ---------------------------------------------------------------------------------------
__global__ void k_rows_from_offsets(Row* __restrict__ row, const int64_t* __restrict__ off, int64_t n, long long base) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        long long s = off[v], e = off[v + 1];
        row[v] = Row{base + s, (int)(e - s), (int)(e - s)};
    }
}

__global__ void k_rows_from_stage(Row* __restrict__ row, const int32_t* __restrict__ ids, const int64_t* __restrict__ off,
                                  int64_t nrows, long long base, int32_t n, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = ids[i];
        if (v < 0 || v >= n) { atomicExch(bad, 1); continue; }
        long long s = off[i] - off[0], e = off[i + 1] - off[0];
        row[v] = Row{base + s, (int)(e - s), (int)(e - s)};
    }
}

// One warp per row: flags rows that are not ascending and counts entries out of range.
__global__ void k_check_rows(const Row* __restrict__ row, const int32_t* __restrict__ pool, int32_t n,
                             int32_t* __restrict__ unsorted, int* __restrict__ n_unsorted, int* __restrict__ bad) {
    for (int v = gwarp_id(); v < n; v += gwarp_count()) {
        Row r = row[v];
        bool ok = true, range_ok = true;
        for (long long i = lane_id(); i < r.len; i += WARP) {
            int32_t x = pool[r.start + i];
            if (x < 0 || x >= n) range_ok = false;
            if (i + 1 < r.len && pool[r.start + i + 1] < x) ok = false;
        }
        ok = __all_sync(0xffffffffu, ok);
        range_ok = __all_sync(0xffffffffu, range_ok);
        if (!range_ok && lane_id() == 0) atomicExch(bad, 1);
        if (!ok && lane_id() == 0) unsorted[atomicAdd(n_unsorted, 1)] = v;
    }
}

// Sort of one unsorted row by one block (bitonic in shared memory, rows up to 8192).
__global__ void k_sort_rows_small(const Row* __restrict__ row, int32_t* __restrict__ pool,
                                  const int32_t* __restrict__ list, int count, int* __restrict__ too_big) {
    __shared__ int32_t s[8192];
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        Row r = row[list[k]];
        if (r.len > 8192) { if (threadIdx.x == 0) atomicExch(too_big, 1); continue; }
        int p = 1;
        while (p < r.len) p <<= 1;
        for (int i = threadIdx.x; i < p; i += blockDim.x) s[i] = i < r.len ? pool[r.start + i] : INT32_MAX;
        __syncthreads();
        for (int size = 2; size <= p; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = threadIdx.x; i < p; i += blockDim.x) {
                    int j = i ^ stride;
                    if (j > i) {
                        bool up = (i & size) == 0;
                        int32_t a = s[i], b = s[j];
                        if ((a > b) == up) { s[i] = b; s[j] = a; }
                    }
                }
                __syncthreads();
            }
        for (int i = threadIdx.x; i < r.len; i += blockDim.x) pool[r.start + i] = s[i];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Classification and half-edit keys
// ---------------------------------------------------------------------------------------
// Key layout: (u << (B + 1)) | (op << B) | v, op 0 = insert, 1 = delete; B = bits(n), so the
// all-ones sentinel sorts after every real key.
__device__ __forceinline__ unsigned long long pack_key(uint32_t u, uint32_t op, uint32_t v, int B) {
    return ((unsigned long long)u << (B + 1)) | ((unsigned long long)op << B) | v;
}

__global__ void k_classify(DGraph g, const scout_edge* __restrict__ e, const uint8_t* __restrict__ ops, int64_t m,
                           int B, unsigned long long* __restrict__ keys, uint8_t* __restrict__ eflag,
                           DevCounters* __restrict__ ctr, int emit) {
    const unsigned long long SENT = (B + B + 1) >= 64 ? ~0ull : ((1ull << (B + B + 1)) - 1);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t u = e[i].u, v = e[i].v;
        bool valid = u >= 0 && u < g.n && v >= 0 && v < g.n && u != v;
        bool ins = false, applied = false;
        if (valid) {
            bool adj = dg_adjacent(g, u, v);
            int op = ops ? ops[i] : SCOUT_OP_TOGGLE;
            if (op == SCOUT_OP_INSERT) { ins = true; applied = !adj; }
            else if (op == SCOUT_OP_DELETE) { ins = false; applied = adj; }
            else { ins = !adj; applied = true; }
        }
        eflag[i] = (uint8_t)((valid ? 1 : 0) | (ins ? 2 : 0) | (applied ? 4 : 0));
        unsigned mi = __ballot_sync(__activemask(), valid && ins);
        unsigned md = __ballot_sync(__activemask(), valid && !ins);
        unsigned ma = __ballot_sync(__activemask(), valid && applied);
        if (lane_id() == (unsigned)(__ffs(__activemask()) - 1)) {
            if (mi) atomicAdd(&ctr->n_ins, __popc(mi));
            if (md) atomicAdd(&ctr->n_del, __popc(md));
            if (ma) atomicAdd(&ctr->n_half, 2 * __popc(ma));
        }
        if (emit) {
            if (valid && applied) {
                uint32_t op = ins ? 0u : 1u;
                keys[2 * i] = pack_key((uint32_t)u, op, (uint32_t)v, B);
                keys[2 * i + 1] = pack_key((uint32_t)v, op, (uint32_t)u, B);
            } else {
                keys[2 * i] = SENT;
                keys[2 * i + 1] = SENT;
            }
        }
    }
}

__device__ __forceinline__ int32_t key_u(unsigned long long k, int B) { return (int32_t)(k >> (B + 1)); }
__device__ __forceinline__ int32_t key_v(unsigned long long k, int B) { return (int32_t)(k & ((1ull << B) - 1)); }
__device__ __forceinline__ int key_op(unsigned long long k, int B) { return (int)((k >> B) & 1ull); }

// Heads of vertex segments get an affected index; slot[u] remembers it for the tails.
__global__ void k_seg_heads(const unsigned long long* __restrict__ keys, int B, DevCounters* __restrict__ ctr,
                            int32_t* __restrict__ aff, int64_t* __restrict__ seg, int32_t* __restrict__ slot) {
    const int64_t nh = ctr->n_half;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nh; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t u = key_u(keys[i], B);
        bool head = i == 0 || key_u(keys[i - 1], B) != u;
        int a = warp_append(head, &ctr->n_aff);
        if (head) {
            aff[a] = u;
            seg[3 * (int64_t)a] = i;
            slot[u] = a;
        }
    }
}

__global__ void k_seg_tails(const unsigned long long* __restrict__ keys, int B, const DevCounters* __restrict__ ctr,
                            int64_t* __restrict__ seg, const int32_t* __restrict__ slot) {
    const int64_t nh = ctr->n_half;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nh; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t u = key_u(keys[i], B);
        bool tail = i == nh - 1 || key_u(keys[i + 1], B) != u;
        if (tail) seg[3 * (int64_t)slot[u] + 2] = i + 1;
        int op = key_op(keys[i], B);
        bool first_del = op == 1 && (i == 0 || key_u(keys[i - 1], B) != u || key_op(keys[i - 1], B) == 0);
        bool no_del_tail = tail && op == 0;
        if (first_del) seg[3 * (int64_t)slot[u] + 1] = i;
        else if (no_del_tail) seg[3 * (int64_t)slot[u] + 1] = i + 1;
    }
}

// Count of x in a sorted int32 span.
__device__ __forceinline__ long long count_in(const int32_t* a, long long n, int32_t x) {
    return upper_bound_i32(a, n, x) - lower_bound_i32(a, n, x);
}

// Deletion keys are read as neighbour ids through this view.
struct KeySpan {
    const unsigned long long* k;
    int B;
    __device__ __forceinline__ int32_t operator[](long long i) const { return key_v(k[i], B); }
};
__device__ __forceinline__ long long lb_keys(KeySpan s, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) { long long mid = (lo + hi) >> 1; if (s[mid] < x) lo = mid + 1; else hi = mid; }
    return lo;
}
__device__ __forceinline__ long long ub_keys(KeySpan s, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) { long long mid = (lo + hi) >> 1; if (s[mid] <= x) lo = mid + 1; else hi = mid; }
    return lo;
}

// Per affected row (one warp). Multiset rule: the r-th copy of d in the deletion list cancels
// the r-th copy of d in the old row (DeltaOverlay::removeEdge forgets one added copy or
// tombstones the base edge, FlashGraph.h:236-243). The warp finds the old entry every
// deletion cancels, the final position of every insertion (j + #old <= y - #cancelled <= y),
// the new length, and only then tombstones the cancelled entries (-1) in the old row, so the
// merge kernels stream the old row without searching it. pos is aligned with the keys.
__global__ void k_row_plan(DGraph g, int32_t* __restrict__ pool_rw, const unsigned long long* __restrict__ keys, int B,
                           DevCounters* __restrict__ ctr, const int32_t* __restrict__ aff,
                           const int64_t* __restrict__ seg, int64_t* __restrict__ new_len,
                           long long* __restrict__ mdp, long long* __restrict__ pos,
                           int32_t* __restrict__ small_list, int32_t* __restrict__ large_list) {
    const int A = ctr->n_aff;
    for (int a = gwarp_id(); a < A; a += gwarp_count()) {
        int32_t u = aff[a];
        long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1], e0 = seg[3 * (int64_t)a + 2];
        Row r = g.row[u];
        const int32_t* O = g.pool + r.start;
        KeySpan I{keys + b0, B};
        KeySpan D{keys + sp, B};
        long long q = e0 - sp, p = sp - b0;
        long long run = 0;
        for (long long base = 0; base < q; base += WARP) {
            long long k = base + lane_id();
            int matched = 0;
            long long at = -1;
            if (k < q) {
                int32_t d = D[k];
                long long rank = k - lb_keys(D, q, d);
                long long lo = lower_bound_i32(O, r.len, d);
                long long cnt = upper_bound_i32(O + lo, r.len - lo, d);
                if (rank < cnt) { matched = 1; at = lo + rank; }
            }
            int inc = warp_incl_scan_i(matched);
            if (k < q) { mdp[sp + k] = run + inc; pos[sp + k] = at; }
            run += __shfl_sync(0xffffffffu, inc, WARP - 1);
        }
        __syncwarp();
        for (long long j = lane_id(); j < p; j += WARP) {
            int32_t y = I[j];
            long long ubo = upper_bound_i32(O, r.len, y);
            long long ubd = ub_keys(D, q, y);
            long long del = ubd > 0 ? mdp[sp + ubd - 1] : 0;
            pos[b0 + j] = j + ubo - del;
        }
        __syncwarp();
        for (long long k = lane_id(); k < q; k += WARP) {
            long long at = pos[sp + k];
            if (at >= 0) pool_rw[r.start + at] = -1;
        }
        if (lane_id() == 0) {
            long long nl = (long long)r.len + p - run;
            new_len[a] = nl;
            long long work = (long long)r.len + p;
            if (work <= SMALL_ROW_LIMIT) small_list[atomicAdd(&ctr->n_small, 1)] = a;
            else large_list[atomicAdd(&ctr->n_large, 1)] = a;
            atomicAdd((unsigned long long*)&ctr->nnz_delta, (unsigned long long)(nl - r.len));
            atomicAdd((unsigned long long*)&ctr->update_bytes,
                      (unsigned long long)(4 * (r.len + nl) + 8 * (p + q) + 16));
        }
    }
}

// Streams a tombstoned old row into its new place: survivor i lands at (#survivors before i)
// + (#insertions < x); the insertion count is searched only inside the range spanned by the
// warp's current values, which is almost always empty.
template <int GROUP>
__device__ __forceinline__ void merge_stream(int tid, const int32_t* __restrict__ O, long long len,
                                             int32_t* __restrict__ out, KeySpan I, long long p,
                                             long long* s_run, unsigned* s_cnt) {
    long long run = 0;
    for (long long base = 0; base < len; base += GROUP) {
        long long i = base + tid;
        int32_t x = i < len ? O[i] : -1;
        bool surv = x >= 0;
        long long lbI = 0;
        if (p > 0) {
            int xmin = __reduce_min_sync(0xffffffffu, surv ? x : INT32_MAX);
            int xmax = __reduce_max_sync(0xffffffffu, surv ? x : -1);
            long long cl = 0, ch = 0;
            if (xmax >= 0 && lane_id() == 0) {
                cl = lb_keys(I, p, xmin);
                ch = lb_keys(I, p, xmax);
            }
            cl = __shfl_sync(0xffffffffu, cl, 0);
            ch = __shfl_sync(0xffffffffu, ch, 0);
            if (surv) {
                long long lo = cl, hi = ch;
                while (lo < hi) {
                    long long mid = (lo + hi) >> 1;
                    if (I[mid] < x) lo = mid + 1; else hi = mid;
                }
                lbI = lo;
            }
        }
        unsigned m = __ballot_sync(0xffffffffu, surv);
        long long before, chunk_total;
        if (GROUP == WARP) {
            before = __popc(m & ((1u << lane_id()) - 1));
            chunk_total = __popc(m);
        } else {
            int w = tid / WARP;
            if (lane_id() == 0) s_cnt[w] = __popc(m);
            __syncthreads();
            if (tid == 0) {
                unsigned acc = 0;
                for (int k = 0; k < GROUP / WARP; k++) { unsigned c = s_cnt[k]; s_cnt[k] = acc; acc += c; }
                *s_run = acc;
            }
            __syncthreads();
            before = s_cnt[w] + __popc(m & ((1u << lane_id()) - 1));
            chunk_total = *s_run;
            __syncthreads();
        }
        if (surv) out[run + before + lbI] = x;
        run += chunk_total;
    }
}

__global__ void k_merge_small(Row* __restrict__ row, const int32_t* __restrict__ pool_in, int32_t* __restrict__ pool_out,
                              const unsigned long long* __restrict__ keys, int B, const DevCounters* __restrict__ ctr,
                              const int32_t* __restrict__ aff, const int64_t* __restrict__ seg,
                              const int64_t* __restrict__ off, const long long* __restrict__ pos,
                              const int32_t* __restrict__ list, long long tail) {
    const int cnt = ctr->n_small;
    for (int k = gwarp_id(); k < cnt; k += gwarp_count()) {
        int a = list[k];
        int32_t u = aff[a];
        long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1];
        Row r = row[u];
        long long start = tail + off[a];
        KeySpan I{keys + b0, B};
        for (long long j = lane_id(); j < sp - b0; j += WARP) pool_out[start + pos[b0 + j]] = I[j];
        merge_stream<WARP>(lane_id(), pool_in + r.start, r.len, pool_out + start, I, sp - b0, nullptr, nullptr);
        __syncwarp();
        int nl = (int)(off[a + 1] - off[a]);
        if (lane_id() == 0) row[u] = Row{start, nl, nl};
    }
}

__global__ void k_merge_large(Row* __restrict__ row, const int32_t* __restrict__ pool_in, int32_t* __restrict__ pool_out,
                              const unsigned long long* __restrict__ keys, int B, const DevCounters* __restrict__ ctr,
                              const int32_t* __restrict__ aff, const int64_t* __restrict__ seg,
                              const int64_t* __restrict__ off, const long long* __restrict__ pos,
                              const int32_t* __restrict__ list, long long tail) {
    __shared__ long long s_run;
    __shared__ unsigned s_cnt[LARGE_THREADS / WARP];
    const int cnt = ctr->n_large;
    for (int k = blockIdx.x; k < cnt; k += gridDim.x) {
        int a = list[k];
        int32_t u = aff[a];
        long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1];
        Row r = row[u];
        long long start = tail + off[a];
        KeySpan I{keys + b0, B};
        for (long long j = threadIdx.x; j < sp - b0; j += LARGE_THREADS) pool_out[start + pos[b0 + j]] = I[j];
        merge_stream<LARGE_THREADS>(threadIdx.x, pool_in + r.start, r.len, pool_out + start, I, sp - b0, &s_run, s_cnt);
        __syncthreads();
        int nl = (int)(off[a + 1] - off[a]);
        if (threadIdx.x == 0) row[u] = Row{start, nl, nl};
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Compaction and download
// ---------------------------------------------------------------------------------------
__global__ void k_row_lens(const Row* __restrict__ row, int64_t n, int64_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        out[v] = row[v].len;
}

// One warp per row: copies the row to its compacted position (16-byte vector body).
__global__ void k_copy_rows(const Row* __restrict__ row, const int32_t* __restrict__ src, int32_t* __restrict__ dst,
                            const int64_t* __restrict__ off, int32_t n) {
    for (int v = gwarp_id(); v < n; v += gwarp_count()) {
        Row r = row[v];
        const int32_t* s = src + r.start;
        int32_t* d = dst + off[v];
        for (long long i = lane_id(); i < r.len; i += WARP) d[i] = s[i];
    }
}

__global__ void k_rows_compacted(Row* __restrict__ row, const int64_t* __restrict__ off, int32_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        long long s = off[v];
        int len = row[v].len;
        row[v] = Row{s, len, len};
    }
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
static int key_bits_for(int64_t n) {
    int B = 1;
    while ((1ll << B) < n + 1) B++;
    return B;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int ws_ensure(scout_ctx* c, int64_t m) {
    int64_t M = std::max<int64_t>(m, 1024);
    if (c->ws && c->ws_m >= M) return SCOUT_OK;
    M = M + M / 2;
    const int64_t H = 2 * M;
    size_t sz[] = {
        (size_t)M * sizeof(scout_edge), (size_t)M, (size_t)M,
        (size_t)H * 8, (size_t)H * 8, (size_t)H * 8,
        (size_t)H * 4, (size_t)3 * H * 8, (size_t)(H + 1) * 8, (size_t)H * 4, (size_t)H * 4};
    size_t total = 0;
    for (size_t s : sz) total += align256(s);
    if (c->ws) dev_free(c, c->ws, (size_t)c->ws_bytes);
    c->ws = nullptr;
    c->ws_m = 0;
    SCOUT_RC(dev_alloc(c, &c->ws, total, "batch workspace"));
    c->ws_bytes = (int64_t)total;
    c->ws_m = M;
    char* p = (char*)c->ws;
    auto take = [&](size_t s) { char* q = p; p += align256(s); return (void*)q; };
    c->d_edits = (scout_edge*)take(sz[0]);
    c->d_ops = (uint8_t*)take(sz[1]);
    c->d_eflag = (uint8_t*)take(sz[2]);
    c->d_keys = (unsigned long long*)take(sz[3]);
    c->d_keys_alt = (unsigned long long*)take(sz[4]);
    c->d_mdp = (long long*)take(sz[5]);
    c->d_aff = (int32_t*)take(sz[6]);
    c->d_aff_seg = (int64_t*)take(sz[7]);
    c->d_aff_len = (int64_t*)take(sz[8]);
    c->d_aff_small = (int32_t*)take(sz[9]);
    c->d_aff_large = (int32_t*)take(sz[10]);
    c->d_hkeys = c->d_keys;
    return SCOUT_OK;
}

int lists_ensure(scout_ctx* c) {
    SCOUT_RC(graph_ensure_scratch(c));
    if (c->d_list[0]) return SCOUT_OK;
    // Queue items are (chunk << 32 | vertex); a vertex pushed once per round occupies at most
    // ceil(len / 1024) items, so n + nnz / 1024 + slack bounds a round.
    c->qcap = c->n + (c->pool_cap / 1024) + 4096;
    for (int i = 0; i < 3; i++) SCOUT_RC(dev_alloc(c, &c->d_qbuf[i], (size_t)c->qcap * 8, "work queues"));
    for (int i = 0; i < 2; i++) SCOUT_RC(dev_alloc(c, (void**)&c->d_list[i], (size_t)c->n * 4, "vertex lists"));
    SCOUT_RC(dev_alloc(c, (void**)&c->d_commit, (size_t)c->n * 8, "commit pairs"));
    return SCOUT_OK;
}

int batch_begin(scout_ctx* c) {
    SCOUT_CU(c, cudaMemsetAsync(c->d_ctr, 0, sizeof(DevCounters), c->s_main));
    SCOUT_CU(c, cudaMemsetAsync(c->d_bar, 0, sizeof(GridBar), c->s_main));
    return SCOUT_OK;
}

int counters_fetch(scout_ctx* c) {
    SCOUT_CU(c, cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, c->s_main));
    SCOUT_CU(c, cudaMemcpyAsync(c->h_bar, c->d_bar, sizeof(GridBar), cudaMemcpyDeviceToHost, c->s_main));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    if (c->h_bar->err == 1)
        return c->fail(SCOUT_E_TIMEOUT, "a device grid barrier timed out (tag " + std::to_string(c->h_bar->where) + ")");
    if (c->h_ctr->pad)
        return c->fail(SCOUT_E_STATE, "the component labels do not describe the components of the graph "
                                      "(an edge joins two labels); upload a consistent labelling");
    if (c->h_bar->err != 0 || c->h_ctr->overflow)
        return c->fail(SCOUT_E_CAPACITY, "a device work list overflowed its capacity");
    return SCOUT_OK;
}

int graph_ensure_scratch(scout_ctx* c) {
    if (c->stamp_a) return SCOUT_OK;
    size_t bytes = (size_t)c->n * sizeof(int32_t);
    int32_t** arrs[] = {&c->stamp_a, &c->stamp_b, &c->stamp_c, &c->aux_v, &c->aux_w};
    for (auto a : arrs) {
        SCOUT_RC(dev_alloc(c, (void**)a, bytes, "per-vertex scratch"));
        SCOUT_CU(c, cudaMemsetAsync(*a, 0, bytes, c->s_main));
    }
    return SCOUT_OK;
}

// Rewrites the pool so rows are contiguous and leaves at least min_free free elements
// (the on-device half of compact_flash_graph).
int graph_compact(scout_ctx* c, int64_t min_free) {
    const int64_t n = c->n;
    int64_t* off = nullptr;
    SCOUT_RC(dev_alloc(c, (void**)&off, (size_t)(n + 1) * sizeof(int64_t), "compaction offsets"));
    int nb = blocks_for(n, 256);
    k_row_lens<<<nb, 256, 0, c->s_main>>>(c->row, n, off);
    SCOUT_LAUNCH(c, "k_row_lens");
    int rc = scan_i64(c, off, n, off + n);
    int64_t live = 0;
    if (rc == SCOUT_OK) {
        cudaMemcpyAsync(&live, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->s_main);
        if (cudaStreamSynchronize(c->s_main) != cudaSuccess) rc = cuda_fail(c, cudaGetLastError(), "compaction");
    }
    int64_t cap = std::max<int64_t>(c->pool_cap, live + min_free);
    // Ping-pong: the previous pool is kept as the next compaction's target, so steady-state
    // compactions allocate nothing. Without budget room for two pools the old one is freed.
    int32_t* np = nullptr;
    if (rc == SCOUT_OK) {
        if (c->spare && c->spare_cap >= cap) {
            np = c->spare;
            cap = c->spare_cap;
            c->spare = nullptr;
            c->spare_cap = 0;
        } else {
            if (c->spare) { dev_free(c, c->spare, (size_t)c->spare_cap * 4); c->spare = nullptr; c->spare_cap = 0; }
            rc = dev_alloc(c, (void**)&np, (size_t)cap * sizeof(int32_t), "element pool");
        }
    }
    if (rc != SCOUT_OK) { dev_free(c, off, (size_t)(n + 1) * 8); return rc; }
    k_copy_rows<<<blocks_for(n * WARP, 256), 256, 0, c->s_main>>>(c->row, c->pool, np, off, (int32_t)n);
    k_rows_compacted<<<nb, 256, 0, c->s_main>>>(c->row, off, (int32_t)n);
    SCOUT_LAUNCH(c, "compaction");
    c->nlaunch += 5;
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    dev_free(c, off, (size_t)(n + 1) * 8);
    if (c->held <= c->budget / 100 * 85) {   // keep the old pool as the next target
        c->spare = c->pool;
        c->spare_cap = c->pool_cap;
    } else {
        dev_free(c, c->pool, (size_t)c->pool_cap * sizeof(int32_t));
    }
    c->compactions++;
    c->pool = np;
    c->pool_cap = cap;
    c->tail = live;
    c->nnz = live;
    return SCOUT_OK;
}

static int upload_edits(scout_ctx* c, const scout_edge* edits, const uint8_t* ops, int64_t m) {
    int64_t bytes = m * (int64_t)sizeof(scout_edge) + (ops ? m : 0);
    SCOUT_RC(pin_grow(c, &c->h_pin_edits, &c->cap_pin_edits, std::max<int64_t>(bytes, 1)));
    std::memcpy(c->h_pin_edits, edits, (size_t)m * sizeof(scout_edge));
    SCOUT_CU(c, cudaMemcpyAsync(c->d_edits, c->h_pin_edits, (size_t)m * sizeof(scout_edge), cudaMemcpyHostToDevice,
                                c->s_main));
    if (ops) {
        char* po = (char*)c->h_pin_edits + m * sizeof(scout_edge);
        std::memcpy(po, ops, (size_t)m);
        SCOUT_CU(c, cudaMemcpyAsync(c->d_ops, po, (size_t)m, cudaMemcpyHostToDevice, c->s_main));
    }
    return SCOUT_OK;
}

int graph_update(scout_ctx* c, const scout_edge* edits, const uint8_t* ops, int64_t m, scout_batch_stats* st) {
    const int64_t n = c->n;
    const int B = key_bits_for(n);
    c->key_bits = B;
    // Free space must hold a rewrite of every live entry plus two entries per edit.
    int64_t need = c->nnz + 2 * m + 1024;
    if (c->pool_cap - c->tail < need) SCOUT_RC(graph_compact(c, need));
    SCOUT_RC(ws_ensure(c, m));
    SCOUT_RC(graph_ensure_scratch(c));
    if (st) st->h2d_bytes += m * (int64_t)sizeof(scout_edge) + (ops ? m : 0);
    if (m == 0) {
        c->d_hkeys = c->d_keys;
        SCOUT_CU(c, cudaEventRecord(c->ev_t[3], c->s_main));
        return SCOUT_OK;
    }
    SCOUT_RC(upload_edits(c, edits, ops, m));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[3], c->s_main));
    DGraph g = dgraph(c);
    k_classify<<<blocks_for(m, 256), 256, 0, c->s_main>>>(g, c->d_edits, ops ? c->d_ops : nullptr, m, B, c->d_keys,
                                                         c->d_eflag, c->d_ctr, 1);
    SCOUT_LAUNCH(c, "k_classify");
    c->nlaunch += 1;
    unsigned long long* sorted = nullptr;
    SCOUT_RC(sort_keys(c, c->d_keys, c->d_keys_alt, 2 * m, 2 * B + 1, &sorted));
    c->d_hkeys = sorted;
    const int64_t H = 2 * m;
    const int64_t Amax = std::min<int64_t>(H, n);
    int nbh = blocks_for(H, 256);
    k_seg_heads<<<nbh, 256, 0, c->s_main>>>(sorted, B, c->d_ctr, c->d_aff, c->d_aff_seg, c->aux_w);
    k_seg_tails<<<nbh, 256, 0, c->s_main>>>(sorted, B, c->d_ctr, c->d_aff_seg, c->aux_w);
    SCOUT_LAUNCH(c, "segments");
    c->nlaunch += 2;
    SCOUT_CU(c, cudaMemsetAsync(c->d_aff_len, 0, (size_t)(Amax + 1) * 8, c->s_main));
    long long* pos = (long long*)(sorted == c->d_keys ? c->d_keys_alt : c->d_keys);   // the free ping-pong half
    k_row_plan<<<blocks_for(Amax * WARP, 256), 256, 0, c->s_main>>>(g, c->pool, sorted, B, c->d_ctr, c->d_aff,
                                                                     c->d_aff_seg, c->d_aff_len, c->d_mdp, pos,
                                                                     c->d_aff_small, c->d_aff_large);
    SCOUT_LAUNCH(c, "k_row_plan");
    c->nlaunch += 1;
    // Exclusive scan over Amax + 1 entries (the tail entries are zero), so the new length of
    // affected row a is off[a + 1] - off[a] for every a.
    SCOUT_RC(scan_i64(c, c->d_aff_len, Amax + 1, (int64_t*)&c->d_ctr->new_elems));
    k_merge_small<<<blocks_for(Amax * WARP, 256), 256, 0, c->s_main>>>(
        c->row, c->pool, c->pool, sorted, B, c->d_ctr, c->d_aff, c->d_aff_seg, c->d_aff_len, pos,
        c->d_aff_small, (long long)c->tail);
    k_merge_large<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(Amax, 4 * c->sm_count)), LARGE_THREADS, 0,
                    c->s_main>>>(c->row, c->pool, c->pool, sorted, B, c->d_ctr, c->d_aff, c->d_aff_seg, c->d_aff_len,
                                 pos, c->d_aff_large, (long long)c->tail);
    SCOUT_LAUNCH(c, "merge");
    c->nlaunch += 2;
    return SCOUT_OK;
}

}  // namespace scout

using namespace scout;

extern "C" {

// ---- graph store ---------------------------------------------------------------------------
int scout_graph_reserve(scout_ctx* c, int64_t n, int64_t nnz) {
    if (!c || n < 1 || n >= INT32_MAX || nnz < 0) return c ? c->fail(SCOUT_E_INVALID, "bad graph size") : SCOUT_E_INVALID;
    if (c->reserved) return c->fail(SCOUT_E_STATE, "graph already reserved");
    cudaSetDevice(c->device);
    c->n = n;
    SCOUT_RC(dev_alloc(c, (void**)&c->row, (size_t)n * sizeof(Row), "row table"));
    SCOUT_CU(c, cudaMemsetAsync(c->row, 0, (size_t)n * sizeof(Row), c->s_main));
    // Room for several batches of rewritten rows between compactions (HBM is plentiful; a
    // budget that cannot hold four times the graph falls back to twice).
    c->pool_cap = 4 * nnz + (1 << 26);
    if ((uint64_t)c->pool_cap * 4 * 2 + c->held > c->budget) c->pool_cap = 2 * nnz + (1 << 22);
    SCOUT_RC(dev_alloc(c, (void**)&c->pool, (size_t)c->pool_cap * sizeof(int32_t), "element pool"));
    c->tail = 0;
    c->nnz = 0;
    c->reserved = true;
    c->sealed = false;
    return SCOUT_OK;
}

static int ensure_slabs(scout_ctx* c, int64_t elems, int64_t rows) {
    if (c->cap_slab < elems) {
        for (int i = 0; i < 2; i++) {
            if (c->h_slab[i]) { cudaEventSynchronize(c->ev_copy[i]); cudaFreeHost(c->h_slab[i]); c->h_slab[i] = nullptr; }
            SCOUT_CU(c, cudaMallocHost(&c->h_slab[i], (size_t)elems * 4));
        }
        c->cap_slab = elems;
    }
    if (c->cap_stage_rows < rows) {
        for (int i = 0; i < 2; i++) {
            if (c->h_slab_ids[i]) { cudaEventSynchronize(c->ev_copy[i]); cudaFreeHost(c->h_slab_ids[i]); cudaFreeHost(c->h_slab_off[i]); }
            if (c->d_stage_ids[i]) { dev_free(c, c->d_stage_ids[i], (size_t)c->cap_stage_rows * 4); dev_free(c, c->d_stage_off[i], (size_t)(c->cap_stage_rows + 1) * 8); }
            SCOUT_CU(c, cudaMallocHost((void**)&c->h_slab_ids[i], (size_t)rows * 4));
            SCOUT_CU(c, cudaMallocHost((void**)&c->h_slab_off[i], (size_t)(rows + 1) * 8));
            SCOUT_RC(dev_alloc(c, (void**)&c->d_stage_ids[i], (size_t)rows * 4, "staging ids"));
            SCOUT_RC(dev_alloc(c, (void**)&c->d_stage_off[i], (size_t)(rows + 1) * 8, "staging offsets"));
        }
        c->cap_stage_rows = rows;
    }
    return SCOUT_OK;
}

// One slab's worth of rows: bounce through pinned memory, async copy on the slot's stream,
// then a kernel points the row descriptors at the copied elements.
static int stage_chunk(scout_ctx* c, int slot, const int32_t* ids, const int64_t* offs, const int32_t* elems,
                       int64_t r0, int64_t r1) {
    int64_t e0 = offs[r0], e1 = offs[r1];
    int64_t ne = e1 - e0, nr = r1 - r0;
    if (c->tail + ne > c->pool_cap) return c->fail(SCOUT_E_CAPACITY, "element pool full while staging rows");
    SCOUT_CU(c, cudaEventSynchronize(c->ev_copy[slot]));
    std::memcpy(c->h_slab[slot], elems + e0, (size_t)ne * 4);
    std::memcpy(c->h_slab_ids[slot], ids + r0, (size_t)nr * 4);
    std::memcpy(c->h_slab_off[slot], offs + r0, (size_t)(nr + 1) * 8);
    cudaStream_t s = c->s_copy[slot];
    SCOUT_CU(c, cudaMemcpyAsync(c->pool + c->tail, c->h_slab[slot], (size_t)ne * 4, cudaMemcpyHostToDevice, s));
    SCOUT_CU(c, cudaMemcpyAsync(c->d_stage_ids[slot], c->h_slab_ids[slot], (size_t)nr * 4, cudaMemcpyHostToDevice, s));
    SCOUT_CU(c, cudaMemcpyAsync(c->d_stage_off[slot], c->h_slab_off[slot], (size_t)(nr + 1) * 8, cudaMemcpyHostToDevice, s));
    k_rows_from_stage<<<blocks_for(nr, 256), 256, 0, s>>>(c->row, c->d_stage_ids[slot], c->d_stage_off[slot], nr,
                                                          (long long)c->tail, (int32_t)c->n, c->d_flags);
    SCOUT_LAUNCH(c, "k_rows_from_stage");
    SCOUT_CU(c, cudaEventRecord(c->ev_copy[slot], s));
    c->tail += ne;
    return SCOUT_OK;
}

int scout_stage_rows(scout_ctx* c, int slot, const int32_t* ids, const int64_t* offs, const int32_t* elems,
                     int64_t nrows, int64_t nelems) {
    if (!c || !ids || !offs || (slot != 0 && slot != 1) || nrows < 0) return c ? c->fail(SCOUT_E_INVALID, "bad staging arguments") : SCOUT_E_INVALID;
    if (!c->reserved) return c->fail(SCOUT_E_STATE, "scout_graph_reserve first");
    if (nrows == 0) return SCOUT_OK;
    if (offs[nrows] - offs[0] != nelems || (!elems && nelems > 0)) return c->fail(SCOUT_E_INVALID, "offsets do not match nelems");
    cudaSetDevice(c->device);
    const int64_t SLAB = 1 << 24;
    int64_t maxrow = 0;
    for (int64_t i = 0; i < nrows; i++) {
        int64_t d = offs[i + 1] - offs[i];
        if (d < 0) return c->fail(SCOUT_E_INVALID, "offsets must be monotone");
        maxrow = std::max(maxrow, d);
    }
    SCOUT_RC(ensure_slabs(c, std::max(SLAB, maxrow), std::min<int64_t>(nrows, 1 << 20)));
    int64_t r = 0;
    int s = slot;
    while (r < nrows) {
        int64_t r1 = r;
        while (r1 < nrows && r1 - r < c->cap_stage_rows && offs[r1 + 1] - offs[r] <= c->cap_slab) r1++;
        SCOUT_RC(stage_chunk(c, s, ids, offs, elems, r, r1));
        r = r1;
        s ^= 1;
    }
    c->sealed = false;
    return SCOUT_OK;
}

int scout_graph_seal(scout_ctx* c) {
    if (!c) return SCOUT_E_INVALID;
    if (!c->reserved) return c->fail(SCOUT_E_STATE, "scout_graph_reserve first");
    cudaSetDevice(c->device);
    for (int i = 0; i < 2; i++) SCOUT_CU(c, cudaStreamWaitEvent(c->s_main, c->ev_copy[i], 0));
    // Rows must be ascending and in range; unsorted rows are sorted here (the reference keeps
    // rows in file order; every rule of this engine is order independent).
    int32_t* list = nullptr;
    int* flags = nullptr;
    SCOUT_RC(dev_alloc(c, (void**)&list, (size_t)c->n * 4, "seal list"));
    int rc = dev_alloc(c, (void**)&flags, 16, "seal flags");
    if (rc != SCOUT_OK) { dev_free(c, list, (size_t)c->n * 4); return rc; }
    cudaMemsetAsync(flags, 0, 16, c->s_main);
    k_check_rows<<<blocks_for(c->n * WARP, 256), 256, 0, c->s_main>>>(c->row, c->pool, (int32_t)c->n, list, flags, flags + 1);
    int h[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(h, flags, 16, cudaMemcpyDeviceToHost, c->s_main);
    int bad_id = 0;
    cudaMemcpyAsync(&bad_id, c->d_flags, 4, cudaMemcpyDeviceToHost, c->s_main);
    cudaError_t e = cudaStreamSynchronize(c->s_main);
    if (e != cudaSuccess) { dev_free(c, list, (size_t)c->n * 4); dev_free(c, flags, 16); return cuda_fail(c, e, "seal"); }
    if (h[1] || bad_id) {
        dev_free(c, list, (size_t)c->n * 4);
        dev_free(c, flags, 16);
        cudaMemsetAsync(c->d_flags, 0, 16, c->s_main);
        return c->fail(SCOUT_E_INVALID, "staged rows hold vertex ids outside [0, n)");
    }
    if (h[0] > 0) {
        k_sort_rows_small<<<blocks_for(h[0], 1, 4096), 512, 0, c->s_main>>>(c->row, c->pool, list, h[0], flags + 2);
        int big = 0;
        cudaMemcpyAsync(&big, flags + 2, 4, cudaMemcpyDeviceToHost, c->s_main);
        cudaStreamSynchronize(c->s_main);
        if (big) {   // rows longer than 8192 entries: sorted on the host
            std::vector<int32_t> ids((size_t)h[0]);
            cudaMemcpy(ids.data(), list, (size_t)h[0] * 4, cudaMemcpyDeviceToHost);
            std::vector<int32_t> tmp;
            for (int32_t v : ids) {
                Row r;
                cudaMemcpy(&r, c->row + v, sizeof(Row), cudaMemcpyDeviceToHost);
                if (r.len <= 8192) continue;
                tmp.resize((size_t)r.len);
                cudaMemcpy(tmp.data(), c->pool + r.start, (size_t)r.len * 4, cudaMemcpyDeviceToHost);
                std::sort(tmp.begin(), tmp.end());
                cudaMemcpy(c->pool + r.start, tmp.data(), (size_t)r.len * 4, cudaMemcpyHostToDevice);
            }
        }
    }
    dev_free(c, list, (size_t)c->n * 4);
    dev_free(c, flags, 16);
    SCOUT_LAUNCH(c, "seal");
    // Contiguous rows, exact nnz and tail.
    SCOUT_RC(graph_compact(c, std::max<int64_t>(c->pool_cap - c->tail, 1 << 22)));
    c->sealed = true;
    return SCOUT_OK;
}

int scout_graph_load_csr(scout_ctx* c, int64_t n, const int64_t* off, const int32_t* adj) {
    if (!c || !off || n < 1) return c ? c->fail(SCOUT_E_INVALID, "bad CSR") : SCOUT_E_INVALID;
    int64_t nnz = off[n];
    if (off[0] != 0 || nnz < 0 || (nnz > 0 && !adj)) return c->fail(SCOUT_E_INVALID, "bad CSR offsets");
    for (int64_t v = 0; v < n; v++)
        if (off[v + 1] < off[v]) return c->fail(SCOUT_E_INVALID, "CSR offsets must be monotone");
    SCOUT_RC(scout_graph_reserve(c, n, nnz));
    // Elements: contiguous pinned-slab copies on two streams.
    const int64_t SLAB = 1 << 24;
    SCOUT_RC(ensure_slabs(c, SLAB, 1024));
    int s = 0;
    for (int64_t e0 = 0; e0 < nnz; e0 += SLAB) {
        int64_t ne = std::min(SLAB, nnz - e0);
        SCOUT_CU(c, cudaEventSynchronize(c->ev_copy[s]));
        std::memcpy(c->h_slab[s], adj + e0, (size_t)ne * 4);
        SCOUT_CU(c, cudaMemcpyAsync(c->pool + e0, c->h_slab[s], (size_t)ne * 4, cudaMemcpyHostToDevice, c->s_copy[s]));
        SCOUT_CU(c, cudaEventRecord(c->ev_copy[s], c->s_copy[s]));
        s ^= 1;
    }
    int64_t* d_off = nullptr;
    SCOUT_RC(dev_alloc(c, (void**)&d_off, (size_t)(n + 1) * 8, "load offsets"));
    SCOUT_CU(c, cudaMemcpyAsync(d_off, off, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, c->s_main));
    k_rows_from_offsets<<<blocks_for(n, 256), 256, 0, c->s_main>>>(c->row, d_off, n, 0);
    SCOUT_LAUNCH(c, "k_rows_from_offsets");
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    dev_free(c, d_off, (size_t)(n + 1) * 8);
    c->tail = nnz;
    return scout_graph_seal(c);
}

int scout_graph_info(scout_ctx* c, int64_t* n, int64_t* nnz, int64_t* used, int64_t* cap) {
    if (!c) return SCOUT_E_INVALID;
    if (n) *n = c->n;
    if (nnz) *nnz = c->nnz;
    if (used) *used = c->tail;
    if (cap) *cap = c->pool_cap;
    return SCOUT_OK;
}

int scout_graph_download(scout_ctx* c, int64_t* off, int32_t* adj, int64_t cap) {
    if (!c || !off) return SCOUT_E_INVALID;
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    cudaSetDevice(c->device);
    const int64_t n = c->n;
    int64_t* d_off = nullptr;
    SCOUT_RC(dev_alloc(c, (void**)&d_off, (size_t)(n + 1) * 8, "download offsets"));
    k_row_lens<<<blocks_for(n, 256), 256, 0, c->s_main>>>(c->row, n, d_off);
    int rc = scan_i64(c, d_off, n, d_off + n);
    if (rc == SCOUT_OK && cudaMemcpyAsync(off, d_off, (size_t)(n + 1) * 8, cudaMemcpyDeviceToHost, c->s_main) != cudaSuccess) rc = SCOUT_E_CUDA;
    if (rc == SCOUT_OK && cudaStreamSynchronize(c->s_main) != cudaSuccess) rc = cuda_fail(c, cudaGetLastError(), "download");
    if (rc != SCOUT_OK) { dev_free(c, d_off, (size_t)(n + 1) * 8); return rc; }
    int64_t total = off[n];
    if (!adj || cap < total) { dev_free(c, d_off, (size_t)(n + 1) * 8); return c->fail(SCOUT_E_CAPACITY, "adjacency buffer too small"); }
    int32_t* tmp = nullptr;
    rc = dev_alloc(c, (void**)&tmp, (size_t)std::max<int64_t>(total, 1) * 4, "download buffer");
    if (rc != SCOUT_OK) { dev_free(c, d_off, (size_t)(n + 1) * 8); return rc; }
    k_copy_rows<<<blocks_for(n * WARP, 256), 256, 0, c->s_main>>>(c->row, c->pool, tmp, d_off, (int32_t)n);
    cudaMemcpyAsync(adj, tmp, (size_t)total * 4, cudaMemcpyDeviceToHost, c->s_main);
    cudaError_t e = cudaStreamSynchronize(c->s_main);
    dev_free(c, tmp, (size_t)std::max<int64_t>(total, 1) * 4);
    dev_free(c, d_off, (size_t)(n + 1) * 8);
    if (e != cudaSuccess) return cuda_fail(c, e, "download");
    return SCOUT_OK;
}

int scout_graph_compact(scout_ctx* c) {
    if (!c) return SCOUT_E_INVALID;
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    cudaSetDevice(c->device);
    return graph_compact(c, std::max<int64_t>(c->nnz, 1 << 22));
}

int scout_classify(scout_ctx* c, const scout_edge* e, int64_t m, uint8_t* out) {
    if (!c || (m > 0 && (!e || !out)) || m < 0) return c ? c->fail(SCOUT_E_INVALID, "bad arguments") : SCOUT_E_INVALID;
    if (!c->sealed) return c->fail(SCOUT_E_STATE, "graph not sealed");
    if (m == 0) return SCOUT_OK;
    cudaSetDevice(c->device);
    SCOUT_RC(ws_ensure(c, m));
    SCOUT_RC(batch_begin(c));
    SCOUT_RC(pin_grow(c, &c->h_pin_edits, &c->cap_pin_edits, m * (int64_t)sizeof(scout_edge) + m));
    std::memcpy(c->h_pin_edits, e, (size_t)m * sizeof(scout_edge));
    SCOUT_CU(c, cudaMemcpyAsync(c->d_edits, c->h_pin_edits, (size_t)m * sizeof(scout_edge), cudaMemcpyHostToDevice, c->s_main));
    k_classify<<<blocks_for(m, 256), 256, 0, c->s_main>>>(dgraph(c), c->d_edits, nullptr, m, 1, nullptr, c->d_eflag, c->d_ctr, 0);
    SCOUT_LAUNCH(c, "k_classify");
    uint8_t* pf = (uint8_t*)c->h_pin_edits + m * sizeof(scout_edge);
    SCOUT_CU(c, cudaMemcpyAsync(pf, c->d_eflag, (size_t)m, cudaMemcpyDeviceToHost, c->s_main));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    for (int64_t i = 0; i < m; i++) out[i] = (pf[i] & 1) ? (uint8_t)((pf[i] >> 1) & 1) : (uint8_t)0xFF;
    return SCOUT_OK;
}

}  // extern "C"
