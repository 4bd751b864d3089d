// graph.cu -- the HBM graph store: row table + element pool, staging from pinned host slabs,
// toggle classification and the per-batch merge of edits into the rows.
//
// Layout. row[v] = {start, len, cap} indexes the int32 pool; every row is kept sorted
// ascending (a sorted multiset: a pair inserted twice in one batch appears twice, as the
// reference's scratchpad appends it twice, core/FlashGraph.h:227-234). A row that gains
// entries, or a long one, is merged into new space at the pool tail and its descriptor
// switched; a short row whose half-edits are all deletions is compacted where it lies (its
// survivors only move towards the row start; only the warp merging it touches it). The host
// compacts the pool when the free space could not hold a full rewrite plus the batch.
//
// Batch merge (replaces DeltaOverlay::insertEdge / removeEdge + neighbors_into,
// core/FlashGraph.h:227-265, done on the device for every affected row at once):
//   k_classify        toggle -> insert/delete by binary search in the shorter row
//                     (HybridGraph::isAdjacent, FlashGraph.h:356-366); emits two half-edit
//                     keys (u, op, v) and (v, op, u) per applied edit
//   sort_keys         groups half-edits by vertex; inserts before deletes; neighbours sorted
//   k_seg_heads/tails affected-vertex list and its key segments
//   k_row_alloc       old descriptor, new space (old length + insertions; none for a short
//                     row that only loses entries), short-row list, slices of long rows
//   scan_i64          new rows' offsets in the pool
//   k_plan_match      per deletion: the old entry it cancels (multiset rule); matched flags
//   scan_i64          matched deletions before every half-edit
//   k_plan_place      per insertion: its final slot in the new row; per matched deletion: the
//                     old entry's tombstone (sign bit); per row: the new descriptor
//   k_merge_small     survivors of short rows, balanced groups of ~UNIT entries per warp
//   k_merge_slices    survivors of longer rows, one warp per slice of SLICE entries, so a hub
//                     row is spread over many warps
//   k_merge_long_inplace  rows longer than a slice that only lose entries, a block per row
#include "ctx.cuh"

#include <algorithm>
#include <cstring>

namespace scout {

constexpr int SLICE = 4096;          // old-row entries streamed by one warp in the slice merge
constexpr int SMALL_LEN = 128;       // rows up to this length go to the short-row merge

// A row whose half-edits are all deletions is rewritten in place: its survivors only move
// towards the row start, it keeps its start and capacity, and it takes no pool space (short
// rows in the short-row merge, rows of one slice by their warp in the slice merge). A longer
// one is compacted in place by one block (k_merge_long_inplace: its slices would overlap) only
// when `long_in_place` is set, in the tiered store, whose HBM room is scarce; in the all-HBM
// store it is rewritten at the pool tail by the slice merge, spread over many warps.
__host__ __device__ __forceinline__ bool in_place_row(long long insertions, int old_len, bool long_in_place) {
    return insertions == 0 && (old_len <= SLICE || long_in_place);
}

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

// Deletion keys are read as neighbour ids through this view.
struct KeySpan {
    const unsigned long long* k;
    int B;
    __device__ __forceinline__ int32_t operator[](long long i) const { return key_v(k[i], B); }
};
template <typename S>
__device__ __forceinline__ long long lb_span(S s, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) { long long mid = (lo + hi) >> 1; if (s[mid] < x) lo = mid + 1; else hi = mid; }
    return lo;
}
template <typename S>
__device__ __forceinline__ long long ub_span(S s, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) { long long mid = (lo + hi) >> 1; if (s[mid] <= x) lo = mid + 1; else hi = mid; }
    return lo;
}

__device__ __forceinline__ long long warp_lower_bound(const int64_t* a, long long n, long long x) {
    // first i in [0, n) with a[i] >= x (n if none), 32 probes per step (all lanes call)
    long long lo = 0, hi = n;
    while (hi - lo > WARP) {
        const long long step = (hi - lo + WARP - 1) / WARP;
        const long long pos = lo + (long long)lane_id() * step;
        const bool less = pos < hi && a[pos] < x;
        const int c = __popc(__ballot_sync(0xffffffffu, less));   // probes below x form a prefix
        const long long nlo = c == 0 ? lo : lo + (long long)(c - 1) * step + 1;
        const long long nhi = c == 0 ? lo : min(hi, lo + (long long)c * step);
        lo = nlo;
        hi = max(nlo, nhi);
        if (c == 0) break;
    }
    const long long pos = lo + lane_id();
    const bool less = pos < hi && a[pos] < x;
    return lo + __popc(__ballot_sync(0xffffffffu, less));
}

// Per affected row: its descriptor before the batch and the space of its new row (old length
// + insertions: slots of matched deletions stay unused until the next compaction). Rows up
// to SMALL_LEN entries go to the short-row merge, longer ones are cut into merge slices
// (rows past one slice that only lose entries go to the in-place block merge instead).
__global__ void k_row_alloc(const Row* __restrict__ row, DevCounters* __restrict__ ctr, const int32_t* __restrict__ aff,
                            const int64_t* __restrict__ seg, Row* __restrict__ old_row, int64_t* __restrict__ alloc,
                            int32_t* __restrict__ small, int64_t* __restrict__ small_len, int64_t* __restrict__ slices,
                            int64_t slice_cap, int32_t* __restrict__ longs, bool long_in_place) {
    const int A = ctr->n_aff;
    const int T = gridDim.x * blockDim.x;
    for (int b = (int)(blockIdx.x * blockDim.x + threadIdx.x) - (int)lane_id(); b < A; b += T) {
        const int a = b + (int)lane_id();
        const bool ok = a < A;
        int ns = 0;
        bool sm = false, lip = false;
        if (ok) {
            const long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1];
            const Row r = row[aff[a]];
            old_row[a] = r;
            const bool ip = in_place_row(sp - b0, r.len, long_in_place);
            alloc[a] = ip ? 0 : (long long)r.len + (sp - b0);
            sm = r.len <= SMALL_LEN;
            lip = ip && r.len > SLICE;   // longer than a slice, compacted in place: one block
            ns = sm || lip ? 0 : (r.len + SLICE - 1) / SLICE;
        }
        const int lat = warp_append(lip, &ctr->n_large);
        if (lip) longs[lat] = a;
        const int at = warp_append(ok && sm, &ctr->n_small);
        if (ok && sm) {
            small[at] = a;
            small_len[at] = old_row[a].len;   // the merge balances its groups by old length
        }
        const int inc = warp_incl_scan_i(ns);
        int base = 0;
        if (lane_id() == WARP - 1 && inc) base = atomicAdd(&ctr->n_slices, inc);
        base = __shfl_sync(0xffffffffu, base, WARP - 1);
        const long long s0 = (long long)base + inc - ns;
        if (s0 + ns > slice_cap) { if (ns) atomicExch(&ctr->overflow, 1); continue; }
        for (int s = 0; s < ns; s++) slices[s0 + s] = ((long long)a << 32) | s;
    }
}

// Searches of an old row whose cancelled entries may already carry the tombstone bit (the
// sign bit, so the masked values stay sorted while the row is being marked).
__device__ __forceinline__ int32_t unmark(int32_t x) { return x & 0x7fffffff; }
__device__ __forceinline__ long long ub_masked(const int32_t* a, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (lo < hi) { long long mid = (lo + hi) >> 1; if (unmark(a[mid]) <= x) lo = mid + 1; else hi = mid; }
    return lo;
}

// Plan, step 1: one thread per half-edit. Multiset rule: the r-th copy of d among a row's
// deletions cancels the r-th copy of d in the old row (DeltaOverlay::removeEdge forgets one
// added copy or tombstones the base edge, FlashGraph.h:236-243). A deletion records dpos =
// (at << 1) | matched, with at the cancelled entry, or the end of d's copies when none is
// left, so dpos is non-decreasing along a row's sorted deletions; flag = matched (0 for
// insertions and for the unused tail up to H) feeds one exclusive scan over all half-edits.
__global__ void k_plan_match(const int32_t* __restrict__ pool, const unsigned long long* __restrict__ keys, int B,
                             const DevCounters* __restrict__ ctr, const int32_t* __restrict__ slot,
                             const int64_t* __restrict__ seg, const Row* __restrict__ old_row,
                             long long* __restrict__ dpos, long long* __restrict__ flag, long long H) {
    const long long nh = ctr->n_half;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < H; k += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = k < nh ? keys[k] : 0ull;
        long long f = 0;
        if (k < nh && key_op(key, B) == 1) {
            const int a = slot[key_u(key, B)];
            const long long sp = seg[3 * (int64_t)a + 1], e0 = seg[3 * (int64_t)a + 2];
            const int32_t d = key_v(key, B);
            long long rank = 0;
            if (k > sp && key_v(keys[k - 1], B) == d) rank = k - (sp + lb_span(KeySpan{keys + sp, B}, e0 - sp, d));
            const Row r = old_row[a];
            const int32_t* O = pool + r.start;
            const long long lo = lower_bound_i32(O, r.len, d);
            const bool matched = lo + rank < r.len && O[lo + rank] == d;
            const long long at = matched ? lo + rank : lo + upper_bound_i32(O + lo, r.len - lo, d);
            dpos[k] = (at << 1) | (matched ? 1 : 0);
            f = matched ? 1 : 0;
        }
        flag[k] = f;
    }
}

// Plan, step 2 (after the scan: E[k] = matched deletions before half-edit k): one thread per
// half-edit. An insertion y (j-th of its row) lands at j + #old <= y - #cancelled <= y of the
// new row and is written there; a matched deletion tombstones its old entry; the first
// half-edit of a row writes the row's new descriptor.
__global__ void k_plan_place(int32_t* __restrict__ pool, Row* __restrict__ row, const unsigned long long* __restrict__ keys,
                             int B, DevCounters* __restrict__ ctr, const int32_t* __restrict__ slot,
                             const int64_t* __restrict__ seg, const Row* __restrict__ old_row,
                             const int64_t* __restrict__ off, long long tail, const long long* __restrict__ dpos,
                             const long long* __restrict__ E, bool long_in_place) {
    const long long nh = ctr->n_half;
    long long nnz_delta = 0, bytes = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nh; k += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = keys[k];
        const int32_t u = key_u(key, B);
        const int a = slot[u];
        const long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1], e0 = seg[3 * (int64_t)a + 2];
        const Row r = old_row[a];
        int32_t* O = pool + r.start;
        if (k < sp) {
            const int32_t y = key_v(key, B);
            const long long ubo = ub_masked(O, r.len, y);
            const long long ubd = ub_span(KeySpan{keys + sp, B}, e0 - sp, y);
            const long long del = E[sp + ubd] - E[sp];
            pool[tail + off[a] + (k - b0) + ubo - del] = y;
        } else {
            const long long dp = dpos[k];
            if (dp & 1) O[dp >> 1] = key_v(key, B) | (int32_t)0x80000000;
        }
        if (k == b0) {
            const long long p = sp - b0, q = e0 - sp;
            const long long nl = (long long)r.len + p - (E[e0] - E[sp]);
            row[u] = in_place_row(p, r.len, long_in_place) ? Row{r.start, (int)nl, r.cap}
                                            : Row{tail + off[a], (int)nl, (int)(r.len + p)};
            nnz_delta += nl - r.len;
            bytes += 4 * (r.len + nl) + 8 * (p + q) + 16;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nnz_delta += __shfl_xor_sync(__activemask(), nnz_delta, o);
        bytes += __shfl_xor_sync(__activemask(), bytes, o);
    }
    if (lane_id() == 0 && (nnz_delta || bytes)) {
        atomicAdd((unsigned long long*)&ctr->nnz_delta, (unsigned long long)nnz_delta);
        atomicAdd((unsigned long long*)&ctr->update_bytes, (unsigned long long)bytes);
    }
}

// Short rows, balanced: the short rows' old lengths are scanned (soff) and cut into groups of
// about UNIT entries (a row belongs to the group its first entry falls in), one warp per
// group. The warp takes the group's rows 32 at a time, one row per lane, and streams their
// entries 32 at a time, every lane finding its row by a search over the lanes' prefix sums.
// A surviving entry x lands at (survivors of its row before it) + (#insertions of its row
// < x); the insertion values of the 32 rows are staged in shared memory when they fit, and
// per-row survivor counts carry across chunks in shared memory.
constexpr int MERGE_THREADS = 256;
constexpr int UNIT = 1024;
constexpr int ICAP = 512;

__global__ void __launch_bounds__(MERGE_THREADS) k_merge_small(
        int32_t* __restrict__ pool, const unsigned long long* __restrict__ keys, int B,
        const DevCounters* __restrict__ ctr, const int64_t* __restrict__ seg, const Row* __restrict__ old_row,
        const int64_t* __restrict__ off, long long tail, const int32_t* __restrict__ small,
        const int64_t* __restrict__ soff) {
    __shared__ int s_cnt[MERGE_THREADS / WARP][WARP];
    __shared__ int32_t s_ins[MERGE_THREADS / WARP][ICAP];
    const int w = threadIdx.x / WARP;
    const unsigned lane = lane_id();
    const int ns = ctr->n_small;
    const long long total = soff[ns];
    const long long G = (total + UNIT - 1) / UNIT;
    for (long long g = gwarp_id(); g < G; g += gwarp_count()) {
        const long long i0 = warp_lower_bound(soff, ns, g * UNIT);
        const long long i1 = warp_lower_bound(soff, ns, (g + 1) * UNIT);
        for (long long rb = i0; rb < i1; rb += WARP) {
            const long long i = rb + lane;
            long long st = 0, ob = 0, ib = 0;
            int len = 0, p = 0;
            if (i < i1) {
                const int a = small[i];
                const Row r = old_row[a];
                st = r.start;
                len = r.len;
                ib = seg[3 * (int64_t)a];
                p = (int)(seg[3 * (int64_t)a + 1] - ib);
                ob = in_place_row(p, len, false) ? st : tail + off[a];   // short: the flag is moot
            }
            s_cnt[w][lane] = 0;
            const int pin = warp_incl_scan_i(p);
            const int ptot = __shfl_sync(0xffffffffu, pin, WARP - 1);
            const int pex = pin - p;
            const bool staged = ptot <= ICAP;
            if (staged)
                for (int t = 0; t < p; t++) s_ins[w][pex + t] = key_v(keys[ib + t], B);
            __syncwarp();
            const int incl = warp_incl_scan_i(len);
            const int tot = __shfl_sync(0xffffffffu, incl, WARP - 1);
            const int excl = incl - len;
            constexpr int U = 4;   // chunks per step: their loads are issued before any store
            for (int e00 = 0; e00 < tot; e00 += U * WARP) {
                int jj[U];
                int32_t xx[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int e = e00 + u * WARP + (int)lane;
                    int lo = 0, hi = WARP - 1;
#pragma unroll
                    for (int it = 0; it < 5; it++) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (__shfl_sync(0xffffffffu, excl, mid) <= e) lo = mid; else hi = mid - 1;
                    }
                    jj[u] = lo;
                    const int ej = __shfl_sync(0xffffffffu, excl, lo);
                    const long long sj = __shfl_sync(0xffffffffu, st, lo);
                    xx[u] = e < tot ? pool[sj + (e - ej)] : -1;
                }
                // rows rewritten in place: every load of this step precedes every store (a
                // survivor's store lands at or before its load, and before any later load)
                __syncwarp();
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int e0 = e00 + u * WARP;
                    if (e0 >= tot) break;   // uniform
                    const int j = jj[u];
                    const int32_t x = xx[u];
                    const int e = e0 + (int)lane;
                    const int ej = __shfl_sync(0xffffffffu, excl, j);
                    const int lj = __shfl_sync(0xffffffffu, len, j);
                    const long long oj = __shfl_sync(0xffffffffu, ob, j);
                    const long long ij = __shfl_sync(0xffffffffu, ib, j);
                    const int pj = __shfl_sync(0xffffffffu, p, j);
                    const int xj = __shfl_sync(0xffffffffu, pex, j);
                    const bool in = e < tot;
                    const bool surv = x >= 0;
                    const unsigned m = __ballot_sync(0xffffffffu, surv);
                    const int fl = max(ej - e0, 0);                    // first lane of row j in this chunk
                    const int ll = min(ej + lj - e0, WARP) - 1;        // last lane of row j in this chunk
                    const unsigned below = (1u << lane) - 1;
                    const unsigned from_fl = ~((1u << fl) - 1);
                    if (surv) {
                        int lbI = 0;
                        if (pj > 0) {
                            if (staged) {
                                int a = 0, b = pj;
                                while (a < b) { int mid = (a + b) >> 1; if (s_ins[w][xj + mid] < x) a = mid + 1; else b = mid; }
                                lbI = a;
                            } else {
                                lbI = (int)lb_span(KeySpan{keys + ij, B}, pj, x);
                            }
                        }
                        pool[oj + s_cnt[w][j] + __popc(m & below & from_fl) + lbI] = x;
                    }
                    __syncwarp();
                    if (in && (int)lane == ll) {
                        const unsigned upto = ll >= WARP - 1 ? 0xffffffffu : ((1u << (ll + 1)) - 1);
                        s_cnt[w][j] += __popc(m & upto & from_fl);
                    }
                    __syncwarp();
                }
            }
        }
    }
}

// Long rows that only lose entries, compacted in place: one block per row streams it front to
// back in chunks of LIP_CHUNK entries; every entry of a chunk is loaded before any survivor
// of that chunk is stored, and a survivor's new position (survivors before it in the row)
// never exceeds its old one, so no store lands on an entry still to be read.
constexpr int LIP_THREADS = 256;
constexpr int LIP_U = 4;
constexpr int LIP_CHUNK = LIP_THREADS * LIP_U;

__global__ void __launch_bounds__(LIP_THREADS) k_merge_long_inplace(int32_t* __restrict__ pool,
                                                                    const DevCounters* __restrict__ ctr,
                                                                    const int32_t* __restrict__ longs,
                                                                    const Row* __restrict__ old_row) {
    __shared__ int s_warp[LIP_U][LIP_THREADS / WARP];
    const int t = threadIdx.x, w = t / WARP;
    const unsigned lt = (1u << lane_id()) - 1;
    const int nl = ctr->n_large;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const Row r = old_row[longs[li]];
        int32_t* O = pool + r.start;
        long long run = 0;
        for (long long b = 0; b < r.len; b += LIP_CHUNK) {
            int32_t x[LIP_U];
            unsigned m[LIP_U];
#pragma unroll
            for (int u = 0; u < LIP_U; u++) {
                const long long i = b + u * LIP_THREADS + t;
                x[u] = i < r.len ? O[i] : -1;
                m[u] = __ballot_sync(0xffffffffu, x[u] >= 0);
                if (lane_id() == 0) s_warp[u][w] = __popc(m[u]);
            }
            __syncthreads();   // every load of the chunk is done; the warp counts are visible
            long long base = run;
#pragma unroll
            for (int u = 0; u < LIP_U; u++) {
                int before = 0, total = 0;
#pragma unroll
                for (int k = 0; k < LIP_THREADS / WARP; k++) {
                    const int cnt = s_warp[u][k];
                    before += k < w ? cnt : 0;
                    total += cnt;
                }
                if (x[u] >= 0) O[base + before + __popc(m[u] & lt)] = x[u];
                base += total;
            }
            run = base;
            __syncthreads();   // the counts are read before the next chunk overwrites them
        }
    }
}

// Rows past SMALL_LEN: one warp per slice of SLICE old-row entries (most rows a batch touches
// in a scale-free graph are its hubs, so this merge carries most of the bytes, with a few
// instructions per entry: a ballot, a population count, and a search of the insertions only
// where they fall inside a chunk's value range). The survivors before the slice are
// its start minus the matched deletions before it (one search in the non-decreasing dpos);
// survivor x lands at (#survivors before it) + (#insertions < x), the insertion count
// searched only inside the range spanned by the chunk's values.
//
// A slice of an HBM row is staged in shared memory by the bulk-copy engine: each warp owns two
// MS_CH-entry buffers and their mbarriers; lane 0 issues cp.async.bulk (non-multicast) of the
// 16-byte-aligned cover of the next chunk while the warp merges the current one from shared
// memory, so the old row is read in MS_CH * 4-byte transfers with no load instruction per
// entry. Every wait on an mbarrier is bounded: past the limit the warp flags sort_err = 3,
// waits (bounded again) for its copies in flight and leaves. Rows in host memory (tiered
// store) and slices whose aligned cover would pass the pool's end are read with direct loads.
constexpr int MS_WARPS = 8;
constexpr int MS_THREADS = MS_WARPS * WARP;
constexpr int MS_CH = 512;                 // entries per staged chunk
constexpr int MS_BUF = MS_CH + 8;          // buffer: chunk + 16-byte alignment slack on both ends
constexpr int MS_ISTAGE = 448;             // insertion keys of a slice (or one merge step) staged per warp (48 KB static limit)
constexpr long long MBAR_SPIN_LIMIT = 1ll << 24;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// lane 0: one arrival that expects `bytes`, then the bulk copy global -> shared completing on bar
__device__ __forceinline__ void bulk_g2s(int32_t* dst, const int32_t* src, unsigned bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// all lanes: bounded wait for the given phase of bar; false when the limit was reached
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (long long it = 0; it < MBAR_SPIN_LIMIT; it++) {
        if (mbar_test(bar, parity)) return true;
        if (it > 64) __nanosleep(128);
    }
    return false;
}

// First index i in [0, n] with I[i] >= x (I ascending), 32 probes per step (every lane calls
// it and gets the same answer): a search of a few thousand keys is three dependent loads.
__device__ __forceinline__ long long warp_lb_key(const KeySpan& I, long long n, int32_t x) {
    long long lo = 0, hi = n;
    while (hi - lo > WARP) {
        const long long step = (hi - lo + WARP - 1) / WARP;
        const long long pos = lo + (long long)lane_id() * step;
        const int c = __popc(__ballot_sync(0xffffffffu, pos < hi && I[pos] < x));   // probes below x
        if (c == 0) { hi = lo; break; }
        const long long nlo = lo + (long long)(c - 1) * step + 1;
        hi = min(hi, lo + (long long)c * step);
        lo = nlo;
    }
    const long long pos = lo + lane_id();
    return lo + __popc(__ballot_sync(0xffffffffu, pos < hi && I[pos] < x));
}

// First index i in [from, p] with I[i] >= t (I ascending), the warp reading 32 keys per step
// forward from `from`; every lane calls it and gets the same answer.
__device__ __forceinline__ long long ins_advance(const KeySpan& I, long long p, long long from, int32_t t) {
    for (long long i = from; i < p; i += WARP) {
        const long long j = i + lane_id();
        const unsigned m = __ballot_sync(0xffffffffu, j < p && I[j] < t);   // a prefix of the lanes
        const int k = __popc(m);
        if (k < WARP) return i + k;
    }
    return p;
}

// Merges old-row entries [b, e) (absolute pool indices) read through `get`, updating the running
// survivor count; every lane calls it. Survivor x lands at run + (survivors before it in its
// step) + (insertions < x). With pre >= 0 the slice's whole insertion range I[i0, i0 + pre)
// is already in s_ins and each survivor searches it there. Otherwise the insertions below the
// step's smallest value are `cur`, which only moves forward along the row (the old entries are
// ascending): each step advances it to its value range [xmin, xmax) with coalesced reads of
// the insertion keys, stages the keys of that range in s_ins when they fit, and searches them.
template <typename Get>
__device__ __forceinline__ void merge_span(long long b, long long e, Get get, int32_t* out, long long& run,
                                           const KeySpan& I, long long p, long long& cur, int32_t* s_ins,
                                           int pre, long long i0, unsigned lt) {
    constexpr int U = 4;
    for (long long base = b; base < e; base += U * WARP) {
        int32_t x[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const long long i = base + u * WARP + lane_id();
            x[u] = i < e ? get(i) : -1;
        }
        if (pre >= 0) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool surv = x[u] >= 0;
                const unsigned m = __ballot_sync(0xffffffffu, surv);
                if (surv) {
                    int lo = 0, hi = pre;
                    while (lo < hi) { const int mid = (lo + hi) >> 1; if (s_ins[mid] < x[u]) lo = mid + 1; else hi = mid; }
                    out[run + __popc(m & lt) + i0 + lo] = x[u];
                }
                run += __popc(m);
            }
            continue;
        }
        long long cl = cur, nin = 0;
        if (cur < p) {
            int xmin = INT32_MAX, xmax = -1;
#pragma unroll
            for (int u = 0; u < U; u++)
                if (x[u] >= 0) { xmin = min(xmin, x[u]); xmax = max(xmax, x[u]); }
            xmin = __reduce_min_sync(0xffffffffu, xmin);
            xmax = __reduce_max_sync(0xffffffffu, xmax);
            if (xmax >= 0) {
                cl = ins_advance(I, p, cur, xmin);
                const long long ch = ins_advance(I, p, cl, xmax);
                nin = ch - cl;
                cur = ch;
                if (nin > 0 && nin <= MS_ISTAGE) {
                    for (long long j = lane_id(); j < nin; j += WARP) s_ins[j] = I[cl + j];
                    __syncwarp();
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool surv = x[u] >= 0;
            const unsigned m = __ballot_sync(0xffffffffu, surv);
            if (surv) {
                long long lbI = cl;
                if (nin > 0) {
                    if (nin <= MS_ISTAGE) {
                        int lo = 0, hi = (int)nin;
                        while (lo < hi) { const int mid = (lo + hi) >> 1; if (s_ins[mid] < x[u]) lo = mid + 1; else hi = mid; }
                        lbI += lo;
                    } else {
                        lbI += lb_span(KeySpan{I.k + cl, I.B}, nin, x[u]);
                    }
                }
                out[run + __popc(m & lt) + lbI] = x[u];
            }
            run += __popc(m);
        }
        __syncwarp();   // s_ins is read before the next step stages another range
    }
}

__global__ void __launch_bounds__(MS_THREADS) k_merge_slices(
        int32_t* __restrict__ pool, long long pool_cap, const unsigned long long* __restrict__ keys, int B,
        DevCounters* __restrict__ ctr, const int64_t* __restrict__ seg, const Row* __restrict__ old_row,
        const int64_t* __restrict__ off, long long tail, const long long* __restrict__ E,
        const long long* __restrict__ dpos, const int64_t* __restrict__ slices, int64_t slice_cap,
        bool long_in_place) {
    __shared__ __align__(16) int32_t s_buf[MS_WARPS][2][MS_BUF];
    __shared__ __align__(8) uint64_t s_bar[MS_WARPS][2];
    __shared__ int32_t s_ins[MS_WARPS][MS_ISTAGE];
    const int w = threadIdx.x / WARP;
    const unsigned lt = (1u << lane_id()) - 1;
    if (lane_id() == 0) {
        mbar_init(&s_bar[w][0]);
        mbar_init(&s_bar[w][1]);
        fence_proxy_async_smem();   // the initialised barriers are visible to the bulk-copy engine
    }
    __syncwarp();
    unsigned phase[2] = {0u, 0u};
    const long long nsl = min((long long)ctr->n_slices, (long long)slice_cap);
    for (long long it = gwarp_id(); it < nsl; it += gwarp_count()) {
        const long long item = slices[it];
        const int a = (int)(item >> 32), s = (int)(item & 0xffffffffLL);
        const Row r = old_row[a];
        const long long b0 = seg[3 * (int64_t)a], sp = seg[3 * (int64_t)a + 1], e0 = seg[3 * (int64_t)a + 2];
        const long long p = sp - b0, q = e0 - sp;
        const long long s0 = (long long)s * SLICE, s1 = min((long long)r.len, s0 + SLICE);
        if (s0 >= s1) continue;
        long long md = 0;
        if (q > 0 && s0 > 0 && lane_id() == 0) {
            long long lo = 0, hi = q;
            while (lo < hi) { long long mid = (lo + hi) >> 1; if ((dpos[sp + mid] >> 1) < s0) lo = mid + 1; else hi = mid; }
            md = E[sp + lo] - E[sp];
        }
        long long run = s0 - __shfl_sync(0xffffffffu, md, 0);
        // a row compacted in place is one slice here: every survivor lands at or before its old
        // position, which its warp has already read
        int32_t* out = pool + (in_place_row(p, r.len, long_in_place) ? r.start : tail + off[a]);
        const KeySpan I{keys + b0, B};
        const long long abs0 = r.start + s0, abs1 = r.start + s1;   // pool indices of the slice
        // The insertions that can land among this slice's entries: I[i0, i1), i0 those below its
        // first value, i1 those below its last (tombstones keep the value under the sign bit).
        // When they fit they are staged in shared memory once for the whole slice.
        long long i0 = 0, i1 = p;
        if (p > 0) {
            if (s0 > 0) i0 = warp_lb_key(I, p, unmark(pool[abs0]));
            if (s1 < r.len) i1 = warp_lb_key(I, p, unmark(pool[abs1 - 1]));
        }
        const int pre = i1 - i0 <= MS_ISTAGE ? (int)(i1 - i0) : -1;
        if (pre > 0) {
            int32_t* si = s_ins[w];
            for (int j0 = 0; j0 < pre; j0 += 4 * WARP) {
                int32_t v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int j = j0 + u * WARP + (int)lane_id();
                    v[u] = j < pre ? I[i0 + j] : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int j = j0 + u * WARP + (int)lane_id();
                    if (j < pre) si[j] = v[u];
                }
            }
            __syncwarp();
        }
        long long cur = i0;
        const bool staged = r.start >= 0 && ((abs1 + 3) & ~3LL) <= pool_cap;
        if (!staged) {
            merge_span(abs0, abs1, [&](long long i) { return pool[i]; }, out, run, I, p, cur, s_ins[w], pre, i0, lt);
            __syncwarp();   // s_ins is read before the next slice stages its insertions
            continue;
        }
        const int nch = (int)((s1 - s0 + MS_CH - 1) / MS_CH);
        auto issue = [&](int k) {   // lane 0
            const long long lo = abs0 + (long long)k * MS_CH, hi = min(abs1, lo + MS_CH);
            const long long a0 = lo & ~3LL, a1 = (hi + 3) & ~3LL;
            bulk_g2s(s_buf[w][k & 1], pool + a0, (unsigned)((a1 - a0) * 4), &s_bar[w][k & 1]);
        };
        if (lane_id() == 0) {
            issue(0);
            if (nch > 1) issue(1);
        }
        for (int k = 0; k < nch; k++) {
            const int bsel = k & 1;
            if (!mbar_wait(&s_bar[w][bsel], phase[bsel])) {
                // give up: flag it, let the copies in flight land (bounded), leave
                if (lane_id() == 0) atomicCAS(&ctr->sort_err, 0, 3);
                mbar_wait(&s_bar[w][bsel], phase[bsel]);
                if (k + 1 < nch) mbar_wait(&s_bar[w][bsel ^ 1], phase[bsel ^ 1]);
                return;
            }
            phase[bsel] ^= 1u;
            const long long lo = abs0 + (long long)k * MS_CH, hi = min(abs1, lo + MS_CH);
            const int32_t* sb = s_buf[w][bsel] - (lo & ~3LL);   // indexed by absolute pool index
            merge_span(lo, hi, [&](long long i) { return sb[i]; }, out, run, I, p, cur, s_ins[w], pre, i0, lt);
            __syncwarp();   // every lane is done with this buffer before it is refilled
            if (k + 2 < nch && lane_id() == 0) {
                fence_proxy_async_smem();   // the warp's reads of the buffer precede the copy's writes
                issue(k + 2);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Compaction and download
// ---------------------------------------------------------------------------------------
__global__ void k_row_lens(const Row* __restrict__ row, int64_t n, int64_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        out[v] = row[v].len;
}

// Merge-path tiles: row r costs one unit and each of its entries one more, so row r starts
// at unit r + off[r] and entry e of row r sits at unit r + 1 + e. One block copies the
// entries of COPY_UNITS units: at most COPY_UNITS + 1 rows and COPY_UNITS entries, whatever
// mix of hubs, short rows and empty rows the range holds. The rows are found with a warp
// search and indexed in shared memory (output and source begin per row); every thread then
// copies COPY_UNITS / COPY_THREADS entries, finding each entry's row by a search of the
// index, with all its loads in flight before the stores.
constexpr int COPY_UNITS = 2048;
constexpr int COPY_THREADS = 256;

// first r in [0, n) with r + off[r] > x (n if none), 32 probes per step (all lanes call)
__device__ __forceinline__ long long warp_first_unit_above(const int64_t* off, long long n, long long x) {
    long long lo = 0, hi = n;
    while (hi - lo > WARP) {
        const long long step = (hi - lo + WARP - 1) / WARP;
        const long long pos = lo + (long long)lane_id() * step;
        const bool le = pos < hi && pos + off[pos] <= x;
        const int c = __popc(__ballot_sync(0xffffffffu, le));
        const long long nlo = c == 0 ? lo : lo + (long long)(c - 1) * step + 1;
        const long long nhi = c == 0 ? lo : min(hi, lo + (long long)c * step);
        lo = nlo;
        hi = max(nlo, nhi);
        if (c == 0) break;
    }
    const long long pos = lo + lane_id();
    const bool le = pos < hi && pos + off[pos] <= x;
    return lo + __popc(__ballot_sync(0xffffffffu, le));
}

__global__ void __launch_bounds__(COPY_THREADS) k_copy_rows(const Row* __restrict__ row, const int32_t* __restrict__ src,
                                                            int32_t* __restrict__ dst, const int64_t* __restrict__ off,
                                                            int32_t n, long long live) {
    __shared__ long long s_ra, s_rb;
    __shared__ int s_ob[COPY_UNITS + 2];
    __shared__ long long s_sb[COPY_UNITS + 2];
    const long long units = (long long)n + live;
    for (long long d0 = (long long)blockIdx.x * COPY_UNITS; d0 < units; d0 += (long long)gridDim.x * COPY_UNITS) {
        const long long d1 = min(units, d0 + COPY_UNITS);
        if (threadIdx.x < WARP) {
            const long long ra = warp_first_unit_above(off, n, d0) - 1;       // last row starting at or before d0
            const long long rb = warp_first_unit_above(off, n, d1 - 1) - 1;   // last row starting before d1
            if (threadIdx.x == 0) { s_ra = ra; s_rb = rb; }
        }
        __syncthreads();
        const long long ra = s_ra;
        const int nr = (int)(s_rb - ra + 1);
        const long long ef = max((long long)off[ra], d0 - ra - 1);            // first entry of the tile
        long long el = min((long long)off[s_rb + 1], d1 - s_rb - 1);          // one past the last
        if (el < ef) el = ef;
        for (int i = threadIdx.x; i < nr; i += COPY_THREADS) {
            const long long r = ra + i;
            const long long b = off[r];
            const long long eb = max(b, d0 - r - 1);
            s_ob[i] = (int)(min(eb, el) - ef);
            s_sb[i] = row[r].start + (eb - b);
        }
        __syncthreads();
        const int span = (int)(el - ef);
        constexpr int U = COPY_UNITS / COPY_THREADS;
        int32_t v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int rel = threadIdx.x + u * COPY_THREADS;
            v[u] = 0;
            if (rel < span) {
                int lo = 0, hi = nr - 1;   // last row whose output begin is <= rel
                while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (s_ob[mid] <= rel) lo = mid; else hi = mid - 1; }
                v[u] = src[s_sb[lo] + (rel - s_ob[lo])];
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int rel = threadIdx.x + u * COPY_THREADS;
            if (rel < span) dst[ef + rel] = v[u];
        }
        __syncthreads();
    }
}

__global__ void k_rows_compacted(Row* __restrict__ row, const int64_t* __restrict__ off, int32_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        long long s = off[v];
        int len = row[v].len;
        row[v] = Row{s, len, len};
    }
}

// ---- tiered store ---------------------------------------------------------------------------
__device__ __forceinline__ bool in_hbm(const Row& r, long long cap) { return r.start >= 0 && r.start < cap; }
__device__ __forceinline__ int len_bin(int len) { return 31 - __clz(len + 1); }

__global__ void k_row_lens_hbm(const Row* __restrict__ row, int64_t n, long long cap, int64_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const Row r = row[v];
        out[v] = in_hbm(r, cap) ? r.len : 0;
    }
}

// HBM entries by floor(log2(1 + row length)) (32 bins), for the eviction threshold.
__global__ void k_hbm_hist(const Row* __restrict__ row, int64_t n, long long cap, unsigned long long* __restrict__ hist) {
    __shared__ unsigned long long sh[32];
    if (threadIdx.x < 32) sh[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const Row r = row[v];
        if (in_hbm(r, cap) && r.len > 0) atomicAdd(&sh[len_bin(r.len)], (unsigned long long)r.len);
    }
    __syncthreads();
    if (threadIdx.x < 32 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

__global__ void k_row_lens_evict(const Row* __restrict__ row, int64_t n, long long cap, int bins,
                                 int64_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const Row r = row[v];
        out[v] = (in_hbm(r, cap) && r.len > 0 && len_bin(r.len) < bins) ? r.len : 0;
    }
}

__global__ void k_rows_evicted(Row* __restrict__ row, const int64_t* __restrict__ off, int64_t n, long long cap,
                               int bins, long long host_base) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const Row r = row[v];
        if (in_hbm(r, cap) && r.len > 0 && len_bin(r.len) < bins) row[v] = Row{host_base + off[v], r.len, r.len};
    }
}

// Split batches: the allocation of an affected row goes to the host lengths when its old
// version lives in the host pool (lenH keeps the HBM rows' allocations).
__global__ void k_split_alloc(const Row* __restrict__ old_row, const DevCounters* __restrict__ ctr, long long cap,
                              int64_t* __restrict__ lenH, int64_t* __restrict__ lenC) {
    const int A = ctr->n_aff;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A; a += gridDim.x * blockDim.x) {
        if (!in_hbm(old_row[a], cap)) {
            lenC[a] = lenH[a];
            lenH[a] = 0;
        }
    }
}

// Absolute destinations (element offsets from the HBM pool) of a split batch's rows.
__global__ void k_abs_off(const Row* __restrict__ old_row, const DevCounters* __restrict__ ctr, long long cap,
                          int64_t* __restrict__ offH, const int64_t* __restrict__ offC, long long hbm_base,
                          long long host_base) {
    const int A = ctr->n_aff;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A; a += gridDim.x * blockDim.x)
        offH[a] = in_hbm(old_row[a], cap) ? hbm_base + offH[a] : host_base + offC[a];
}

// After the HBM rows were copied to the new pool: HBM rows point at their copies, host rows
// keep their address (their offset is re-based on the new pool).
__global__ void k_rows_compacted_tiered(Row* __restrict__ row, const int64_t* __restrict__ off, int32_t n,
                                        long long cap, long long rebase) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const Row r = row[v];
        if (in_hbm(r, cap)) row[v] = Row{(long long)off[v], r.len, r.len};
        else row[v] = Row{r.start + rebase, r.len, r.cap};
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
        (size_t)H * 8, (size_t)H * 8, (size_t)(H + 1) * 8,
        (size_t)H * 4, (size_t)3 * H * 8, (size_t)(H + 1) * 8, (size_t)H * 4, (size_t)(H + 1) * 8, (size_t)H * sizeof(Row),
        (size_t)(H + 1) * 8, (size_t)H * 4};
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
    c->d_small_off = (int64_t*)take(sz[10]);
    c->d_old_row = (Row*)take(sz[11]);
    c->d_aff_len2 = (int64_t*)take(sz[12]);
    c->d_aff_long = (int32_t*)take(sz[13]);
    c->d_hkeys = c->d_keys;
    return SCOUT_OK;
}

int graph_reserve_batch(scout_ctx* c, int64_t m) {
    SCOUT_RC(lists_ensure(c));
    SCOUT_RC(ws_ensure(c, m));
    const int64_t Amax = std::min<int64_t>(2 * m, c->n);
    SCOUT_RC(dev_grow(c, &c->d_slices, &c->cap_slices, c->pool_cap / SLICE + Amax + 1024, "merge slices"));
    SCOUT_RC(sort_reserve(c, std::max<int64_t>(2 * c->ws_m, c->n + 1)));
    if (!c->d_coff) SCOUT_RC(dev_alloc(c, (void**)&c->d_coff, (size_t)(c->n + 1) * sizeof(int64_t), "compaction offsets"));
    // the compaction target, when the budget leaves room for a second pool
    if (!c->spare && c->held + (uint64_t)c->pool_cap * 4 <= c->budget / 100 * 85) {
        SCOUT_RC(dev_alloc(c, (void**)&c->spare, (size_t)c->pool_cap * 4, "element pool"));
        c->spare_cap = c->pool_cap;
    }
    SCOUT_RC(pin_grow(c, &c->h_pin_edits, &c->cap_pin_edits, m * (int64_t)sizeof(scout_edge) + m + 1));
    return SCOUT_OK;
}

int lists_ensure(scout_ctx* c) {
    SCOUT_RC(graph_ensure_scratch(c));
    if (c->d_list[0]) return SCOUT_OK;
    // Queue items are (chunk << 32 | vertex); a vertex pushed once per round occupies at most
    // ceil(len / chunk) items with chunk >= 256 entries, so n + nnz / 256 + slack bounds a round.
    c->qcap = c->n + (c->pool_cap / 256) + 4096;
    for (int i = 0; i < 3; i++) SCOUT_RC(dev_alloc(c, &c->d_qbuf[i], (size_t)c->qcap * 8, "work queues"));
    for (int i = 0; i < 2; i++) SCOUT_RC(dev_alloc(c, (void**)&c->d_list[i], (size_t)c->n * 4, "vertex lists"));
    SCOUT_RC(dev_alloc(c, (void**)&c->d_commit, (size_t)c->n * 8, "commit pairs"));
    return SCOUT_OK;
}

int batch_begin(scout_ctx* c) {
    SCOUT_RC(gather_finish(c, nullptr, nullptr, nullptr));   // no graph work while a gather runs
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
    if (c->h_ctr->sort_err == 1) return c->fail(SCOUT_E_TIMEOUT, "a sort look-back wait timed out");
    if (c->h_ctr->sort_err == 3) return c->fail(SCOUT_E_TIMEOUT, "a bulk copy of a row slice into shared memory did not complete");
    if (c->h_ctr->sort_err == 4) return c->fail(SCOUT_E_TIMEOUT, "a scan look-back wait timed out");
    if (c->h_ctr->sort_err) return c->fail(SCOUT_E_STATE, "the sort computed a position out of range");
    if (c->h_bar->err != 0 || c->h_ctr->overflow)
        return c->fail(SCOUT_E_CAPACITY, "a device work list overflowed its capacity");
    return SCOUT_OK;
}

int graph_ensure_scratch(scout_ctx* c) {
    if (c->stamp_a) return SCOUT_OK;
    size_t bytes = (size_t)c->n * sizeof(int32_t);
    int32_t** arrs[] = {&c->stamp_a, &c->stamp_b, &c->stamp_c, &c->stamp_d, &c->aux_v, &c->aux_w};
    for (auto a : arrs) {
        SCOUT_RC(dev_alloc(c, (void**)a, bytes, "per-vertex scratch"));
        SCOUT_CU(c, cudaMemsetAsync(*a, 0, bytes, c->s_main));
    }
    return SCOUT_OK;
}

// Rewrites the pool so rows are contiguous and leaves at least min_free free elements
// (the on-device half of compact_flash_graph). With nnz_exact the host's live count is used
// and nothing waits for the device; otherwise (after staging) the live count is read back.
static inline long long elem_delta(const int32_t* a, const int32_t* b) {
    return (long long)(((intptr_t)a - (intptr_t)b) / (intptr_t)sizeof(int32_t));
}

// Host pool compaction (tiered store), on the host: the host rows are moved down in order of
// their position (memmove, every destination at or below its source), and the row table is
// rewritten.
static int host_compact(scout_ctx* c) {
    const int64_t n = c->n;
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    std::vector<Row> rows((size_t)n);
    SCOUT_CU(c, cudaMemcpy(rows.data(), c->row, (size_t)n * sizeof(Row), cudaMemcpyDeviceToHost));
    const long long rel = elem_delta(c->host_pool, c->pool);
    std::vector<int32_t> ids;
    for (int64_t v = 0; v < n; v++) {
        const Row& r = rows[v];
        if (!(r.start >= 0 && r.start < c->pool_cap) && r.len > 0) ids.push_back((int32_t)v);
    }
    std::sort(ids.begin(), ids.end(), [&](int32_t a, int32_t b) { return rows[a].start < rows[b].start; });
    int64_t pos = 0;
    for (int32_t v : ids) {
        Row& r = rows[v];
        const int64_t from = r.start - rel;
        if (from != pos) std::memmove(c->host_pool + pos, c->host_pool + from, (size_t)r.len * 4);
        r.start = rel + pos;
        r.cap = r.len;
        pos += r.len;
    }
    SCOUT_CU(c, cudaMemcpy(c->row, rows.data(), (size_t)n * sizeof(Row), cudaMemcpyHostToDevice));
    c->host_tail = pos;
    return SCOUT_OK;
}

// Tiered compaction: only HBM rows move. When they and min_free do not fit the HBM pool, the
// shortest ones (whole log2 length classes, shortest first) are evicted to the host pool.
static int graph_compact_tiered(scout_ctx* c, int64_t min_free) {
    const int64_t n = c->n;
    if (!c->d_coff) SCOUT_RC(dev_alloc(c, (void**)&c->d_coff, (size_t)(n + 1) * sizeof(int64_t), "compaction offsets"));
    int64_t* off = c->d_coff;
    const int nb = blocks_for(n, 256);
    auto hbm_live = [&](int64_t* live) -> int {
        k_row_lens_hbm<<<nb, 256, 0, c->s_main>>>(c->row, n, (long long)c->pool_cap, off);
        SCOUT_LAUNCH(c, "k_row_lens_hbm");
        SCOUT_RC(scan_i64(c, off, n, off + n));
        SCOUT_CU(c, cudaMemcpyAsync(live, off + n, 8, cudaMemcpyDeviceToHost, c->s_main));
        SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
        return SCOUT_OK;
    };
    int64_t live = 0;
    SCOUT_RC(hbm_live(&live));
    if (live + min_free > c->pool_cap) {
        // 32 histogram slots in the scan partials (free between scans)
        SCOUT_RC(dev_grow(c, &c->d_scan_tmp, &c->cap_scan, 64, "scan partials"));
        unsigned long long* hist = (unsigned long long*)c->d_scan_tmp;
        SCOUT_CU(c, cudaMemsetAsync(hist, 0, 32 * 8, c->s_main));
        k_hbm_hist<<<nb, 256, 0, c->s_main>>>(c->row, n, (long long)c->pool_cap, hist);
        SCOUT_LAUNCH(c, "k_hbm_hist");
        unsigned long long h[32];
        SCOUT_CU(c, cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, c->s_main));
        SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
        int bins = 0;
        int64_t keep = live;
        while (bins < 32 && keep + min_free > c->pool_cap) keep -= (int64_t)h[bins++];
        if (keep + min_free > c->pool_cap)
            return c->fail(SCOUT_E_CAPACITY, "tiered store: the HBM pool cannot hold the rows of one batch");
        k_row_lens_evict<<<nb, 256, 0, c->s_main>>>(c->row, n, (long long)c->pool_cap, bins, off);
        SCOUT_LAUNCH(c, "k_row_lens_evict");
        SCOUT_RC(scan_i64(c, off, n, off + n));
        int64_t ev = 0;
        SCOUT_CU(c, cudaMemcpyAsync(&ev, off + n, 8, cudaMemcpyDeviceToHost, c->s_main));
        SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
        if (c->host_tail + ev > c->host_cap) {   // the HBM rows and their offsets stay as they are
            SCOUT_RC(host_compact(c));
            if (c->host_tail + ev > c->host_cap) return c->fail(SCOUT_E_CAPACITY, "tiered store: the host pool is full");
        }
        const int64_t tiles = (n + ev + COPY_UNITS - 1) / COPY_UNITS;
        k_copy_rows<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 32 * c->sm_count)), COPY_THREADS, 0,
                      c->s_main>>>(c->row, c->pool, c->host_pool + c->host_tail, off, (int32_t)n, (long long)ev);
        k_rows_evicted<<<nb, 256, 0, c->s_main>>>(c->row, off, n, (long long)c->pool_cap, bins,
                                                  elem_delta(c->host_pool, c->pool) + c->host_tail);
        SCOUT_LAUNCH(c, "eviction");
        c->host_tail += ev;
        c->evictions++;
        c->evicted_entries += ev;
        c->nlaunch += 8;
        SCOUT_RC(hbm_live(&live));
    }
    int64_t cap = c->pool_cap;
    int32_t* np = nullptr;
    if (c->spare && c->spare_cap >= cap) {
        np = c->spare;
        cap = c->spare_cap;
        c->spare = nullptr;
        c->spare_cap = 0;
    } else {
        if (c->spare) { dev_free(c, c->spare, (size_t)c->spare_cap * 4); c->spare = nullptr; c->spare_cap = 0; }
        SCOUT_RC(dev_alloc(c, (void**)&np, (size_t)cap * sizeof(int32_t), "element pool"));
    }
    const int64_t tiles = (n + live + COPY_UNITS - 1) / COPY_UNITS;
    k_copy_rows<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 32 * c->sm_count)), COPY_THREADS, 0,
                  c->s_main>>>(c->row, c->pool, np, off, (int32_t)n, (long long)live);
    k_rows_compacted_tiered<<<nb, 256, 0, c->s_main>>>(c->row, off, (int32_t)n, (long long)c->pool_cap,
                                                       elem_delta(c->pool, np));
    SCOUT_LAUNCH(c, "tiered compaction");
    c->nlaunch += 6;
    if (c->held <= c->budget / 100 * 85) {
        c->spare = c->pool;
        c->spare_cap = c->pool_cap;
    } else {
        dev_free(c, c->pool, (size_t)c->pool_cap * sizeof(int32_t));
    }
    c->compactions++;
    c->pool = np;
    c->pool_cap = cap;
    c->tail = live;
    return SCOUT_OK;
}

int graph_compact(scout_ctx* c, int64_t min_free, bool nnz_exact) {
    if (c->tiered) return graph_compact_tiered(c, min_free);
    const int64_t n = c->n;
    if (!c->d_coff) SCOUT_RC(dev_alloc(c, (void**)&c->d_coff, (size_t)(n + 1) * sizeof(int64_t), "compaction offsets"));
    int64_t* off = c->d_coff;
    int nb = blocks_for(n, 256);
    k_row_lens<<<nb, 256, 0, c->s_main>>>(c->row, n, off);
    SCOUT_LAUNCH(c, "k_row_lens");
    SCOUT_RC(scan_i64(c, off, n, off + n));
    int64_t live = c->nnz;
    if (!nnz_exact) {
        SCOUT_CU(c, cudaMemcpyAsync(&live, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->s_main));
        SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    }
    int64_t cap = std::max<int64_t>(c->pool_cap, live + min_free);
    // Ping-pong: the previous pool is kept as the next compaction's target, so steady-state
    // compactions allocate nothing. Without budget room for two pools the old one is freed.
    int32_t* np = nullptr;
    if (c->spare && c->spare_cap >= cap) {
        np = c->spare;
        cap = c->spare_cap;
        c->spare = nullptr;
        c->spare_cap = 0;
    } else {
        if (c->spare) { dev_free(c, c->spare, (size_t)c->spare_cap * 4); c->spare = nullptr; c->spare_cap = 0; }
        SCOUT_RC(dev_alloc(c, (void**)&np, (size_t)cap * sizeof(int32_t), "element pool"));
    }
    const int64_t tiles = (n + live + COPY_UNITS - 1) / COPY_UNITS;
    k_copy_rows<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 32 * c->sm_count)), COPY_THREADS, 0,
                  c->s_main>>>(c->row, c->pool, np, off, (int32_t)n, (long long)live);
    k_rows_compacted<<<nb, 256, 0, c->s_main>>>(c->row, off, (int32_t)n);
    SCOUT_LAUNCH(c, "compaction");
    c->nlaunch += 6;
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

static bool is_pinned(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Host memcpy into the pinned staging buffer, split over the host threads for large batches.
void stage_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t PART = (size_t)1 << 20;
    if (bytes < 4 * PART) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const int64_t parts = (int64_t)((bytes + PART - 1) / PART);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < parts; i++) {
        size_t o = (size_t)i * PART;
        std::memcpy((char*)dst + o, (const char*)src + o, std::min(PART, bytes - o));
    }
}

// Edits in pinned host memory are copied to the device directly; pageable ones go through the
// context's pinned staging buffer.
// Edits hinted by scout_prefetch and declared by this call are already on their way to the
// device (copy stream, ev_pf): the main stream waits for that copy and reads them there.
static int upload_edits(scout_ctx* c, const scout_edge* edits, const uint8_t* ops, int64_t m,
                        const scout_edge** d_src) {
    const bool hinted = c->pf_use && c->pf_ready && c->pf_ready_m == m && !ops;
    c->pf_use = false;
    if (c->pf_ready) c->pf_ready = false;   // consumed now, or stale (the next hint replaces it)
    if (hinted) {
        SCOUT_CU(c, cudaStreamWaitEvent(c->s_main, c->ev_pf, 0));
        *d_src = c->d_pf_edits[c->pf_slot];
        return SCOUT_OK;
    }
    *d_src = c->d_edits;
    const size_t eb = (size_t)m * sizeof(scout_edge);
    const bool pe = is_pinned(edits), po = !ops || is_pinned(ops);
    if (!pe || !po) {
        int64_t bytes = (int64_t)((pe ? 0 : eb) + (po ? 0 : (size_t)m));
        SCOUT_RC(pin_grow(c, &c->h_pin_edits, &c->cap_pin_edits, std::max<int64_t>(bytes, 1)));
    }
    const void* se = edits;
    if (!pe) {
        stage_copy(c->h_pin_edits, edits, eb);
        se = c->h_pin_edits;
    }
    SCOUT_CU(c, cudaMemcpyAsync(c->d_edits, se, eb, cudaMemcpyHostToDevice, c->s_main));
    if (ops) {
        const void* so = ops;
        if (!po) {
            char* dst = (char*)c->h_pin_edits + (pe ? 0 : eb);
            stage_copy(dst, ops, (size_t)m);
            so = dst;
        }
        SCOUT_CU(c, cudaMemcpyAsync(c->d_ops, so, (size_t)m, cudaMemcpyHostToDevice, c->s_main));
    }
    return SCOUT_OK;
}

int graph_update(scout_ctx* c, const scout_edge* edits, const uint8_t* ops, int64_t m, scout_batch_stats* st) {
    const int64_t n = c->n;
    const int B = key_bits_for(n);
    c->key_bits = B;
    // Free space must hold a rewrite of every live entry plus two entries per edit (tiered
    // store: the batch's exact growth is checked after the row allocation instead).
    int64_t need = c->tiered ? 2 * m + 1024 : c->nnz + 2 * m + 1024;
    SCOUT_CU(c, cudaEventRecord(c->ev_t[6], c->s_main));
    if (c->pool_cap - c->tail < need) SCOUT_RC(graph_compact(c, need, true));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[7], c->s_main));
    SCOUT_RC(ws_ensure(c, m));
    SCOUT_RC(graph_ensure_scratch(c));
    if (st) st->h2d_bytes += m * (int64_t)sizeof(scout_edge) + (ops ? m : 0);
    c->merge_tail = c->tail;
    if (m == 0) {
        c->d_hkeys = c->d_keys;
        SCOUT_CU(c, cudaEventRecord(c->ev_t[3], c->s_main));
        return SCOUT_OK;
    }
    const scout_edge* d_src = nullptr;
    SCOUT_RC(upload_edits(c, edits, ops, m, &d_src));
    SCOUT_CU(c, cudaEventRecord(c->ev_t[3], c->s_main));
    DGraph g = dgraph(c);
    k_classify<<<blocks_for(m, 256), 256, 0, c->s_main>>>(g, d_src, ops ? c->d_ops : nullptr, m, B, c->d_keys,
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
    // merge slices: the long rows' ceil(len / SLICE) sum to at most nnz / SLICE + Amax
    SCOUT_RC(dev_grow(c, &c->d_slices, &c->cap_slices, c->nnz / SLICE + Amax + 1024, "merge slices"));
    // split: tiered store, rows whose old version lives in HBM are rewritten into HBM and host
    // rows into the host pool (two scans); otherwise one scan for one destination
    auto row_alloc = [&](bool again, bool split) -> int {
        SCOUT_CU(c, cudaMemsetAsync(c->d_aff_len, 0, (size_t)(Amax + 1) * 8, c->s_main));
        SCOUT_CU(c, cudaMemsetAsync(c->d_small_off, 0, (size_t)(Amax + 1) * 8, c->s_main));
        if (again) SCOUT_CU(c, cudaMemsetAsync(&c->d_ctr->n_small, 0, 4 * sizeof(int), c->s_main));   // n_small .. n_pad
        k_row_alloc<<<blocks_for(Amax, 256), 256, 0, c->s_main>>>(c->row, c->d_ctr, c->d_aff, c->d_aff_seg,
                                                                  c->d_old_row, c->d_aff_len, c->d_aff_small,
                                                                  c->d_small_off, c->d_slices, c->cap_slices,
                                                                  c->d_aff_long, c->tiered);
        SCOUT_LAUNCH(c, "k_row_alloc");
        c->nlaunch += 1;
        if (split) {
            SCOUT_CU(c, cudaMemsetAsync(c->d_aff_len2, 0, (size_t)(Amax + 1) * 8, c->s_main));
            k_split_alloc<<<blocks_for(Amax, 256), 256, 0, c->s_main>>>(c->d_old_row, c->d_ctr, (long long)c->pool_cap,
                                                                        c->d_aff_len, c->d_aff_len2);
            SCOUT_LAUNCH(c, "k_split_alloc");
            c->nlaunch += 1;
            SCOUT_RC(scan_i64(c, c->d_aff_len2, Amax + 1, (int64_t*)&c->d_ctr->new_elems_host));
        } else if (again) {
            SCOUT_CU(c, cudaMemsetAsync(&c->d_ctr->new_elems_host, 0, 8, c->s_main));
        }
        // Exclusive scan over Amax + 1 entries (the tail entries are zero): the new row of
        // affected row a starts at tail + off[a]; the total is this batch's pool growth.
        return scan_i64(c, c->d_aff_len, Amax + 1, (int64_t*)&c->d_ctr->new_elems);
    };
    c->batch_dest = c->tiered ? 2 : 0;
    SCOUT_RC(row_alloc(false, c->tiered));
    long long dest = c->tail;   // element offset from the HBM pool where the new rows start
    if (c->tiered) {
        // the exact growth, before anything is written. HBM part too large: compact (evicting
        // short rows to the host pool); larger than three quarters of the HBM pool: the whole
        // batch goes to the host pool. Host pool full: compacted in place on the host.
        long long grow[2] = {0, 0};   // HBM, host
        auto read_grow = [&]() -> int {
            SCOUT_CU(c, cudaMemcpyAsync(grow, &c->d_ctr->new_elems, 16, cudaMemcpyDeviceToHost, c->s_main));
            SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
            return SCOUT_OK;
        };
        SCOUT_RC(read_grow());
        // a hinted next batch is gathered into the free HBM above this merge: keep room for about
        // its endpoint rows at the average degree (two per edit), at most a quarter of the pool.
        // More room means evicting more rows to the host pool on every compaction, which costs
        // more over the host link than the merge saves on the gathered rows.
        long long headroom = 0;
        if (c->pf_pending && c->pf_m > 0) {
            const long long avg = c->n > 0 ? (c->nnz + c->n - 1) / c->n : 1;
            headroom = std::min<long long>(c->pool_cap / 4, 2 * c->pf_m * avg + 4096);
        }
        if (c->tail + grow[0] + 1024 + headroom > c->pool_cap) {
            if (grow[0] + 1024 + headroom <= c->pool_cap / 4 * 3) {
                SCOUT_RC(graph_compact(c, grow[0] + 1024 + headroom, true));
            } else if (c->tail + grow[0] + 1024 <= c->pool_cap) {
                // the gather gets what is left
            } else if (grow[0] + 1024 <= c->pool_cap / 4 * 3) {
                SCOUT_RC(graph_compact(c, grow[0] + 1024, true));
            } else {
                c->batch_dest = 1;
                c->host_batches++;
            }
            SCOUT_RC(row_alloc(true, c->batch_dest == 2));
            SCOUT_RC(read_grow());
        }
        const long long host_need = c->batch_dest == 1 ? grow[0] : grow[1];
        if (c->host_tail + host_need > c->host_cap) {
            SCOUT_RC(host_compact(c));
            if (c->host_tail + host_need > c->host_cap)
                return c->fail(SCOUT_E_CAPACITY, "tiered store: the host pool cannot take this batch's rows");
            SCOUT_RC(row_alloc(true, c->batch_dest == 2));
        }
        c->merge_tail = c->tail + (c->batch_dest == 1 ? 0 : grow[0]);
        const long long host_base = elem_delta(c->host_pool, c->pool) + c->host_tail;
        if (c->batch_dest == 1) {
            dest = host_base;
        } else {
            k_abs_off<<<blocks_for(Amax, 256), 256, 0, c->s_main>>>(c->d_old_row, c->d_ctr, (long long)c->pool_cap,
                                                                    c->d_aff_len, c->d_aff_len2, (long long)c->tail,
                                                                    host_base);
            SCOUT_LAUNCH(c, "k_abs_off");
            c->nlaunch += 1;
            dest = 0;   // the offsets are absolute
        }
    }
    long long* dpos = (long long*)(sorted == c->d_keys ? c->d_keys_alt : c->d_keys);   // the free ping-pong half
    long long* E = c->d_mdp;   // matched flags, then their exclusive scan (H + 1 entries)
    k_plan_match<<<blocks_for(H, 256), 256, 0, c->s_main>>>(c->pool, sorted, B, c->d_ctr, c->aux_w, c->d_aff_seg,
                                                            c->d_old_row, dpos, E, (long long)H);
    SCOUT_LAUNCH(c, "k_plan_match");
    SCOUT_CU(c, cudaMemsetAsync(E + H, 0, sizeof(long long), c->s_main));
    SCOUT_RC(scan_i64(c, (int64_t*)E, H + 1, nullptr));
    k_plan_place<<<blocks_for(H, 256), 256, 0, c->s_main>>>(c->pool, c->row, sorted, B, c->d_ctr, c->aux_w,
                                                            c->d_aff_seg, c->d_old_row, c->d_aff_len,
                                                            dest, dpos, E, c->tiered);
    SCOUT_LAUNCH(c, "k_plan_place");
    SCOUT_RC(scan_i64(c, c->d_small_off, Amax + 1, nullptr));
    // the row merges loop over their work lists: a grid of at most four blocks per SM
    const int64_t groups = std::min<int64_t>(c->nnz, Amax * (int64_t)SMALL_LEN) / UNIT + 1;
    const int res4 = 4 * c->sm_count;
    k_merge_small<<<std::min(blocks_for(groups * WARP, MERGE_THREADS), res4), MERGE_THREADS, 0, c->s_main>>>(
        c->pool, sorted, B, c->d_ctr, c->d_aff_seg, c->d_old_row, c->d_aff_len, dest, c->d_aff_small,
        c->d_small_off);
    k_merge_long_inplace<<<(unsigned)std::min<int64_t>(std::max<int64_t>(1, Amax), 8 * (int64_t)c->sm_count),
                           LIP_THREADS, 0, c->s_main>>>(c->pool, c->d_ctr, c->d_aff_long, c->d_old_row);
    k_merge_slices<<<std::min(blocks_for(std::min<int64_t>(c->cap_slices, c->nnz / SLICE + Amax + 1024) * WARP,
                                         MS_THREADS),
                              res4),
                     MS_THREADS,
                     0, c->s_main>>>(c->pool, (long long)c->pool_cap, sorted, B, c->d_ctr, c->d_aff_seg,
                                     c->d_old_row, c->d_aff_len, dest, E, dpos, c->d_slices, c->cap_slices,
                                     c->tiered);
    SCOUT_LAUNCH(c, "merge");
    c->nlaunch += 6;
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
    // Room for several batches of rewritten rows between compactions: a compaction copies every
    // live row whatever the garbage, so the larger the pool, the rarer they are. HBM is
    // plentiful (the pool and its compaction spare at eight times a 128 M-entry graph are
    // 8.6 GB); a budget that cannot hold that falls back to four, then two times the graph.
    const int64_t mult[3] = {8, 4, 2};
    for (int i = 0; i < 3; i++) {
        c->pool_cap = mult[i] * nnz + (i < 2 ? (1 << 26) : (1 << 22));
        if ((uint64_t)c->pool_cap * 4 * 2 + c->held <= c->budget) break;
    }
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
    // Contiguous rows, exact nnz and tail (a tiered load lays its rows out contiguously).
    if (!c->tiered) SCOUT_RC(graph_compact(c, std::max<int64_t>(c->pool_cap - c->tail, 1 << 22)));
    c->sealed = true;
    return SCOUT_OK;
}

int scout_graph_load_csr(scout_ctx* c, int64_t n, const int64_t* off, const int32_t* adj) {
    if (!c || !off || n < 1) return c ? c->fail(SCOUT_E_INVALID, "bad CSR") : SCOUT_E_INVALID;
    int64_t nnz = off[n];
    if (off[0] != 0 || nnz < 0 || (nnz > 0 && !adj)) return c->fail(SCOUT_E_INVALID, "bad CSR offsets");
    for (int64_t v = 0; v < n; v++)
        if (off[v + 1] < off[v]) return c->fail(SCOUT_E_INVALID, "CSR offsets must be monotone");
    // A budget that cannot hold the smallest single-tier store (row table, two pools of
    // 2 nnz + 4M entries, about 160 B of per-vertex state) gets the tiered store.
    const uint64_t single = (uint64_t)(16 * n + 160 * n) + 2ull * 4ull * (uint64_t)(2 * nnz + (1 << 22));
    if (c->held + single > c->budget) return scout_graph_load_tiered(c, n, off, adj, 0);
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

// Tiered load: the highest-degree rows (up to half the HBM pool, the rest of it left for rows
// the batches rewrite) are copied to HBM; every other row goes to a mapped page-locked host
// pool that the kernels read in place. Rows are sorted here, on the host.
int scout_graph_load_tiered(scout_ctx* c, int64_t n, const int64_t* off, const int32_t* adj, int64_t hbm_entries) {
    if (!c || !off || n < 1 || n >= INT32_MAX) return c ? c->fail(SCOUT_E_INVALID, "bad CSR") : SCOUT_E_INVALID;
    if (c->reserved) return c->fail(SCOUT_E_STATE, "graph already reserved");
    const int64_t nnz = off[n];
    if (off[0] != 0 || nnz < 0 || (nnz > 0 && !adj)) return c->fail(SCOUT_E_INVALID, "bad CSR offsets");
    for (int64_t v = 0; v < n; v++)
        if (off[v + 1] < off[v] || off[v + 1] - off[v] > INT32_MAX) return c->fail(SCOUT_E_INVALID, "CSR offsets must be monotone");
    cudaSetDevice(c->device);
    if (hbm_entries <= 0) {
        // what the budget leaves after the row table and about 160 B of per-vertex state, for
        // two HBM pools (the pool and its compaction target)
        const int64_t fixed = (int64_t)c->held + 16 * n + 160 * n;
        hbm_entries = std::max<int64_t>(1 << 20, ((int64_t)c->budget - fixed) / 8);
    }
    c->n = n;
    SCOUT_RC(dev_alloc(c, (void**)&c->row, (size_t)n * sizeof(Row), "row table"));
    c->pool_cap = hbm_entries;
    SCOUT_RC(dev_alloc(c, (void**)&c->pool, (size_t)c->pool_cap * sizeof(int32_t), "element pool"));
    // after a host compaction the pool holds at most the live graph, and one batch adds at
    // most a rewrite of every row it touches: 2 nnz (plus slack for insertions)
    c->host_cap = 2 * nnz + (1 << 22);
    {
        void* hp = nullptr;
        cudaError_t e = cudaHostAlloc(&hp, (size_t)c->host_cap * 4, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) { cudaGetLastError(); return c->fail(SCOUT_E_CAPACITY, std::string("host pool: ") + cudaGetErrorString(e)); }
        void* dp = nullptr;
        SCOUT_CU(c, cudaHostGetDevicePointer(&dp, hp, 0));
        if (dp != hp) return c->fail(SCOUT_E_NODEV, "tiered store needs unified addressing of page-locked memory");
        c->host_pool = (int32_t*)hp;
    }
    c->tiered = true;
    // placement: hot rows by descending degree while they fit half the HBM pool
    std::vector<int32_t> order(n);
    for (int64_t v = 0; v < n; v++) order[v] = (int32_t)v;
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        const int64_t da = off[a + 1] - off[a], db = off[b + 1] - off[b];
        return da != db ? da > db : a < b;
    });
    std::vector<Row> rows(n);
    std::vector<char> hot(n, 0);
    int64_t hbm_used = 0;
    for (int64_t i = 0; i < n; i++) {
        const int32_t v = order[i];
        const int64_t d = off[v + 1] - off[v];
        if (hbm_used + d > hbm_entries / 2) break;
        rows[v] = Row{hbm_used, (int)d, (int)d};
        hot[v] = 1;
        hbm_used += d;
    }
    const long long host_rel = elem_delta(c->host_pool, c->pool);
    int64_t host_used = 0;
    std::vector<int64_t> hpos(n, -1);
    for (int64_t v = 0; v < n; v++) {
        if (hot[v]) continue;
        const int64_t d = off[v + 1] - off[v];
        hpos[v] = host_used;
        rows[v] = Row{host_rel + host_used, (int)d, (int)d};
        host_used += d;
    }
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < n; v++) {
        if (hpos[v] < 0) continue;
        int32_t* dst = c->host_pool + hpos[v];
        const int64_t d = off[v + 1] - off[v];
        std::memcpy(dst, adj + off[v], (size_t)d * 4);
        if (!std::is_sorted(dst, dst + d)) std::sort(dst, dst + d);
    }
    // hot rows: gathered in HBM order into the pinned slabs, sorted, copied on two streams
    const int64_t SLAB = 1 << 24;
    SCOUT_RC(ensure_slabs(c, SLAB, 1024));
    int s = 0;
    int64_t i = 0, pos = 0;
    while (pos < hbm_used) {
        SCOUT_CU(c, cudaEventSynchronize(c->ev_copy[s]));
        int32_t* slab = (int32_t*)c->h_slab[s];
        const int64_t p0 = pos;
        while (i < n && hot[order[i]]) {
            const int32_t v = order[i];
            const int64_t d = off[v + 1] - off[v];
            if (pos - p0 + d > SLAB) {
                if (pos == p0) return c->fail(SCOUT_E_CAPACITY, "a row is longer than the staging slab");
                break;
            }
            int32_t* dst = slab + (pos - p0);
            std::memcpy(dst, adj + off[v], (size_t)d * 4);
            if (!std::is_sorted(dst, dst + d)) std::sort(dst, dst + d);
            pos += d;
            i++;
        }
        SCOUT_CU(c, cudaMemcpyAsync(c->pool + p0, slab, (size_t)(pos - p0) * 4, cudaMemcpyHostToDevice, c->s_copy[s]));
        SCOUT_CU(c, cudaEventRecord(c->ev_copy[s], c->s_copy[s]));
        s ^= 1;
    }
    SCOUT_CU(c, cudaMemcpy(c->row, rows.data(), (size_t)n * sizeof(Row), cudaMemcpyHostToDevice));
    c->tail = hbm_used;
    c->host_tail = host_used;
    c->nnz = nnz;
    c->reserved = true;
    c->sealed = false;
    return scout_graph_seal(c);
}

int scout_graph_tier_info(scout_ctx* c, int64_t* hbm_cap, int64_t* hbm_used, int64_t* host_cap, int64_t* host_used,
                          int64_t* evictions, int64_t* host_batches) {
    if (!c) return SCOUT_E_INVALID;
    if (host_batches) *host_batches = c->host_batches;
    if (hbm_cap) *hbm_cap = c->pool_cap;
    if (hbm_used) *hbm_used = c->tail;
    if (host_cap) *host_cap = c->tiered ? c->host_cap : 0;
    if (host_used) *host_used = c->tiered ? c->host_tail : 0;
    if (evictions) *evictions = c->evicted_entries;
    return SCOUT_OK;
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
    SCOUT_RC(gather_finish(c, nullptr, nullptr, nullptr));
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
    k_copy_rows<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + total + COPY_UNITS - 1) / COPY_UNITS,
                                                                    32 * c->sm_count)),
                  COPY_THREADS, 0, c->s_main>>>(c->row, c->pool, tmp, d_off, (int32_t)n, (long long)total);
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
    SCOUT_RC(gather_finish(c, nullptr, nullptr, nullptr));
    return graph_compact(c, std::max<int64_t>(c->nnz, 1 << 22), true);
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
