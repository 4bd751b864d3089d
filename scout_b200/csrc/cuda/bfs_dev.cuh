// bfs_dev.cuh -- device code of the bfs repair kernel (k_bfs): its parameters, helpers and
// body, shared by bfs.cu (the kernel and its host launcher) and union.cu (the one persistent
// kernel that runs several problems' repairs of a round).
#pragma once

#include "ctx.cuh"

namespace scout {

constexpr int BFS_THREADS = 256;
constexpr int PSCAN = 4;   // row entries per lane and step in the seed scan

struct BfsParams {
    DGraph g;
    int32_t* level;
    int32_t source;
    const unsigned long long* hkeys;
    int B;
    unsigned long long* q[3];
    int64_t qcap;
    int32_t* inval;
    int32_t* touched;
    int32_t* st_inval;
    int32_t* st_touch;
    uint32_t* st_q;
    int32_t* found;     // == tag: a chunk of a long candidate found a valid parent this round
    int32_t epoch;
    uint32_t qtag0;
    DevCounters* ctr;
    GridBar* bar;
    int mode;             // 0 incremental, 1 top-down traversal, 2 direction-optimizing traversal
    const int* mode_dev;  // when set, the mode is read here (written on the device by the scheduler)
    int32_t* lv_new;      // n: levels of a full traversal before they are diffed into `level`
    long long nnz_pre;    // directed entries before this batch (the batch's delta is in ctr)
    int chunk, chunk_log2;    // row entries per queue item (a power of two, 256 .. 8192)
    const int32_t* sources;   // when nsrc > 0: every listed vertex is a level-0 root (a union of
    int nsrc;                 // disjoint graphs, one source each); else `source` alone
    int max_share;            // most warps that share one queue item (lanes_per_vertex / 32)
};

__device__ __forceinline__ int32_t ld_level(const int32_t* p) { return ld_volatile(p); }

// Warp-cooperative push (all 32 lanes call): lanes with `pred` push vertex y into queue qn
// once per round (tag), split into chunk-sized items; first touches of the batch are
// appended to the touched list.
__device__ __forceinline__ void push_vertex(const BfsParams& p, bool pred, int32_t y, int qi, uint32_t tag,
                                            bool chunked, bool touch) {
    bool first = false;
    if (pred) first = atomicExch(&p.st_q[y], tag) != tag;
    if (touch) {
        bool nt = false;
        if (pred) nt = atomicExch(&p.st_touch[y], p.epoch) != p.epoch;
        int ti = warp_append(nt, &p.ctr->changed);
        if (nt) p.touched[ti] = y;
    }
    int nit = 0;
    if (first) {
        if (chunked) {
            int len = p.g.row[y].len;
            nit = max(1, (len + p.chunk - 1) >> p.chunk_log2);   // an empty row still gets its item
        } else {
            nit = 1;
        }
    }
    int incl = warp_incl_scan_i(nit);
    int tot = __shfl_sync(0xffffffffu, incl, WARP - 1);
    if (tot == 0) return;
    int base = 0;
    if (lane_id() == WARP - 1) base = atomicAdd(&p.ctr->q_count[qi], tot);
    base = __shfl_sync(0xffffffffu, base, WARP - 1);
    long long start = (long long)base + incl - nit;
    for (int k = 0; k < nit; k++) {
        long long pos = start + k;
        if (pos < p.qcap) p.q[qi][pos] = ((unsigned long long)k << 32) | (uint32_t)y;
        else atomicExch(&p.ctr->overflow, 1);
    }
}

// push_vertex (chunked, no touch list) of two vertices per lane at once: the dedupe atomics and
// row-length loads of both are in flight together, and one atomicAdd reserves both's items.
__device__ __forceinline__ void push_vertex2(const BfsParams& p, bool pa, int32_t ya, bool pb, int32_t yb, int qi,
                                             uint32_t tag) {
    bool fa = false, fb = false;
    if (pa) fa = atomicExch(&p.st_q[ya], tag) != tag;
    if (pb) fb = atomicExch(&p.st_q[yb], tag) != tag;   // ya == yb: only the first push counts
    int na = 0, nb = 0;
    if (fa) na = max(1, (p.g.row[ya].len + p.chunk - 1) >> p.chunk_log2);
    if (fb) nb = max(1, (p.g.row[yb].len + p.chunk - 1) >> p.chunk_log2);
    const int nit = na + nb;
    const int incl = warp_incl_scan_i(nit);
    const int tot = __shfl_sync(0xffffffffu, incl, WARP - 1);
    if (tot == 0) return;
    int base = 0;
    if (lane_id() == WARP - 1) base = atomicAdd(&p.ctr->q_count[qi], tot);
    base = __shfl_sync(0xffffffffu, base, WARP - 1);
    const long long start = (long long)base + incl - nit;
    for (int k = 0; k < nit; k++) {
        const long long pos = start + k;
        const int32_t v = k < na ? ya : yb;
        const int kk = k < na ? k : k - na;
        if (pos < p.qcap) p.q[qi][pos] = ((unsigned long long)kk << 32) | (uint32_t)v;
        else atomicExch(&p.ctr->overflow, 1);
    }
}

__device__ __forceinline__ int qcount(const BfsParams& p, int qi) {
    int c = ld_volatile(&p.ctr->q_count[qi]);
    return (long long)c > p.qcap ? (int)p.qcap : c;
}

// Work split of a round over `cnt` queue items (each at most `chunk` row entries) among the
// grid's W warps. With at least W / 2 items, a warp takes per = ceil(cnt / W) consecutive
// items per pass (one per lane, at most 32) and expands their entries together. With fewer
// items, g warps share every item (g a power of two with g * cnt <= W and at least 32 entries
// per share), each expanding its own contiguous 1/g of the item's entries: a round of a few
// hub chunks then spreads over the whole grid instead of over a handful of warps.
__device__ __forceinline__ int items_per_warp(int cnt, int W) {
    const int per = (int)(((long long)cnt + W - 1) / W);
    return per < 1 ? 1 : (per > WARP ? WARP : per);
}
__device__ __forceinline__ int warps_per_item(int cnt, int W, int chunk, int max_share) {
    int g = 1;
    while ((long long)g * 2 * cnt <= W && g * 2 * WARP <= chunk && g * 2 <= max_share) g *= 2;
    return g;
}

// Expansion of one item share [b, e) of a row segment starting at s, 32 entries at a time;
// every lane calls it (the pushes are warp-collective). Levels only decrease during the relax
// rounds, so a neighbour whose level (read without an atomic, possibly stale and then larger)
// is already at most lv + 1 needs no atomicMin.
__device__ __forceinline__ void relax_share(const BfsParams& p, long long s, int b, int e, int lv, int nxt,
                                            uint32_t tag) {
    const unsigned cand = (unsigned)(lv + 1);
    for (int k0 = b; k0 < e; k0 += WARP) {
        const int k = k0 + (int)lane_id();
        bool dec = false;
        int32_t y = 0;
        if (k < e) {
            y = p.g.pool[s + k];
            if ((unsigned)ld_level(p.level + y) > cand) dec = atomicMin((unsigned*)(p.level + y), cand) > cand;
        }
        push_vertex(p, dec, y, nxt, tag, true, true);
    }
}

// One relax round over queue `cur` into `nxt` (warp-level load-balanced expansion).
static __device__ void relax_round(const BfsParams& p, int cur, int nxt, uint32_t tag, long long& bytes) {
    const int cnt = qcount(p, cur);
    const int W = gwarp_count();
    if ((long long)cnt * 2 <= W) {
        const int g = warps_per_item(cnt, W, p.chunk, p.max_share);
        for (long long wv = gwarp_id(); wv < (long long)cnt * g; wv += W) {
            const int item = (int)(wv / g), part = (int)(wv % g);
            const unsigned long long it = p.q[cur][item];
            const int32_t v = (int32_t)(it & 0xffffffffu);
            const int chunk = (int)(it >> 32);
            const Row r = p.g.row[v];
            const int lv = ld_level(p.level + v);
            const int len = lv < 0 ? 0 : max(0, min(p.chunk, r.len - (chunk << p.chunk_log2)));
            const int b = (int)((long long)len * part / g), e = (int)((long long)len * (part + 1) / g);
            if (lane_id() == 0) bytes += 8LL * (e - b) + (part == 0 ? 24 : 0);
            relax_share(p, r.start + ((long long)chunk << p.chunk_log2), b, e, lv, nxt, tag);
        }
        return;
    }
    const int per = items_per_warp(cnt, W);
    for (long long gbase = (long long)gwarp_id() * per; gbase < cnt; gbase += (long long)W * per) {
        long long idx = gbase + lane_id();
        bool valid = (int)lane_id() < per && idx < cnt;
        unsigned long long item = valid ? p.q[cur][idx] : 0ull;
        int32_t v = (int32_t)(item & 0xffffffffu);
        int chunk = (int)(item >> 32);
        long long s = 0;
        int len = 0, lv = -1;
        if (valid) {
            Row r = p.g.row[v];
            s = r.start + ((long long)chunk << p.chunk_log2);
            len = min(p.chunk, r.len - (chunk << p.chunk_log2));
            if (len < 0) len = 0;
            lv = ld_level(p.level + v);
            if (lv < 0) len = 0;
        }
        int incl = warp_incl_scan_i(len);
        int total = __shfl_sync(0xffffffffu, incl, WARP - 1);
        int excl = incl - len;
        bytes += (long long)len * 8 + (valid ? 24 : 0);
        for (int e0 = 0; e0 < total; e0 += WARP) {
            int e = e0 + (int)lane_id();
            int lo = 0, hi = WARP - 1;
#pragma unroll
            for (int it = 0; it < 5; it++) {
                int mid = (lo + hi + 1) >> 1;
                int em = __shfl_sync(0xffffffffu, excl, mid);
                if (em <= e) lo = mid; else hi = mid - 1;
            }
            long long so = __shfl_sync(0xffffffffu, s, lo);
            int eo = __shfl_sync(0xffffffffu, excl, lo);
            int lo_lv = __shfl_sync(0xffffffffu, lv, lo);
            bool dec = false;
            int32_t y = 0;
            if (e < total) {
                y = p.g.pool[so + (e - eo)];
                unsigned cand = (unsigned)(lo_lv + 1);
                if ((unsigned)ld_level(p.level + y) > cand) dec = atomicMin((unsigned*)(p.level + y), cand) > cand;
            }
            push_vertex(p, dec, y, nxt, tag, true, true);
        }
    }
}

// ---- full traversals (modes 1 and 2) ---------------------------------------------------------
// Frontier bookkeeping rotates over three slots like the queues: list_count[s] holds the
// vertices and aux64[s] the adjacency entries of the frontier in q[s].
constexpr int DO_ALPHA = 14;   // top-down -> bottom-up once frontier entries > unexplored / 14
constexpr int DO_BETA = 24;    // bottom-up -> top-down once the frontier has < n / 24 vertices

// Warp-cooperative push of newly levelled vertices (each pushed by exactly one lane, so no
// dedupe tag is needed): chunk items into q[qi], vertex and entry counts into slot qi.
__device__ __forceinline__ void push_new(const BfsParams& p, bool pred, int32_t y, int len, int qi) {
    int nit = pred ? max(1, (len + p.chunk - 1) >> p.chunk_log2) : 0;
    int incl = warp_incl_scan_i(nit);
    int tot = __shfl_sync(0xffffffffu, incl, WARP - 1);
    if (tot == 0) return;
    long long deg = pred ? len : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) deg += __shfl_xor_sync(0xffffffffu, deg, o);
    const int nv = __popc(__ballot_sync(0xffffffffu, pred));
    int base = 0;
    if (lane_id() == WARP - 1) {
        base = atomicAdd(&p.ctr->q_count[qi], tot);
        atomicAdd(&p.ctr->list_count[qi], nv);
        atomicAdd((unsigned long long*)&p.ctr->aux64[qi], (unsigned long long)deg);
    }
    base = __shfl_sync(0xffffffffu, base, WARP - 1);
    long long start = (long long)base + incl - nit;
    for (int k = 0; k < nit; k++) {
        long long pos = start + k;
        if (pos < p.qcap) p.q[qi][pos] = ((unsigned long long)k << 32) | (uint32_t)y;
        else atomicExch(&p.ctr->overflow, 1);
    }
}

// Top-down step: every entry of every frontier item claims its unlevelled neighbours (the
// same work split as the relax rounds).
__device__ __forceinline__ void td_share(const BfsParams& p, int32_t* lv, long long s, int b, int e, int d, int nxt) {
    for (int k0 = b; k0 < e; k0 += WARP) {
        const int k = k0 + (int)lane_id();
        bool got = false;
        int32_t y = 0;
        int ylen = 0;
        if (k < e) {
            y = p.g.pool[s + k];
            if (ld_volatile(lv + y) < 0) got = atomicCAS(lv + y, -1, d + 1) == -1;
            if (got) ylen = p.g.row[y].len;
        }
        push_new(p, got, y, ylen, nxt);
    }
}

static __device__ void td_step(const BfsParams& p, int32_t* lv, int cur, int nxt, int d, long long& bytes) {
    const int cnt = qcount(p, cur);
    const int W = gwarp_count();
    if ((long long)cnt * 2 <= W) {
        const int g = warps_per_item(cnt, W, p.chunk, p.max_share);
        for (long long wv = gwarp_id(); wv < (long long)cnt * g; wv += W) {
            const int item = (int)(wv / g), part = (int)(wv % g);
            const unsigned long long it = p.q[cur][item];
            const int32_t v = (int32_t)(it & 0xffffffffu);
            const int chunk = (int)(it >> 32);
            const Row r = p.g.row[v];
            const int len = max(0, min(p.chunk, r.len - (chunk << p.chunk_log2)));
            const int b = (int)((long long)len * part / g), e = (int)((long long)len * (part + 1) / g);
            if (lane_id() == 0) bytes += 8LL * (e - b) + (part == 0 ? 24 : 0);
            td_share(p, lv, r.start + ((long long)chunk << p.chunk_log2), b, e, d, nxt);
        }
        return;
    }
    const int per = items_per_warp(cnt, W);
    for (long long gbase = (long long)gwarp_id() * per; gbase < cnt; gbase += (long long)W * per) {
        long long idx = gbase + lane_id();
        bool valid = (int)lane_id() < per && idx < cnt;
        unsigned long long item = valid ? p.q[cur][idx] : 0ull;
        int32_t v = (int32_t)(item & 0xffffffffu);
        int chunk = (int)(item >> 32);
        long long s = 0;
        int len = 0;
        if (valid) {
            Row r = p.g.row[v];
            s = r.start + ((long long)chunk << p.chunk_log2);
            len = max(0, min(p.chunk, r.len - (chunk << p.chunk_log2)));
        }
        int incl = warp_incl_scan_i(len);
        int total = __shfl_sync(0xffffffffu, incl, WARP - 1);
        int excl = incl - len;
        bytes += (long long)len * 8 + (valid ? 24 : 0);
        for (int e0 = 0; e0 < total; e0 += WARP) {
            int e = e0 + (int)lane_id();
            int lo = 0, hi = WARP - 1;
#pragma unroll
            for (int it = 0; it < 5; it++) {
                int mid = (lo + hi + 1) >> 1;
                int em = __shfl_sync(0xffffffffu, excl, mid);
                if (em <= e) lo = mid; else hi = mid - 1;
            }
            long long so = __shfl_sync(0xffffffffu, s, lo);
            int eo = __shfl_sync(0xffffffffu, excl, lo);
            bool got = false;
            int32_t y = 0;
            int ylen = 0;
            if (e < total) {
                y = p.g.pool[so + (e - eo)];
                if (ld_volatile(lv + y) < 0) got = atomicCAS(lv + y, -1, d + 1) == -1;
                if (got) ylen = p.g.row[y].len;
            }
            push_new(p, got, y, ylen, nxt);
        }
    }
}

// Bottom-up step: every unlevelled vertex looks for a neighbour on level d and stops at the
// first one. Short rows are scanned by their own lane, longer ones by the whole warp.
static __device__ void bu_step(const BfsParams& p, int32_t* lv, int nxt, int d, long long& bytes) {
    const int64_t n = p.g.n;
    const int W = gwarp_count();
    for (int64_t base = (int64_t)gwarp_id() * WARP; base < n; base += (int64_t)W * WARP) {
        const int64_t v = base + lane_id();
        bool un = v < n && ld_volatile(lv + v) < 0;
        Row r{0, 0, 0};
        if (un) r = p.g.row[v];
        bool found = false;
        const bool big = un && r.len > WARP;
        long long scanned = un ? 4 + 16 : (v < n ? 4 : 0);
        if (un && !big) {
            for (int k = 0; k < r.len; k++) {
                scanned += 8;
                if (ld_volatile(lv + p.g.pool[r.start + k]) == d) { found = true; break; }
            }
        }
        unsigned bigm = __ballot_sync(0xffffffffu, big);
        while (bigm) {
            const int j = __ffs(bigm) - 1;
            bigm &= bigm - 1;
            const long long js = __shfl_sync(0xffffffffu, r.start, j);
            const int jl = __shfl_sync(0xffffffffu, r.len, j);
            bool hit = false;
            for (int b0 = 0; b0 < jl && !hit; b0 += WARP) {
                int k = b0 + (int)lane_id();
                bool ok = k < jl && ld_volatile(lv + p.g.pool[js + k]) == d;
                if (k < jl) scanned += 8;
                hit = __any_sync(0xffffffffu, ok);
            }
            if ((int)lane_id() == j) found = hit;
        }
        if (found) lv[v] = d + 1;
        bytes += scanned;
        push_new(p, found, (int32_t)v, found ? r.len : 0, nxt);
    }
}

// Full traversal into lv_new, then the diff into level. Returns false when a barrier failed.
static __device__ bool full_bfs(const BfsParams& p, int mode, long long& bytes, int& rounds) {
    int32_t* lv = p.lv_new;
    const int64_t n = p.g.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    for (int64_t v = tid; v < n; v += T) lv[v] = -1;
    if (tid == 0) bytes += 4LL * n;
    if (!grid_sync(p.bar, 22)) return false;
    if (leader) {
        const int ns = p.nsrc > 0 ? p.nsrc : 1;
        int items = 0;
        long long deg = 0;
        for (int i = 0; i < ns; i++) {
            const int32_t s = p.nsrc > 0 ? p.sources[i] : p.source;
            lv[s] = 0;
            const int len = p.g.row[s].len;
            const int nit = max(1, (len + p.chunk - 1) >> p.chunk_log2);
            for (int k = 0; k < nit && items + k < p.qcap; k++)
                p.q[0][items + k] = ((unsigned long long)k << 32) | (uint32_t)s;
            items += nit;
            deg += len;
        }
        if (items > p.qcap) { p.ctr->overflow = 1; items = (int)p.qcap; }
        p.ctr->q_count[0] = items;
        p.ctr->list_count[0] = ns;
        p.ctr->aux64[0] = deg;
        p.ctr->q_count[1] = p.ctr->list_count[1] = 0;
        p.ctr->q_count[2] = p.ctr->list_count[2] = 0;
        p.ctr->aux64[1] = p.ctr->aux64[2] = 0;
    }
    if (!grid_sync(p.bar, 20)) return false;
    const long long total = p.nnz_pre + ld_volatile(&p.ctr->nnz_delta);
    long long visited = 0;
    bool bottom_up = false;
    int cur = 0;
    for (int d = 0;; d++) {
        const int nf = ld_volatile(&p.ctr->list_count[cur]);
        if (nf == 0) break;
        const long long mf = ld_volatile(&p.ctr->aux64[cur]);
        visited += mf;
        if (mode == 2) {
            if (!bottom_up && mf > (total - visited) / DO_ALPHA) bottom_up = true;
            else if (bottom_up && (long long)nf * DO_BETA < n) bottom_up = false;
        }
        const int nxt = (cur + 1) % 3, zer = (cur + 2) % 3;
        if (leader) { p.ctr->q_count[zer] = 0; p.ctr->list_count[zer] = 0; p.ctr->aux64[zer] = 0; }
        if (bottom_up) bu_step(p, lv, nxt, d, bytes);
        else td_step(p, lv, cur, nxt, d, bytes);
        rounds++;
        if (!grid_sync(p.bar, 21)) return false;
        cur = nxt;
    }
    // diff: store and list the levels that changed
    for (int64_t b = tid - (tid & (WARP - 1)); b < n; b += T) {
        const int64_t v = b + lane_id();
        bool ch = false;
        int32_t nv = 0;
        if (v < n) {
            nv = lv[v];
            ch = nv != p.level[v];
            if (ch) p.level[v] = nv;
        }
        int ti = warp_append(ch, &p.ctr->changed);
        if (ch) p.touched[ti] = (int32_t)v;
    }
    if (tid == 0) bytes += 12LL * n;
    return true;
}

// At least four blocks per SM: the register budget this grants (64 per thread) holds the
// kernel without spills (the unconstrained build spilled to local memory at 40 registers).
__device__ __forceinline__ void bfs_body(const BfsParams& p) {
    const int W = gwarp_count();
    const int wid = gwarp_id();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    long long bytes = 0;
    int rounds = 0;
    uint32_t tag = p.qtag0;
    int cur = 0;
    phase_mark(&p.ctr->phase_ns[0]);

    const int mode = p.mode_dev ? *p.mode_dev : p.mode;
    if (mode != 0) {
        if (!full_bfs(p, mode, bytes, rounds)) return;
        phase_mark(&p.ctr->phase_ns[3]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
        if (leader) {
            p.ctr->rounds = rounds;
            p.ctr->affected = p.g.n;
            p.ctr->recomputes = 1;
        }
        return;
    }
    {
        // ---- A: invalidation -------------------------------------------------------------
        // Candidates are queued as chunk-sized items of their rows. A single-chunk candidate
        // is settled by one warp (parent check, invalidation, children pushed). A longer one
        // is checked chunk by chunk (any chunk with a valid parent marks found = tag); after
        // a barrier its first item decides, and after another every chunk of an invalidated
        // candidate pushes its children, so a hub's row is spread over many warps.
        const int nh = ld_volatile(&p.ctr->n_half);
        tag++;
        // two half-edits per thread and step (k and k + T): their loads overlap, and both
        // candidates go out in one warp-collective push
        for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += 2 * T) {
            bool cand[2] = {false, false};
            int32_t y[2] = {0, 0};
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int64_t k = b + h * T + lane_id();
                if (k < nh) {
                    const unsigned long long key = p.hkeys[k];
                    const int op = (int)((key >> p.B) & 1ull);
                    const int32_t x = (int32_t)(key >> (p.B + 1));
                    y[h] = (int32_t)(key & ((1ull << p.B) - 1));
                    if (op == 1) {
                        const int lx = ld_level(p.level + x), ly = ld_level(p.level + y[h]);
                        cand[h] = lx >= 0 && ly == lx + 1;
                    }
                }
            }
            const int nc = __popc(__ballot_sync(0xffffffffu, cand[0])) + __popc(__ballot_sync(0xffffffffu, cand[1]));
            if (lane_id() == 0 && nc) atomicAdd(&p.ctr->del_eff, nc);   // tree-edge deletions
            push_vertex2(p, cand[0], y[0], cand[1], y[1], 0, tag);
        }
        if (!grid_sync(p.bar, 2)) return;
        cur = 0;
        while (true) {
            const int cnt = qcount(p, cur);
            if (cnt == 0) break;
            const int nxt = (cur + 1) % 3, zer = (cur + 2) % 3;
            if (leader) p.ctr->q_count[zer] = 0;
            tag++;
            // Software pipeline over the warp's candidates: the queue item two candidates ahead,
            // and the row, level and invalidation mark of the next one, are loaded while the
            // current one is checked. None of them changes during this pass: levels are fixed in
            // this phase, and a single-chunk candidate is queued once per round and invalidated
            // only by its own warp (a long one's mark is set after the barrier below).
            unsigned long long it_n = wid < cnt ? p.q[cur][wid] : 0ull;
            Row r_n{0, 0, 0};
            int lc_n = 0, si_n = 0;
            if (wid < cnt) {
                const int32_t cn = (int32_t)(it_n & 0xffffffffu);
                r_n = p.g.row[cn];
                lc_n = ld_level(p.level + cn);
                si_n = ld_volatile(p.st_inval + cn);
            }
            unsigned long long it_nn = wid + W < cnt ? p.q[cur][wid + W] : 0ull;
            for (int i = wid; i < cnt; i += W) {
                const unsigned long long item = it_n;
                const Row r = r_n;
                const int lc = lc_n;
                const int si = si_n;
                it_n = it_nn;
                if (i + W < cnt) {   // the next candidate's item arrived during this one's wait
                    const int32_t cn = (int32_t)(it_n & 0xffffffffu);
                    r_n = p.g.row[cn];
                    lc_n = ld_level(p.level + cn);
                    si_n = ld_volatile(p.st_inval + cn);
                }
                it_nn = (long long)i + 2 * W < cnt ? p.q[cur][i + 2 * W] : 0ull;
                const int32_t c = (int32_t)(item & 0xffffffffu);
                const int chunk = (int)(item >> 32);
                const bool big = r.len > p.chunk;
                if (c == p.source || lc <= 0 || si == p.epoch) {
                    if (big && lane_id() == 0) p.found[c] = (int32_t)tag;   // nothing to decide
                    continue;
                }
                const long long c0 = ((long long)chunk << p.chunk_log2);
                const int clen = (int)min((long long)p.chunk, (long long)r.len - c0);
                const int32_t* rw = p.g.pool + r.start + c0;
                bool found = false;
                // 32 entries per step: most candidates keep a parent early in the row, and wider
                // steps (measured with four entries per lane) only add random level reads
                for (int b0 = 0; b0 < clen && !found; b0 += WARP) {
                    const int k = b0 + (int)lane_id();
                    bool ok = false;
                    if (k < clen) {
                        const int32_t w = rw[k];
                        ok = ld_level(p.level + w) == lc - 1 && ld_volatile(p.st_inval + w) != p.epoch;
                        bytes += 8;
                    }
                    found = __any_sync(0xffffffffu, ok);
                }
                if (big) {
                    if (lane_id() == 0) {
                        if (found) p.found[c] = (int32_t)tag;
                        if (chunk == 0) p.ctr->list_count[2] = 1;   // a long candidate this round
                    }
                    continue;
                }
                if (found) continue;
                if (lane_id() == 0) {
                    p.st_inval[c] = p.epoch;
                    int at = atomicAdd(&p.ctr->list_count[0], 1);
                    p.inval[at] = c;
                }
                __syncwarp();
                for (int b0 = 0; b0 < clen; b0 += WARP) {
                    int k = b0 + (int)lane_id();
                    bool ch = false;
                    int32_t w = 0;
                    if (k < clen) {
                        w = rw[k];
                        ch = ld_level(p.level + w) == lc + 1 && ld_volatile(p.st_inval + w) != p.epoch;
                    }
                    push_vertex(p, ch, w, nxt, tag, true, false);
                }
                if (lane_id() == 0) bytes += 8LL * clen + 24;
            }
            if (!grid_sync(p.bar, 3)) return;
            if (ld_volatile(&p.ctr->list_count[2])) {
                // long candidates: decide on the first item, then push children from every chunk
                for (int64_t b = tid - (tid & (WARP - 1)); b < cnt; b += T) {
                    const int64_t i = b + lane_id();
                    bool nt = false;
                    int32_t c = 0;
                    if (i < cnt) {
                        const unsigned long long item = p.q[cur][i];
                        c = (int32_t)(item & 0xffffffffu);
                        if ((item >> 32) == 0 && p.g.row[c].len > p.chunk && ld_volatile(p.found + c) != (int32_t)tag)
                            nt = atomicExch(&p.st_inval[c], p.epoch) != p.epoch;
                    }
                    int at = warp_append(nt, &p.ctr->list_count[0]);
                    if (nt) p.inval[at] = c;
                }
                if (!grid_sync(p.bar, 8)) return;
                if (leader) p.ctr->list_count[2] = 0;
                for (int i = wid; i < cnt; i += W) {
                    const unsigned long long item = p.q[cur][i];
                    const int32_t c = (int32_t)(item & 0xffffffffu);
                    const Row r = p.g.row[c];
                    if (r.len <= p.chunk || ld_volatile(p.found + c) == (int32_t)tag ||
                        ld_volatile(p.st_inval + c) != p.epoch)
                        continue;
                    const int lc = ld_level(p.level + c);
                    const long long c0 = ((long long)(item >> 32) << p.chunk_log2);
                    const int clen = (int)min((long long)p.chunk, (long long)r.len - c0);
                    const int32_t* rw = p.g.pool + r.start + c0;
                    for (int b0 = 0; b0 < clen; b0 += WARP) {
                        int k = b0 + (int)lane_id();
                        bool ch = false;
                        int32_t w = 0;
                        if (k < clen) {
                            w = rw[k];
                            ch = ld_level(p.level + w) == lc + 1 && ld_volatile(p.st_inval + w) != p.epoch;
                        }
                        push_vertex(p, ch, w, nxt, tag, true, false);
                    }
                    if (lane_id() == 0) bytes += 8LL * clen;
                }
                if (!grid_sync(p.bar, 9)) return;
            }
            rounds++;
            cur = nxt;
        }
        phase_mark(&p.ctr->phase_ns[1]);
        // ---- B: reset and seed --------------------------------------------------------------
        // Every invalidated vertex restarts at +inf and queues its row's chunks in q[2]; each
        // chunk then offers (min level of its valid neighbours) + 1. Inserted edges seed their
        // endpoints. Both push into q[0], where the relax rounds start.
        if (leader) { p.ctr->q_count[0] = 0; p.ctr->q_count[1] = 0; p.ctr->q_count[2] = 0; }
        if (!grid_sync(p.bar, 4)) return;
        const int ninv = ld_volatile(&p.ctr->list_count[0]);
        tag++;
        for (int64_t b = tid - (tid & (WARP - 1)); b < ninv; b += T) {
            int64_t i = b + lane_id();
            bool ok = i < ninv;
            int32_t c = ok ? p.inval[i] : 0;
            bool nt = false;
            if (ok) {
                nt = atomicExch(&p.st_touch[c], p.epoch) != p.epoch;
                p.level[c] = -1;
            }
            int ti = warp_append(nt, &p.ctr->changed);
            if (nt) p.touched[ti] = c;
            push_vertex(p, ok, c, 2, tag, true, false);
        }
        if (!grid_sync(p.bar, 5)) return;
        tag++;
        // boundary seeds: warp per chunk of an invalidated vertex's row
        const int nseed = qcount(p, 2);
        for (int i = wid; i < nseed; i += W) {
            const unsigned long long item = p.q[2][i];
            const int32_t c = (int32_t)(item & 0xffffffffu);
            const Row r = p.g.row[c];
            const long long c0 = ((long long)(item >> 32) << p.chunk_log2);
            const int clen = (int)min((long long)p.chunk, (long long)r.len - c0);
            const int32_t* rw = p.g.pool + r.start + c0;
            unsigned best = 0xffffffffu;
            for (int b0 = 0; b0 < clen; b0 += PSCAN * WARP) {   // both loads of PSCAN entries in flight
                int32_t w[PSCAN];
#pragma unroll
                for (int u = 0; u < PSCAN; u++) {
                    const int k = b0 + u * WARP + (int)lane_id();
                    w[u] = k < clen ? rw[k] : -1;
                }
#pragma unroll
                for (int u = 0; u < PSCAN; u++) {
                    if (w[u] < 0) continue;
                    const int32_t si = ld_volatile(p.st_inval + w[u]);
                    const int lw = ld_level(p.level + w[u]);
                    if (si != p.epoch && lw >= 0) best = min(best, (unsigned)lw);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (lane_id() == 0) bytes += 8LL * max(clen, 0) + 24;
            bool dec = false;
            if (lane_id() == 0 && best != 0xffffffffu) {
                unsigned cand = best + 1;
                unsigned old = atomicMin((unsigned*)(p.level + c), cand);
                dec = old > cand;
            }
            push_vertex(p, dec, c, 0, tag, true, false);
        }
        // insertion seeds: thread per half-edit
        for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += T) {
            int64_t k = b + lane_id();
            bool dec = false;
            int32_t y = 0;
            if (k < nh) {
                unsigned long long key = p.hkeys[k];
                int op = (int)((key >> p.B) & 1ull);
                int32_t x = (int32_t)(key >> (p.B + 1));
                y = (int32_t)(key & ((1ull << p.B) - 1));
                if (op == 0) {
                    int lx = ld_level(p.level + x);
                    if (lx >= 0) {
                        unsigned cand = (unsigned)lx + 1;
                        unsigned old = atomicMin((unsigned*)(p.level + y), cand);
                        dec = old > cand;
                    }
                }
            }
            const unsigned md = __ballot_sync(0xffffffffu, dec);   // insertions that lowered a level
            if (lane_id() == 0 && md) atomicAdd(&p.ctr->ins_eff, __popc(md));
            push_vertex(p, dec, y, 0, tag, true, true);
        }
        if (!grid_sync(p.bar, 6)) return;
        cur = 0;
    }
    phase_mark(&p.ctr->phase_ns[2]);
    // ---- C: relax rounds -------------------------------------------------------------------
    while (true) {
        const int cnt = qcount(p, cur);
        if (cnt == 0) break;
        const int nxt = (cur + 1) % 3, zer = (cur + 2) % 3;
        if (leader) p.ctr->q_count[zer] = 0;
        tag++;
        relax_round(p, cur, nxt, tag, bytes);
        rounds++;
        if (!grid_sync(p.bar, 7)) return;
        cur = nxt;
    }
    phase_mark(&p.ctr->phase_ns[3]);
    // ---- counters ----------------------------------------------------------------------------
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
    if (leader) {
        p.ctr->rounds = rounds;
        p.ctr->affected = p.ctr->changed;
    }
}
// host: the kernel parameters of the context's current batch (bfs.cu)
int bfs_params(scout_ctx* c, int mode, const int* mode_dev, BfsParams* out);

}  // namespace scout
