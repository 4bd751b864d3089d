// cc_dev.cuh -- device code of the cc repair kernel (k_cc): its parameters, helpers and
// body, shared by cc.cu (the kernel and its host launcher) and union.cu (the one persistent
// kernel that runs several problems' repairs of a round).
#pragma once

#include "ctx.cuh"

namespace scout {

constexpr int CC_THREADS = 256;
constexpr int CC_HCAP = 8192;     // shared hash-set slots per side
constexpr int CC_FCAP = 4096;     // frontier capacity
constexpr int CC_MAX_BOUND = 4000;
constexpr int CC_BIG = 4096;      // rows longer than this are scanned by a whole block in P3
constexpr size_t CC_SMEM = (size_t)(2 * CC_HCAP + 3 * CC_FCAP) * sizeof(int32_t);

struct CcParams {
    DGraph g;
    int32_t* label;
    const unsigned long long* hkeys;
    int B;
    int32_t* uf;        // union-find over labels (identity at rest)
    int32_t* cnt;       // splits per class (zero at rest)
    int32_t* dirty;     // == epoch: class recomputed this batch
    int32_t* remf;      // == epoch: class remainder needs its new minimum
    int32_t* newmin;    // remainder minimum per class (INT32_MAX at rest)
    int32_t* vp;        // vertex union-find for recomputes
    int32_t* firstw;    // first surviving split endpoint per class (-1 at rest)
    int32_t* hard;      // deletions left to the block searches (half-edit indices)
    int hard_cap;
    int32_t* hcnt;      // deletions left to search, per class (zero at rest)
    int search_limit;   // above this many per class, the class is recomputed instead
    int32_t* merged;    // labels hooked this batch (n)
    unsigned long long* rec;   // split records: (class << 32 | min), (offset << 32 | size)
    int64_t rec_cap;
    int32_t* side;      // split vertex buffer
    int64_t side_cap;
    int32_t* touched;
    int32_t* st_touch;
    int32_t* st_side;   // == epoch: vertex is in a split side this batch
    int32_t epoch;
    int bound;
    int variant;        // 0 incremental, 1 recompute every class, 2 recompute every class a
                        // deletion that no common neighbour settles touches (search limit 0)
    const int* mode_dev;  // when set, the variant is read here (decided on the device by the scheduler)
    DevCounters* ctr;
    GridBar* bar;
};

__device__ __forceinline__ int32_t uf_find(int32_t* uf, int32_t x) {
    int32_t p = ld_volatile(uf + x);
    while (p != x) {
        int32_t gp = ld_volatile(uf + p);
        if (gp != p) atomicCAS(uf + x, p, gp);   // path halving
        x = p;
        p = gp;
    }
    return x;
}

// Lower root wins; returns the root that was hooked (or -1 when already joined).
__device__ __forceinline__ int32_t uf_union(int32_t* uf, int32_t a, int32_t b) {
    while (true) {
        a = uf_find(uf, a);
        b = uf_find(uf, b);
        if (a == b) return -1;
        int32_t hi = a > b ? a : b, lo = a > b ? b : a;
        if (atomicCAS(uf + hi, hi, lo) == hi) return hi;
    }
}

__device__ __forceinline__ void cc_touch(const CcParams& p, bool pred, int32_t v) {
    bool nt = false;
    if (pred) nt = atomicExch(&p.st_touch[v], p.epoch) != p.epoch;
    int at = warp_append(nt, &p.ctr->changed);
    if (nt) p.touched[at] = v;
}

// ---- shared-memory hash set (open addressing, -1 empty) ------------------------------------
__device__ __forceinline__ unsigned hslot(int32_t x) { return ((unsigned)x * 2654435761u) & (CC_HCAP - 1); }
__device__ __forceinline__ bool hs_has(const int32_t* hs, int32_t x) {
    unsigned h = hslot(x);
    for (int i = 0; i < CC_HCAP; i++) {
        int32_t s = hs[h];
        if (s == x) return true;
        if (s == -1) return false;
        h = (h + 1) & (CC_HCAP - 1);
    }
    return false;
}
// 1 inserted, 0 present, -1 full
__device__ __forceinline__ int hs_insert(int32_t* hs, int32_t x) {
    unsigned h = hslot(x);
    for (int i = 0; i < CC_HCAP; i++) {
        int32_t prev = atomicCAS(hs + h, -1, x);
        if (prev == -1) return 1;
        if (prev == x) return 0;
        h = (h + 1) & (CC_HCAP - 1);
    }
    return -1;
}

// Bounded bidirectional search of one deletion (u, v) by the whole block.
// Returns 0 connected, 1 split (side written to p.side), 2 inconclusive.
static __device__ int cc_search(const CcParams& p, int32_t u, int32_t v, int32_t cls, long long& bytes, bool record) {
    extern __shared__ int32_t sm[];
    int32_t* hs[2] = {sm, sm + CC_HCAP};
    int32_t* fr[2] = {sm + 2 * CC_HCAP, sm + 2 * CC_HCAP + CC_FCAP};
    int32_t* nf = sm + 2 * CC_HCAP + 2 * CC_FCAP;
    __shared__ int s_fn[2], s_nn, s_touched, s_met, s_over;
    const int t = threadIdx.x;
    // common-neighbour check: both endpoints adjacent to some w (settles hub-hub deletions)
    if (t == 0) s_met = 0;
    __syncthreads();
    {
        Row ru = p.g.row[u], rv = p.g.row[v];
        if (rv.len < ru.len) { Row tmp = ru; ru = rv; rv = tmp; }
        const int32_t* a = p.g.pool + ru.start;
        const int32_t* b = p.g.pool + rv.start;
        for (int i = t; i < ru.len && !ld_volatile(&s_met); i += CC_THREADS) {
            long long k = lower_bound_i32(b, rv.len, a[i]);
            if (k < rv.len && b[k] == a[i]) s_met = 1;
        }
        bytes += 4LL * ((ru.len + CC_THREADS - 1 - t) / CC_THREADS) * 8;
    }
    __syncthreads();
    if (s_met) return 0;
    for (int i = t; i < 2 * CC_HCAP; i += CC_THREADS) sm[i] = -1;
    __syncthreads();
    __shared__ long long s_vol[2], s_nvol;
    if (t == 0) {
        hs_insert(hs[0], u);
        hs_insert(hs[1], v);
        fr[0][0] = u;
        fr[1][0] = v;
        s_fn[0] = 1;
        s_fn[1] = 1;
        s_vol[0] = p.g.row[u].len;
        s_vol[1] = p.g.row[v].len;
        s_touched = 2;
        s_met = 0;
        s_over = 0;
    }
    __syncthreads();
    while (s_fn[0] > 0 && s_fn[1] > 0) {
        // Expand the side whose frontier has fewer adjacency entries to scan (the reference
        // compares vertex counts; the volume keeps a hub endpoint from being expanded while
        // its partner's side is still small, which is what overruns the bound).
        const int sd = s_vol[0] <= s_vol[1] ? 0 : 1;
        const int fn = s_fn[sd];
        if (t == 0) { s_nn = 0; s_nvol = 0; }
        __syncthreads();
        // warp per frontier vertex, lanes over its row
        for (int i = t / WARP; i < fn; i += CC_THREADS / WARP) {
            int32_t x = fr[sd][i];
            Row r = p.g.row[x];
            const int32_t* rw = p.g.pool + r.start;
            for (int b0 = 0; b0 < r.len; b0 += WARP) {
                if (ld_volatile(&s_met) || ld_volatile(&s_over)) break;
                int k = b0 + (int)lane_id();
                if (k < r.len) {
                    int32_t y = rw[k];
                    // meet: y already reached by the other side, or adjacent to its endpoint
                    // (a binary search that stands in for the other side's first level)
                    if (hs_has(hs[sd ^ 1], y) || dg_adjacent(p.g, y, sd == 0 ? v : u)) {
                        s_met = 1;
                    } else {
                        int ins = hs_insert(hs[sd], y);
                        if (ins < 0) s_over = 1;
                        else if (ins == 1) {
                            int tt = atomicAdd(&s_touched, 1) + 1;
                            int at = atomicAdd(&s_nn, 1);
                            if (tt > p.bound || at >= CC_FCAP) s_over = 1;
                            else {
                                nf[at] = y;
                                atomicAdd((unsigned long long*)&s_nvol, (unsigned long long)p.g.row[y].len);
                            }
                        }
                    }
                    bytes += 8;
                }
            }
        }
        __syncthreads();
        if (s_met) return 0;
        if (s_over) return 2;
        const int nn = s_nn;
        for (int i = t; i < nn; i += CC_THREADS) fr[sd][i] = nf[i];
        __syncthreads();
        if (t == 0) { s_fn[sd] = nn; s_vol[sd] = s_nvol; }
        __syncthreads();
    }
    // one side is exhausted: its visited set is a whole component
    const int ex = s_fn[0] == 0 ? 0 : 1;
    __shared__ int s_size, s_min;
    __shared__ long long s_off;
    if (t == 0) { s_size = 0; s_min = INT32_MAX; }
    __syncthreads();
    for (int i = t; i < CC_HCAP; i += CC_THREADS) {
        int32_t x = hs[ex][i];
        if (x >= 0) { atomicAdd(&s_size, 1); atomicMin(&s_min, x); }
    }
    __syncthreads();
    if (!record) return 1;
    if (t == 0) {
        s_off = atomicAdd((unsigned long long*)&p.ctr->aux64[0], (unsigned long long)s_size);
        int rid = atomicAdd(&p.ctr->list_count[2], 1);
        if (s_off + s_size > p.side_cap || 3LL * rid + 2 >= p.rec_cap) {
            // no room to record the side: recompute the class
            if (atomicExch(p.dirty + cls, p.epoch) != p.epoch) atomicAdd(&p.ctr->recomputes, 1);
            s_off = -1;
        } else {
            p.rec[3 * rid] = ((unsigned long long)(uint32_t)cls << 32) | (uint32_t)s_min;
            p.rec[3 * rid + 1] = ((unsigned long long)s_off << 32) | (uint32_t)s_size;
            p.rec[3 * rid + 2] = (uint32_t)(ex == 0 ? v : u);   // the endpoint left in the remainder
            atomicAdd(p.cnt + cls, 1);
        }
    }
    __syncthreads();
    if (s_off >= 0) {
        __shared__ int s_w;
        if (t == 0) s_w = 0;
        __syncthreads();
        for (int i = t; i < CC_HCAP; i += CC_THREADS) {
            int32_t x = hs[ex][i];
            if (x >= 0) p.side[s_off + atomicAdd(&s_w, 1)] = x;
        }
        __syncthreads();
    }
    return 1;
}

__device__ __forceinline__ void cc_body(const CcParams& p) {
    const int W = gwarp_count(), wid = gwarp_id();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t n = p.g.n;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    const int nh = ld_volatile(&p.ctr->n_half);
    long long bytes = 0;
    __shared__ int s_task;
    const int variant = p.mode_dev ? *p.mode_dev : p.variant;
    const int full = variant == 1;
    const int limit = variant == 2 ? 0 : p.search_limit;

    phase_mark(&p.ctr->phase_ns[0]);
    if (!full) {
        // ---- P0: unions of inserted edges ---------------------------------------------------
        for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += T) {
            int64_t k = b + lane_id();
            int32_t hooked = -1;
            if (k < nh) {
                unsigned long long key = p.hkeys[k];
                int op = (int)((key >> p.B) & 1ull);
                int32_t x = (int32_t)(key >> (p.B + 1));
                int32_t y = (int32_t)(key & ((1ull << p.B) - 1));
                if (op == 0 && x < y) hooked = uf_union(p.uf, ld_volatile(p.label + x), ld_volatile(p.label + y));
            }
            int at = warp_append(hooked >= 0, &p.ctr->list_count[1]);
            if (hooked >= 0) p.merged[at] = hooked;
        }
        if (!grid_sync(p.bar, 30)) return;
        const int nm = ld_volatile(&p.ctr->list_count[1]);
        if (leader) p.ctr->ins_eff = nm;   // every successful hook merged two classes
        if (nm > 0) {
            for (int64_t b = tid - (tid & (WARP - 1)); b < n; b += T) {
                int64_t v = b + lane_id();
                bool ch = false;
                if (v < n) {
                    int32_t l = p.label[v];
                    if (ld_volatile(p.uf + l) != l) { p.label[v] = uf_find(p.uf, l); ch = true; }
                }
                cc_touch(p, ch, (int32_t)v);
            }
            if (tid == 0) bytes += 8LL * n;
            if (!grid_sync(p.bar, 31)) return;
            for (int64_t i = tid; i < nm; i += T) {
                int32_t l = p.merged[i];
                p.uf[l] = l;
            }
        }
        phase_mark(&p.ctr->phase_ns[1]);
        // ---- P1a: one warp per deletion: a common neighbour settles it (most deletions in a
        // dense component, hub-hub ones included); the rest go to the hard list -------------
        for (int64_t b = (int64_t)wid * WARP; b < nh; b += (int64_t)W * WARP) {
            // 32 half-edits per warp iteration, then each candidate checked by the whole warp
            int64_t k0 = b + lane_id();
            bool cand = false;
            int32_t x = 0, y = 0;
            if (k0 < nh) {
                unsigned long long key = p.hkeys[k0];
                x = (int32_t)(key >> (p.B + 1));
                y = (int32_t)(key & ((1ull << p.B) - 1));
                cand = ((key >> p.B) & 1ull) == 1ull && x < y && ld_volatile(p.label + x) == ld_volatile(p.label + y);
            }
            unsigned cm = __ballot_sync(0xffffffffu, cand);
            while (cm) {
                const int l = __ffs(cm) - 1;
                cm &= cm - 1;
                const int32_t cx = __shfl_sync(0xffffffffu, x, l), cy = __shfl_sync(0xffffffffu, y, l);
                Row ra = p.g.row[cx], rb = p.g.row[cy];
                if (rb.len < ra.len) { Row tmp = ra; ra = rb; rb = tmp; }
                const int32_t* av = p.g.pool + ra.start;
                const int32_t* bv = p.g.pool + rb.start;
                bool met = false;
                for (int i0 = 0; i0 < ra.len && !met; i0 += WARP) {
                    int i = i0 + (int)lane_id();
                    bool h = false;
                    if (i < ra.len) {
                        long long kk = lower_bound_i32(bv, rb.len, av[i]);
                        h = kk < rb.len && bv[kk] == av[i];
                    }
                    met = __any_sync(0xffffffffu, h);
                    if (i < ra.len) bytes += 4LL * 8;
                }
                if (lane_id() == 0) {
                    atomicAdd(&p.ctr->searches, 1);
                    if (!met) {
                        // a class with more deletions to search than the limit is recomputed
                        // instead; every unsettled deletion is listed so P1b can reset hcnt
                        const int32_t cls = ld_volatile(p.label + cx);
                        const int before = atomicAdd(p.hcnt + cls, 1);
                        const int at = atomicAdd(&p.ctr->list_count[0], 1);
                        if (at < p.hard_cap) p.hard[at] = (int32_t)(b + l);
                        const bool over = at >= p.hard_cap || (limit >= 0 && before >= limit);
                        if (over && atomicExch(p.dirty + cls, p.epoch) != p.epoch)
                            atomicAdd(&p.ctr->recomputes, 1);
                    }
                }
            }
        }
        if (!grid_sync(p.bar, 39)) return;
        phase_mark(&p.ctr->phase_ns[2]);
        // ---- P1b: one block per remaining deletion: the bounded bidirectional search ---------
        const int nhard = min(ld_volatile(&p.ctr->list_count[0]), p.hard_cap);
        if (leader) p.ctr->noop = ld_volatile(&p.ctr->searches) - nhard;   // settled by a common neighbour
        while (true) {
            if (threadIdx.x == 0) {
                int j = atomicAdd(&p.ctr->list_count[3], 1);
                if (j < nhard) {
                    // the class of a listed deletion is fixed since P0; a dirty one is not searched
                    unsigned long long key = p.hkeys[p.hard[j]];
                    int32_t cls = ld_volatile(p.label + (int32_t)(key >> (p.B + 1)));
                    p.hcnt[cls] = 0;
                    if (ld_volatile(p.dirty + cls) == p.epoch) j = -1;
                }
                s_task = j;
            }
            __syncthreads();
            const int j = s_task;
            __syncthreads();
            if (j >= nhard) break;
            if (j < 0) continue;
            unsigned long long key = p.hkeys[p.hard[j]];
            int32_t x = (int32_t)(key >> (p.B + 1));
            int32_t y = (int32_t)(key & ((1ull << p.B) - 1));
            int32_t cls = ld_volatile(p.label + x);
            int res = cc_search(p, x, y, cls, bytes, true);
            if (threadIdx.x == 0 && res == 2 && atomicExch(p.dirty + cls, p.epoch) != p.epoch)
                atomicAdd(&p.ctr->recomputes, 1);
            __syncthreads();
        }
        if (!grid_sync(p.bar, 32)) return;
        phase_mark(&p.ctr->phase_ns[3]);
        // ---- P2: relabel the split sides -------------------------------------------------------
        // A class whose deletions all ended connected or split is exact once its remainder R
        // (the class minus the split sides) is known to be connected. Every component of R
        // holds the surviving endpoint of some split deletion, so R is connected iff those
        // endpoints are: trivially with one split; with several, each endpoint is searched
        // against the class's first one. Any other outcome marks the class dirty.
        const int nrec = min(ld_volatile(&p.ctr->list_count[2]), (int)(p.rec_cap / 3));
        for (int i = (int)tid; i < nrec; i += (int)T) {
            int32_t cls = (int32_t)(p.rec[3 * i] >> 32);
            if (ld_volatile(p.dirty + cls) != p.epoch && ld_volatile(p.cnt + cls) >= 2)
                atomicCAS(p.firstw + cls, -1, (int32_t)p.rec[3 * i + 2]);
        }
        if (!grid_sync(p.bar, 40)) return;
        while (true) {
            if (threadIdx.x == 0) s_task = atomicAdd(&p.ctr->q_count[0], 1);
            __syncthreads();
            const int i = s_task;
            __syncthreads();
            if (i >= nrec) break;
            int32_t cls = (int32_t)(p.rec[3 * i] >> 32);
            if (ld_volatile(p.cnt + cls) < 2 || ld_volatile(p.dirty + cls) == p.epoch) continue;
            int32_t w = (int32_t)p.rec[3 * i + 2], f = ld_volatile(p.firstw + cls);
            if (w == f || f < 0) continue;
            int res = cc_search(p, w, f, cls, bytes, false);
            if (threadIdx.x == 0 && res != 0 && atomicExch(p.dirty + cls, p.epoch) != p.epoch)
                atomicAdd(&p.ctr->recomputes, 1);
            __syncthreads();
        }
        if (!grid_sync(p.bar, 41)) return;
        for (int i = wid; i < nrec; i += W) {
            unsigned long long r0 = p.rec[3 * i], r1 = p.rec[3 * i + 1];
            int32_t cls = (int32_t)(r0 >> 32), mn = (int32_t)(r0 & 0xffffffffu);
            long long off = (long long)(r1 >> 32);
            int size = (int)(r1 & 0xffffffffu);
            if (ld_volatile(p.dirty + cls) == p.epoch) continue;
            if (lane_id() == 0) {
                atomicAdd(&p.ctr->splits, 1);
                if (mn == cls) p.remf[cls] = p.epoch;
            }
            for (int b0 = 0; b0 < size; b0 += WARP) {
                int j = b0 + (int)lane_id();
                bool ok = j < size;
                int32_t w = ok ? p.side[off + j] : 0;
                bool ch = false;
                if (ok) {
                    p.st_side[w] = p.epoch;
                    if (p.label[w] != mn) { p.label[w] = mn; ch = true; }
                }
                cc_touch(p, ch, w);
            }
        }
        if (!grid_sync(p.bar, 33)) return;
        // remainder of a class whose minimum left with the split side: its own minimum
        for (int64_t v = tid; v < n; v += T) {
            int32_t l = p.label[v];
            if (ld_volatile(p.remf + l) == p.epoch && ld_volatile(p.st_side + v) != p.epoch &&
                ld_volatile(p.dirty + l) != p.epoch)
                atomicMin(p.newmin + l, (int32_t)v);
        }
        if (tid == 0) bytes += 12LL * n;
        if (!grid_sync(p.bar, 34)) return;
        for (int64_t b = tid - (tid & (WARP - 1)); b < n; b += T) {
            int64_t v = b + lane_id();
            bool ch = false;
            if (v < n) {
                int32_t l = p.label[v];
                if (ld_volatile(p.remf + l) == p.epoch && ld_volatile(p.st_side + v) != p.epoch &&
                    ld_volatile(p.dirty + l) != p.epoch) {
                    int32_t m = ld_volatile(p.newmin + l);
                    if (m != l) { p.label[v] = m; ch = true; }
                }
            }
            cc_touch(p, ch, (int32_t)v);
        }
        if (!grid_sync(p.bar, 35)) return;
        // restore per-class scratch of split classes
        for (int i = (int)tid; i < nrec; i += (int)T) {
            int32_t cls = (int32_t)(p.rec[3 * i] >> 32);
            p.cnt[cls] = 0;
            p.newmin[cls] = INT32_MAX;
            p.firstw[cls] = -1;
        }
    } else {
        // every class is recomputed; the final pass lists only the labels that change
        if (leader) p.ctr->recomputes = 1;
    }
    // ---- P3: exact recompute of dirty classes (every class when full) ------------------------
    if (!grid_sync(p.bar, 38)) return;
    if (!full && ld_volatile(&p.ctr->recomputes) == 0) {
        goto done;
    }
    for (int64_t v = tid; v < n; v += T) {
        bool d = full || ld_volatile(p.dirty + p.label[v]) == p.epoch;
        p.vp[v] = d ? (int32_t)v : -1;
    }
    if (!grid_sync(p.bar, 36)) return;
    {
        // Afforest (Sutton, Ben-Nun, Barak, IPDPS 2018): link every dirty vertex to its first
        // two neighbours, compress, estimate the dominant root by sampling, then only vertices
        // outside that root scan the rest of their rows (an edge between the dominant tree
        // and another vertex is linked from the other vertex's row). An edge leaving a dirty
        // class means the uploaded labels did not describe the components of the graph: it is
        // flagged (SCOUT_E_STATE) instead of followed.
        constexpr int AF_FIRST = 2;
        for (int r = 0; r < AF_FIRST; r++) {
            for (int64_t v = tid; v < n; v += T) {
                if (ld_volatile(p.vp + v) < 0) continue;
                Row rr = p.g.row[v];
                if (r < rr.len) {
                    int32_t w = p.g.pool[rr.start + r];
                    if (ld_volatile(p.vp + w) < 0) atomicExch(&p.ctr->pad, 1);
                    else uf_union(p.vp, (int32_t)v, w);
                }
            }
            if (!grid_sync(p.bar, 42 + r)) return;
        }
        for (int64_t v = tid; v < n; v += T)
            if (ld_volatile(p.vp + v) >= 0) p.vp[v] = uf_find(p.vp, (int32_t)v);
        if (tid == 0) bytes += 24LL * n;
        if (!grid_sync(p.bar, 44)) return;
        if (blockIdx.x == 0) {   // mode of the roots of up to 1024 sampled dirty vertices
            __shared__ int32_t s_key[2048];
            __shared__ int s_cnt[2048];
            __shared__ unsigned long long s_best;
            for (int i = threadIdx.x; i < 2048; i += CC_THREADS) { s_key[i] = -1; s_cnt[i] = 0; }
            if (threadIdx.x == 0) s_best = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < 4096; i += CC_THREADS) {
                int64_t v = (int64_t)(((unsigned long long)i * 2654435761ull) % (unsigned long long)n);
                int32_t r = ld_volatile(p.vp + v);
                if (r < 0) continue;
                unsigned h = ((unsigned)r * 2654435761u) & 2047u;
                for (int pr = 0; pr < 2048; pr++) {
                    int32_t prev = atomicCAS(&s_key[h], -1, r);
                    if (prev == -1 || prev == r) { atomicAdd(&s_cnt[h], 1); break; }
                    h = (h + 1) & 2047u;
                }
            }
            __syncthreads();
            for (int i = threadIdx.x; i < 2048; i += CC_THREADS)
                if (s_cnt[i] > 0)
                    atomicMax(&s_best, ((unsigned long long)s_cnt[i] << 32) | (uint32_t)s_key[i]);
            __syncthreads();
            if (threadIdx.x == 0) p.ctr->aux64[1] = s_best ? (long long)(uint32_t)(s_best & 0xffffffffu) : -1;
        }
        if (!grid_sync(p.bar, 45)) return;
        const int32_t gr = (int32_t)ld_volatile(&p.ctr->aux64[1]);
        // compact lists of the vertices outside the dominant root (short rows / long rows)
        if (leader) { p.ctr->q_count[1] = 0; p.ctr->q_count[2] = 0; }
        if (!grid_sync(p.bar, 46)) return;
        for (int64_t b = tid - (tid & (WARP - 1)); b < n; b += T) {
            int64_t v = b + lane_id();
            bool sm_ = false, bg = false;
            if (v < n) {
                int32_t pv = ld_volatile(p.vp + v);
                if (pv >= 0 && pv != gr) {
                    int len = p.g.row[v].len;
                    if (len > AF_FIRST) { bg = len > CC_BIG; sm_ = !bg; }
                }
            }
            int a = warp_append(sm_, &p.ctr->q_count[1]);
            if (sm_) p.merged[a] = (int32_t)v;
            int c2 = warp_append(bg, &p.ctr->q_count[2]);
            if (bg) p.side[c2] = (int32_t)v;
        }
        if (tid == 0) bytes += 8LL * n;
        if (!grid_sync(p.bar, 47)) return;
        const int nsmall = ld_volatile(&p.ctr->q_count[1]), nbig = ld_volatile(&p.ctr->q_count[2]);
        for (int i = wid; i < nsmall; i += W) {   // rows up to CC_BIG: one warp each
            const int32_t v = p.merged[i];
            Row r = p.g.row[v];
            const int32_t* rw = p.g.pool + r.start;
            for (int b0 = AF_FIRST; b0 < r.len; b0 += WARP) {
                int k = b0 + (int)lane_id();
                if (k < r.len) {
                    int32_t w = rw[k];
                    if (ld_volatile(p.vp + w) < 0) atomicExch(&p.ctr->pad, 1);
                    else uf_union(p.vp, v, w);
                }
            }
            if (lane_id() == 0) bytes += 8LL * r.len;
        }
        for (int i = blockIdx.x; i < nbig; i += gridDim.x) {   // longer rows: one block each
            const int32_t v = p.side[i];
            Row r = p.g.row[v];
            const int32_t* rw = p.g.pool + r.start;
            for (long long k = AF_FIRST + threadIdx.x; k < r.len; k += CC_THREADS) {
                int32_t w = rw[k];
                if (ld_volatile(p.vp + w) < 0) atomicExch(&p.ctr->pad, 1);
                else uf_union(p.vp, v, w);
            }
            if (threadIdx.x == 0) bytes += 8LL * r.len;
        }
    }
    if (!grid_sync(p.bar, 37)) return;
    for (int64_t b = tid - (tid & (WARP - 1)); b < n; b += T) {
        int64_t v = b + lane_id();
        bool ch = false;
        if (v < n && ld_volatile(p.vp + v) >= 0) {
            int32_t root = uf_find(p.vp, (int32_t)v);
            if (p.label[v] != root) { p.label[v] = root; ch = true; }
        }
        cc_touch(p, ch, (int32_t)v);
    }
    if (tid == 0) bytes += 16LL * n;
done:
    phase_mark(&p.ctr->phase_ns[4]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
    if (leader) p.ctr->affected = full ? (int)n : p.ctr->changed;
}
// host: the kernel parameters of the context's current batch (cc.cu)
int cc_params(scout_ctx* c, const scout_sched* sched, int variant, const int* mode_dev, CcParams* out);

}  // namespace scout
