// mis_dev.cuh -- device code of the mis repair kernel (k_mis): its parameters, helpers and
// body, shared by mis.cu (the kernel and its host launcher) and union.cu (the one persistent
// kernel that runs several problems' repairs of a round).
#pragma once

#include "ctx.cuh"

namespace scout {

constexpr int MIS_THREADS = 256;

struct MisParams {
    DGraph g;
    int32_t* mis;
    const unsigned long long* hkeys;
    int B;
    int32_t* list[2];      // undecided candidates (n each)
    int32_t* removed;      // dropped vertices (n)
    int32_t* touched;
    int32_t* st_cand;      // == epoch: candidate this batch
    int32_t* st_done;      // == epoch: decided this batch
    int32_t* st_touch;
    int32_t epoch;
    DevCounters* ctr;
    GridBar* bar;
};

__device__ __forceinline__ void mis_touch(const MisParams& p, bool pred, int32_t v) {
    bool nt = false;
    if (pred) nt = atomicExch(&p.st_touch[v], p.epoch) != p.epoch;
    int at = warp_append(nt, &p.ctr->changed);
    if (nt) p.touched[at] = v;
}

// Warp-cooperative: lanes with pred add v to the candidate list once per batch.
__device__ __forceinline__ void mis_candidate(const MisParams& p, bool pred, int32_t v) {
    bool first = false;
    if (pred) first = atomicExch(&p.st_cand[v], p.epoch) != p.epoch;
    int at = warp_append(first, &p.ctr->list_count[0]);
    if (first) p.list[0][at] = v;
}

__device__ __forceinline__ void mis_body(const MisParams& p) {
    const int W = gwarp_count(), wid = gwarp_id();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    const int nh = ld_volatile(&p.ctr->n_half);
    long long bytes = 0;
    int rounds = 0;

    // ---- 1: conflicts of inserted edges, evaluated on the pre-batch set ----------------
    for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += T) {
        int64_t k = b + lane_id();
        bool drop = false;
        int32_t r = 0;
        if (k < nh) {
            unsigned long long key = p.hkeys[k];
            int op = (int)((key >> p.B) & 1ull);
            int32_t x = (int32_t)(key >> (p.B + 1));
            int32_t y = (int32_t)(key & ((1ull << p.B) - 1));
            if (op == 0 && x < y && ld_volatile(p.mis + x) && ld_volatile(p.mis + y)) {
                r = y;
                drop = atomicExch(&p.st_done[y], p.epoch) != p.epoch;
                atomicAdd(&p.ctr->conflicts, 1);
            }
        }
        int at = warp_append(drop, &p.ctr->list_count[2]);
        if (drop) p.removed[at] = r;
    }
    if (!grid_sync(p.bar, 20)) return;
    // ---- 2: drop them; candidates = dropped vertices, their neighbours, deletion endpoints ---
    const int nrem = ld_volatile(&p.ctr->list_count[2]);
    for (int64_t b = tid - (tid & (WARP - 1)); b < nrem; b += T) {
        int64_t i = b + lane_id();
        bool ok = i < nrem;
        int32_t r = ok ? p.removed[i] : 0;
        if (ok) p.mis[r] = 0;
        mis_touch(p, ok, r);
    }
    if (!grid_sync(p.bar, 21)) return;
    for (int i = wid; i < nrem; i += W) {
        int32_t r = p.removed[i];
        Row rr = p.g.row[r];
        const int32_t* rw = p.g.pool + rr.start;
        mis_candidate(p, lane_id() == 0, r);
        for (int b0 = 0; b0 < rr.len; b0 += WARP) {
            int k = b0 + (int)lane_id();
            mis_candidate(p, k < rr.len, k < rr.len ? rw[k] : 0);
        }
        if (lane_id() == 0) bytes += 4LL * rr.len + 16;
    }
    for (int64_t b = tid - (tid & (WARP - 1)); b < nh; b += T) {
        int64_t k = b + lane_id();
        bool del = false;
        int32_t x = 0;
        if (k < nh) {
            unsigned long long key = p.hkeys[k];
            del = ((key >> p.B) & 1ull) == 1ull;
            x = (int32_t)(key >> (p.B + 1));
        }
        mis_candidate(p, del, x);
    }
    if (!grid_sync(p.bar, 22)) return;
    if (leader) p.ctr->affected = ld_volatile(&p.ctr->list_count[0]);
    // ---- 3: id-priority rounds --------------------------------------------------------------
    int cur = 0;
    while (true) {
        const int cnt = ld_volatile(&p.ctr->list_count[cur]);
        if (cnt == 0) break;
        const int nxt = cur ^ 1;
        if (leader) p.ctr->list_count[nxt] = 0;
        if (!grid_sync(p.bar, 23)) return;
        // st_done: == epoch marks a vertex dropped in step 1 (still undecided); DONE_IN / DONE_OUT
        // a vertex decided in these rounds. The decision and its value live in one word, so a
        // neighbour read once is either undecided or decided with its final membership (a
        // separate flag read after the set entry could pair a new flag with a stale entry).
        const int32_t DONE_IN = p.epoch + 0x40000000, DONE_OUT = p.epoch + 0x20000000;
        for (int i = wid; i < cnt; i += W) {
            int32_t c = p.list[cur][i];
            Row r = p.g.row[c];
            const int32_t* rw = p.g.pool + r.start;
            const bool was_in = ld_volatile(p.mis + c) != 0;
            bool member_nb = false, lower_undecided = false;
            if (!was_in) {
                for (int b0 = 0; b0 < r.len && !member_nb; b0 += WARP) {
                    int k = b0 + (int)lane_id();
                    bool m = false, l = false;
                    if (k < r.len) {
                        int32_t w = rw[k];
                        const int32_t sd = ld_volatile(p.st_done + w);
                        if (sd == DONE_IN) {
                            m = true;
                        } else if (sd != DONE_OUT) {
                            m = ld_volatile(p.mis + w) != 0;
                            l = w < c && ld_volatile(p.st_cand + w) == p.epoch;
                        }
                    }
                    member_nb = __any_sync(0xffffffffu, m);
                    lower_undecided = lower_undecided || __any_sync(0xffffffffu, l);
                    if (k < r.len) bytes += 8;
                }
            }
            const bool joined = !was_in && !member_nb && !lower_undecided;
            if (lane_id() == 0) {
                if (was_in) {
                    p.st_done[c] = DONE_IN;    // kept
                } else if (member_nb) {
                    p.st_done[c] = DONE_OUT;
                } else if (joined) {
                    p.mis[c] = 1;
                    p.st_done[c] = DONE_IN;
                } else {
                    p.list[nxt][atomicAdd(&p.ctr->list_count[nxt], 1)] = c;   // wait
                }
            }
            mis_touch(p, lane_id() == 0 && joined, c);
        }
        rounds++;
        if (!grid_sync(p.bar, 24)) return;
        cur = nxt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (lane_id() == 0) atomicAdd((unsigned long long*)&p.ctr->hbm_bytes, (unsigned long long)bytes);
    if (leader) p.ctr->rounds = rounds;
}
// host: the kernel parameters of the context's current batch (mis.cu)
int mis_params(scout_ctx* c, MisParams* out);

}  // namespace scout
