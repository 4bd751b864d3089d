// sched.cu -- the learned scheduler of the BFS and CC repairs.
//
// The reference picks its repair strategy with fixed constants: a cascade bound of 200
// touched vertices for BFS (scout_bfs.cu:475-476), a search bound of 5000 or none for CC
// (scout_cc.cu:68-69, 469), and a deferred recompute past them (core/local_repair.h:13-26).
// Here every BFS/CC batch can run one of several exact repair variants (BFS: incremental,
// top-down traversal, direction-optimizing traversal; CC: incremental, recompute of every
// class, recompute of the classes an unsettled deletion touches), all with identical
// results, and the scheduler chooses one on the device, between
// the batch merge and the repair, without a host round trip:
//   k_sched_feat   per-batch features from the merged batch (affected rows, half-edits and
//                  the solution as it stood before the repair)
//   k_sched_infer  the 24-64-64-4 cost model (bf16 parameters, fp32 accumulation) predicts
//                  log2 of each variant's repair time; the cheapest variant (a variant other
//                  than the incremental one only for a predicted gain of about 15%) is written to
//                  ctr->decision, which the persistent repair kernel reads when it starts.
// Without an installed model the decision stays 0 (incremental): the plain engine.
//
// Features (all O(1) in magnitude):
//   0  log2(1 + applied edits) / 24         1  insertion share        2  deletion share
//   3..18  share of affected rows with floor(log2(1 + degree)) = 0..15 (last bin open)
//   19 log2(1 + n) / 32                     20 log2(1 + nnz / n) / 8
//   21 log2(1 + affected rows) / log2(2 + n)
//   22 BFS: share of deleted half-edges x->y with level(y) = level(x) + 1 (tree-edge
//      candidates); CC: share of deleted half-edges whose endpoint y is left with degree <= 2
//   23 log2(1 + previous batch's repair time in microseconds) / 16
// Outputs: 0..2 = log2(1 + repair microseconds) / 4 of variants 0..2; 3 = log2(1 + vertices
// whose value changed) / 24.
#include "ctx.cuh"
#include "mlp.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <vector>

namespace scout {

constexpr int SCHED_BINS = 16;
constexpr float SCHED_MARGIN = 0.05f;

struct FeatParams {
    const int32_t* aff;
    const Row* row;
    const unsigned long long* hkeys;
    int B;
    const int32_t* level;   // BFS levels before the repair, or null
    int problem;
    DevCounters* ctr;
};

__global__ void k_sched_feat(FeatParams p) {
    __shared__ int sh[SCHED_BINS];
    __shared__ int s_hit, s_del;
    if (threadIdx.x < SCHED_BINS) sh[threadIdx.x] = 0;
    if (threadIdx.x == 0) { s_hit = 0; s_del = 0; }
    __syncthreads();
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int na = p.ctr->n_aff, nh = p.ctr->n_half;
    for (int64_t i = tid; i < na; i += T) {
        const int d = p.row[p.aff[i]].len;
        atomicAdd(&sh[min(SCHED_BINS - 1, 31 - __clz(d + 1))], 1);
    }
    int hit = 0, del = 0;
    for (int64_t k = tid; k < nh; k += T) {
        const unsigned long long key = p.hkeys[k];
        if (((key >> p.B) & 1ull) == 0) continue;   // insertion
        const int32_t x = (int32_t)(key >> (p.B + 1));
        const int32_t y = (int32_t)(key & ((1ull << p.B) - 1));
        del++;
        if (p.level) {
            const int lx = p.level[x], ly = p.level[y];
            hit += lx >= 0 && ly == lx + 1;
        } else {
            hit += p.row[y].len <= 2;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        hit += __shfl_xor_sync(0xffffffffu, hit, o);
        del += __shfl_xor_sync(0xffffffffu, del, o);
    }
    if (lane_id() == 0 && (hit | del)) { atomicAdd(&s_hit, hit); atomicAdd(&s_del, del); }
    __syncthreads();
    if (threadIdx.x < SCHED_BINS && sh[threadIdx.x]) atomicAdd(&p.ctr->sched_hist[threadIdx.x], sh[threadIdx.x]);
    if (threadIdx.x == 0 && (s_hit | s_del)) {
        atomicAdd(&p.ctr->sched_del_hit, s_hit);
        atomicAdd(&p.ctr->sched_del, s_del);
    }
}

// One block of 64 threads: features, then the model (thread j owns hidden unit j).
__global__ void __launch_bounds__(64) k_sched_infer(DevCounters* __restrict__ ctr, int64_t n, long long nnz_pre,
                                                    float prev_feature, const __nv_bfloat16* __restrict__ w,
                                                    int nvariants) {
    using namespace mlp;
    __shared__ float f[IN], h1[H], h2[H], y[OUT];
    const int t = threadIdx.x;
    if (t == 0) {
        const int ins = ctr->n_ins, del = ctr->n_del, na = ctr->n_aff;
        const int ed = ins + del;
        const float nnz = (float)(nnz_pre + ctr->nnz_delta);
        f[0] = log2f(1.f + ed) / 24.f;
        f[1] = ed ? (float)ins / ed : 0.f;
        f[2] = ed ? (float)del / ed : 0.f;
        for (int b = 0; b < 16; b++) f[3 + b] = na ? (float)ctr->sched_hist[b] / na : 0.f;
        f[19] = log2f(1.f + (float)n) / 32.f;
        f[20] = log2f(1.f + nnz / fmaxf(1.f, (float)n)) / 8.f;
        f[21] = log2f(1.f + na) / log2f(2.f + (float)n);
        f[22] = ctr->sched_del ? (float)ctr->sched_del_hit / ctr->sched_del : 0.f;
        f[23] = prev_feature;
    }
    __syncthreads();
    if (w) {
        float a = __bfloat162float(w[OFF_B1 + t]);
#pragma unroll
        for (int k = 0; k < IN; k++) a = fmaf(__bfloat162float(w[OFF_W1 + t * IN + k]), f[k], a);
        h1[t] = fmaxf(a, 0.f);
        __syncthreads();
        a = __bfloat162float(w[OFF_B2 + t]);
#pragma unroll 8
        for (int k = 0; k < H; k++) a = fmaf(__bfloat162float(w[OFF_W2 + t * H + k]), h1[k], a);
        h2[t] = fmaxf(a, 0.f);
        __syncthreads();
        if (t < OUT) {
            a = __bfloat162float(w[OFF_B3 + t]);
#pragma unroll 8
            for (int k = 0; k < H; k++) a = fmaf(__bfloat162float(w[OFF_W3 + t * H + k]), h2[k], a);
            y[t] = a;
        }
        __syncthreads();
    }
    if (t < IN) ctr->feat[t] = f[t];
    if (t == 0) {
        int best = 0;
        if (w) {
            // another variant replaces the incremental repair only for a predicted gain of more
            // than SCHED_MARGIN (log2 microseconds / 4: 0.05 is about 15%)
            float by = y[0] - SCHED_MARGIN;
            for (int v = 1; v < nvariants; v++) if (y[v] < by) { best = v; by = y[v]; }
            for (int o = 0; o < OUT; o++) ctr->pred[o] = y[o];
        }
        ctr->decision = best;
        ctr->sched_flags = w ? 3 : 1;
    }
}

int sched_variants(int problem) { return problem == SCOUT_BFS || problem == SCOUT_CC ? 3 : 1; }

int sched_decide(scout_ctx* c, int problem, int64_t m, bool use_model, const int** mode_dev) {
    *mode_dev = nullptr;
    FeatParams fp;
    fp.aff = c->d_aff;
    fp.row = c->row;
    fp.hkeys = c->d_hkeys;
    fp.B = c->key_bits;
    fp.level = problem == SCOUT_BFS ? c->level : nullptr;
    fp.problem = problem;
    fp.ctr = c->d_ctr;
    if (m > 0 && c->d_hkeys) {
        k_sched_feat<<<blocks_for(2 * m, 256, 4 * c->sm_count), 256, 0, c->s_main>>>(fp);
        SCOUT_LAUNCH(c, "k_sched_feat");
        c->nlaunch += 1;
    }
    const __nv_bfloat16* w = use_model ? (const __nv_bfloat16*)c->model[problem] : nullptr;
    const float prev = std::log2(1.0 + 1000.0 * c->prev_repair_ms[problem]) / 16.0;
    k_sched_infer<<<1, 64, 0, c->s_main>>>(c->d_ctr, c->n, (long long)c->nnz, prev, w, sched_variants(problem));
    SCOUT_LAUNCH(c, "k_sched_infer");
    c->nlaunch += 1;
    if (w) *mode_dev = &c->d_ctr->decision;
    return SCOUT_OK;
}

void sched_release(scout_ctx* c) {
    for (int i = 0; i < 4; i++) {
        if (c->model[i]) dev_free(c, c->model[i], mlp::NPARAM * 2);
        c->model[i] = nullptr;
    }
    if (c->probe_buf) dev_free(c, c->probe_buf, (size_t)(2 * c->n + 64) * 4);
    c->probe_buf = nullptr;
    if (c->d_ctr_snap) dev_free(c, c->d_ctr_snap, sizeof(DevCounters));
    c->d_ctr_snap = nullptr;
}

}  // namespace scout

using namespace scout;

extern "C" {

int scout_sched_install(scout_ctx* c, int problem, const float* params, int64_t count) {
    if (!c) return SCOUT_E_INVALID;
    if (problem != SCOUT_BFS && problem != SCOUT_CC)
        return c->fail(SCOUT_E_INVALID, "the learned scheduler applies to BFS and CC only");
    cudaSetDevice(c->device);
    if (!params) {   // uninstall: back to the plain policy
        if (c->model[problem]) dev_free(c, c->model[problem], mlp::NPARAM * 2);
        c->model[problem] = nullptr;
        return SCOUT_OK;
    }
    if (count != mlp::NPARAM) return c->fail(SCOUT_E_INVALID, "model must have 6020 parameters");
    for (int64_t i = 0; i < count; i++)
        if (!std::isfinite(params[i])) return c->fail(SCOUT_E_INVALID, "model parameter is not finite");
    std::vector<__nv_bfloat16> wb(count);
    for (int64_t i = 0; i < count; i++) wb[i] = __float2bfloat16_rn(params[i]);
    if (!c->model[problem]) SCOUT_RC(dev_alloc(c, &c->model[problem], mlp::NPARAM * 2, "scheduler model"));
    SCOUT_CU(c, cudaMemcpyAsync(c->model[problem], wb.data(), mlp::NPARAM * 2, cudaMemcpyHostToDevice, c->s_main));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    return SCOUT_OK;
}

int scout_sched_last(scout_ctx* c, float* features, float* pred, int32_t* decision) {
    if (!c) return SCOUT_E_INVALID;
    const DevCounters& h = *c->h_ctr;
    if (!(h.sched_flags & 1)) return c->fail(SCOUT_E_STATE, "the last repair computed no scheduler features");
    if (features) for (int i = 0; i < mlp::IN; i++) features[i] = h.feat[i];
    if (pred) for (int i = 0; i < mlp::OUT; i++) pred[i] = (h.sched_flags & 2) ? h.pred[i] : NAN;
    if (decision) *decision = h.decision;
    return SCOUT_OK;
}

}  // extern "C"
