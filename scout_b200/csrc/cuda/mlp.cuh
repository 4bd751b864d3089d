// mlp.cuh -- layout of the scheduler's cost model, shared by the training kernels (mlp.cu)
// and the on-device inference of the learned scheduler (sched.cu).
//
// The model is a 24 -> 64 -> 64 -> 4 perceptron with ReLU hidden layers. Parameters are one
// flat fp32 vector (the training master copy); inference reads a bf16 copy of it.
//   W1[64][24] b1[64] W2[64][64] b2[64] W3[4][64] b3[4]     (6,020 values)
// Row j of a weight matrix holds the input weights of output unit j.
#pragma once

#include <cuda_bf16.h>

namespace scout {
namespace mlp {

constexpr int IN = 24;
constexpr int H = 64;
constexpr int OUT = 4;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * IN;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + OUT * H;
constexpr int NPARAM = OFF_B3 + OUT;
static_assert(NPARAM == 6020, "parameter count of the 24-64-64-4 model");

__device__ __forceinline__ float ld_param(const float* w, int i) { return w[i]; }
__device__ __forceinline__ float ld_param(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// Forward pass of one sample by one thread (used for evaluation and for the scheduler's
// single-sample inference). Accumulation is fp32 whatever the parameter type.
template <typename P>
__device__ void forward_one(const P* w, const float* x, float* y) {
    float h1[H];
#pragma unroll 4
    for (int j = 0; j < H; j++) {
        float a = ld_param(w, OFF_B1 + j);
#pragma unroll
        for (int k = 0; k < IN; k++) a = fmaf(ld_param(w, OFF_W1 + j * IN + k), x[k], a);
        h1[j] = fmaxf(a, 0.f);
    }
    float h2[H];
#pragma unroll 2
    for (int j = 0; j < H; j++) {
        float a = ld_param(w, OFF_B2 + j);
#pragma unroll
        for (int k = 0; k < H; k++) a = fmaf(ld_param(w, OFF_W2 + j * H + k), h1[k], a);
        h2[j] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int o = 0; o < OUT; o++) {
        float a = ld_param(w, OFF_B3 + o);
#pragma unroll
        for (int k = 0; k < H; k++) a = fmaf(ld_param(w, OFF_W3 + o * H + k), h2[k], a);
        y[o] = a;
    }
}

}  // namespace mlp
}  // namespace scout
