// mlp.cu -- training and evaluation of the scheduler's cost model on the device.
//
// Hand-written kernels, no library: a fused forward + backward kernel over tiles of 32
// samples (activations staged in shared memory, gradients of the tile reduced in shared
// memory and added to the global gradient with one atomic per parameter per tile), an Adam
// step (Kingma and Ba, "Adam: a method for stochastic optimization", ICLR 2015, with bias
// correction), and a per-sample forward pass over fp32 or bf16 parameters. The minibatch
// loop of one epoch is captured once in a CUDA graph and replayed every epoch with a fresh
// permutation of the samples.
//
// Loss: masked mean squared error, L = sum_{s,o} mask[s][o] (y[s][o] - t[s][o])^2 / sum(mask)
// over the minibatch (a target with mask 0 is not measured, e.g. a repair variant that a
// problem does not have).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../../include/scout_gpu.h"
#include "mlp.cuh"

namespace scout {
int host_fail(int code, const std::string& msg);

namespace mlp {

constexpr int TILE = 32;       // samples per block in the fused kernel
constexpr int THREADS = 256;

struct Buffers {
    float* x = nullptr;       // [n][IN]
    float* t = nullptr;       // [n][OUT]
    float* m = nullptr;       // [n][OUT]
    int32_t* idx = nullptr;   // sample order of the current epoch
    float* y = nullptr;       // [n][OUT] forward outputs
    int64_t cap = 0;
};

}  // namespace mlp
}  // namespace scout

struct scout_mlp {
    int device = 0;
    cudaStream_t s = nullptr;
    float* w = nullptr;       // fp32 master parameters
    float* g = nullptr;       // gradient
    float* am = nullptr;      // Adam first moment
    float* av = nullptr;      // Adam second moment
    __nv_bfloat16* wb = nullptr;   // bf16 copy for inference
    float* loss = nullptr;    // [2]: minibatch loss sum, epoch loss sum
    int* step = nullptr;      // Adam step counter (device)
    scout::mlp::Buffers d;
};

namespace scout {
namespace mlp {

// Fused forward + backward over one tile of samples idx[b0 .. b0 + cnt).
// inv_norm = 1 / sum(mask) of the minibatch (gradient scale); inv_epoch = 1 / sum(mask)
// over the whole epoch (loss report).
__global__ void __launch_bounds__(THREADS) k_grad(const float* __restrict__ w, float* __restrict__ g,
                                                  const float* __restrict__ X, const float* __restrict__ Tg,
                                                  const float* __restrict__ M, const int32_t* __restrict__ idx,
                                                  int64_t b0, int cnt, const float* __restrict__ norms,
                                                  int norm_slot, float* __restrict__ loss) {
    __shared__ float sx[TILE][IN];
    __shared__ float h1[TILE][H];
    __shared__ float h2[TILE][H];
    __shared__ float d2[TILE][H];
    __shared__ float d1[TILE][H];
    __shared__ float dy[TILE][OUT];
    __shared__ float red[THREADS / 32];
    const int t = threadIdx.x;
    const int s0 = blockIdx.x * TILE;
    const int ns = min(TILE, cnt - s0);
    if (ns <= 0) return;
    const float inv_norm = norms[2 * norm_slot], inv_epoch = norms[2 * norm_slot + 1];
    for (int i = t; i < TILE * IN; i += THREADS) {
        int s = i / IN, k = i % IN;
        sx[s][k] = s < ns ? X[(int64_t)idx[b0 + s0 + s] * IN + k] : 0.f;
    }
    __syncthreads();
    const int j = t & (H - 1), sq = t / H;   // unit j, samples sq, sq + 4, ...
    {
        float wr[IN];
#pragma unroll
        for (int k = 0; k < IN; k++) wr[k] = w[OFF_W1 + j * IN + k];
        const float b = w[OFF_B1 + j];
        for (int s = sq; s < TILE; s += THREADS / H) {
            float a = b;
#pragma unroll
            for (int k = 0; k < IN; k++) a = fmaf(wr[k], sx[s][k], a);
            h1[s][j] = s < ns ? fmaxf(a, 0.f) : 0.f;
        }
    }
    __syncthreads();
    for (int s = sq; s < TILE; s += THREADS / H) {
        float a = w[OFF_B2 + j];
#pragma unroll 8
        for (int k = 0; k < H; k++) a = fmaf(w[OFF_W2 + j * H + k], h1[s][k], a);
        h2[s][j] = s < ns ? fmaxf(a, 0.f) : 0.f;
    }
    __syncthreads();
    float lsum = 0.f;
    if (t < TILE * OUT) {
        const int s = t / OUT, o = t % OUT;
        float d = 0.f;
        if (s < ns) {
            float a = w[OFF_B3 + o];
#pragma unroll 8
            for (int k = 0; k < H; k++) a = fmaf(w[OFF_W3 + o * H + k], h2[s][k], a);
            const int64_t r = (int64_t)idx[b0 + s0 + s] * OUT + o;
            const float mk = M[r];
            const float diff = a - Tg[r];
            d = 2.f * mk * diff * inv_norm;
            lsum = mk * diff * diff;
        }
        dy[s][o] = d;
    }
    // loss: block reduction, two atomics per block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((t & 31) == 0) red[t / 32] = lsum;
    __syncthreads();
    if (t == 0) {
        float a = 0.f;
        for (int i = 0; i < THREADS / 32; i++) a += red[i];
        atomicAdd(loss + 0, a * inv_norm);
        atomicAdd(loss + 1, a * inv_epoch);
    }
    // layer 3 gradients: one (o, k) per thread
    {
        const int o = t / H, k = t % H;
        float a = 0.f;
        for (int s = 0; s < ns; s++) a = fmaf(dy[s][o], h2[s][k], a);
        atomicAdd(g + OFF_W3 + o * H + k, a);
        if (t < OUT) {
            float b = 0.f;
            for (int s = 0; s < ns; s++) b += dy[s][t];
            atomicAdd(g + OFF_B3 + t, b);
        }
    }
    // dh2 = W3^T dy masked by the ReLU
    for (int s = sq; s < TILE; s += THREADS / H) {
        float a = 0.f;
#pragma unroll
        for (int o = 0; o < OUT; o++) a = fmaf(w[OFF_W3 + o * H + j], dy[s][o], a);
        d2[s][j] = h2[s][j] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // layer 2 gradients: 16 (j, k) pairs per thread, and dh1 = W2^T dh2 masked by the ReLU
    for (int i = t; i < H * H; i += THREADS) {
        const int jj = i / H, k = i % H;
        float a = 0.f;
        for (int s = 0; s < ns; s++) a = fmaf(d2[s][jj], h1[s][k], a);
        atomicAdd(g + OFF_W2 + i, a);
    }
    if (t < H) {
        float b = 0.f;
        for (int s = 0; s < ns; s++) b += d2[s][t];
        atomicAdd(g + OFF_B2 + t, b);
    }
    for (int s = sq; s < TILE; s += THREADS / H) {
        float a = 0.f;
#pragma unroll 8
        for (int jj = 0; jj < H; jj++) a = fmaf(w[OFF_W2 + jj * H + j], d2[s][jj], a);
        d1[s][j] = h1[s][j] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // layer 1 gradients
    for (int i = t; i < H * IN; i += THREADS) {
        const int jj = i / IN, k = i % IN;
        float a = 0.f;
        for (int s = 0; s < ns; s++) a = fmaf(d1[s][jj], sx[s][k], a);
        atomicAdd(g + OFF_W1 + i, a);
    }
    if (t < H) {
        float b = 0.f;
        for (int s = 0; s < ns; s++) b += d1[s][t];
        atomicAdd(g + OFF_B1 + t, b);
    }
}

// Zeroes the gradient and the minibatch loss; advances the Adam step counter.
__global__ void k_zero(float* __restrict__ g, float* __restrict__ loss, int* __restrict__ step) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) g[i] = 0.f;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        loss[0] = 0.f;
        *step += 1;
    }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, const int* __restrict__ step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int tstep = *step;
    const float c1 = 1.f - powf(b1, (float)tstep), c2 = 1.f - powf(b2, (float)tstep);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

template <typename P>
__global__ void k_forward(const P* __restrict__ w, const float* __restrict__ X, int64_t n, float* __restrict__ Y) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        float x[IN], y[OUT];
#pragma unroll
        for (int k = 0; k < IN; k++) x[k] = X[s * IN + k];
        forward_one(w, x, y);
#pragma unroll
        for (int o = 0; o < OUT; o++) Y[s * OUT + o] = y[o];
    }
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

static int cu(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return SCOUT_OK;
    cudaGetLastError();
    return host_fail(SCOUT_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define MLP_CU(call) do { int rc_ = cu((call), #call); if (rc_ != SCOUT_OK) return rc_; } while (0)

static int ensure_data(scout_mlp* m, int64_t n) {
    if (m->d.cap >= n) return SCOUT_OK;
    cudaFree(m->d.x); cudaFree(m->d.t); cudaFree(m->d.m); cudaFree(m->d.idx); cudaFree(m->d.y);
    m->d = Buffers{};
    const int64_t c = std::max<int64_t>(n, 1024);
    MLP_CU(cudaMalloc((void**)&m->d.x, (size_t)c * IN * 4));
    MLP_CU(cudaMalloc((void**)&m->d.t, (size_t)c * OUT * 4));
    MLP_CU(cudaMalloc((void**)&m->d.m, (size_t)c * OUT * 4));
    MLP_CU(cudaMalloc((void**)&m->d.idx, (size_t)c * 4));
    MLP_CU(cudaMalloc((void**)&m->d.y, (size_t)c * OUT * 4));
    m->d.cap = c;
    return SCOUT_OK;
}

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number generators", 2014)
static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unif(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

// He-uniform weights (bound sqrt(6 / fan_in)), zero biases.
static void init_params(std::vector<float>& w, uint64_t seed) {
    w.assign(NPARAM, 0.f);
    uint64_t s = seed ^ 0x5C0u;
    auto fill = [&](int off, int rows, int fan_in) {
        const double b = std::sqrt(6.0 / fan_in);
        for (int i = 0; i < rows * fan_in; i++) w[off + i] = (float)((2.0 * unif(s) - 1.0) * b);
    };
    fill(OFF_W1, H, IN);
    fill(OFF_W2, H, H);
    fill(OFF_W3, OUT, H);
}

}  // namespace mlp
}  // namespace scout

using namespace scout;
using namespace scout::mlp;

extern "C" {

int scout_mlp_create(int device, uint64_t seed, scout_mlp** out) {
    if (!out) return host_fail(SCOUT_E_INVALID, "scout_mlp_create: null output");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return host_fail(SCOUT_E_NODEV, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return host_fail(SCOUT_E_INVALID, "device id out of range");
    MLP_CU(cudaSetDevice(device));
    scout_mlp* m = new scout_mlp();
    m->device = device;
    auto fail = [&](int rc) { scout_mlp_destroy(m); return rc; };
    int rc;
    if ((rc = cu(cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking), "stream")) != SCOUT_OK) return fail(rc);
    float** bufs[] = {&m->w, &m->g, &m->am, &m->av};
    for (float** b : bufs) {
        if ((rc = cu(cudaMalloc((void**)b, NPARAM * 4), "cudaMalloc")) != SCOUT_OK) return fail(rc);
        cudaMemset(*b, 0, NPARAM * 4);
    }
    if ((rc = cu(cudaMalloc((void**)&m->wb, NPARAM * 2), "cudaMalloc")) != SCOUT_OK) return fail(rc);
    if ((rc = cu(cudaMalloc((void**)&m->loss, 8 * 4), "cudaMalloc")) != SCOUT_OK) return fail(rc);
    if ((rc = cu(cudaMalloc((void**)&m->step, 4), "cudaMalloc")) != SCOUT_OK) return fail(rc);
    cudaMemset(m->step, 0, 4);
    std::vector<float> w;
    init_params(w, seed);
    if ((rc = scout_mlp_set_params(m, w.data(), NPARAM)) != SCOUT_OK) return fail(rc);
    *out = m;
    return SCOUT_OK;
}

int scout_mlp_destroy(scout_mlp* m) {
    if (!m) return SCOUT_OK;
    cudaSetDevice(m->device);
    if (m->s) cudaStreamSynchronize(m->s);
    void* ps[] = {m->w, m->g, m->am, m->av, m->wb, m->loss, m->step, m->d.x, m->d.t, m->d.m, m->d.idx, m->d.y};
    for (void* p : ps) if (p) cudaFree(p);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return SCOUT_OK;
}

int scout_mlp_get_params(scout_mlp* m, float* out, int64_t count) {
    if (!m || !out || count != NPARAM) return host_fail(SCOUT_E_INVALID, "scout_mlp_get_params: bad arguments");
    MLP_CU(cudaSetDevice(m->device));
    MLP_CU(cudaMemcpyAsync(out, m->w, NPARAM * 4, cudaMemcpyDeviceToHost, m->s));
    MLP_CU(cudaStreamSynchronize(m->s));
    return SCOUT_OK;
}

int scout_mlp_set_params(scout_mlp* m, const float* in, int64_t count) {
    if (!m || !in || count != NPARAM) return host_fail(SCOUT_E_INVALID, "scout_mlp_set_params: bad arguments");
    MLP_CU(cudaSetDevice(m->device));
    MLP_CU(cudaMemcpyAsync(m->w, in, NPARAM * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemsetAsync(m->am, 0, NPARAM * 4, m->s));
    MLP_CU(cudaMemsetAsync(m->av, 0, NPARAM * 4, m->s));
    MLP_CU(cudaMemsetAsync(m->step, 0, 4, m->s));
    k_to_bf16<<<24, 256, 0, m->s>>>(m->w, m->wb);
    MLP_CU(cudaGetLastError());
    MLP_CU(cudaStreamSynchronize(m->s));
    return SCOUT_OK;
}

int scout_mlp_forward(scout_mlp* m, const float* x, int64_t n, int use_bf16, float* y) {
    if (!m || n < 0 || (n > 0 && (!x || !y))) return host_fail(SCOUT_E_INVALID, "scout_mlp_forward: bad arguments");
    if (n == 0) return SCOUT_OK;
    MLP_CU(cudaSetDevice(m->device));
    int rc = ensure_data(m, n);
    if (rc != SCOUT_OK) return rc;
    MLP_CU(cudaMemcpyAsync(m->d.x, x, (size_t)n * IN * 4, cudaMemcpyHostToDevice, m->s));
    const int blocks = (int)std::min<int64_t>((n + 127) / 128, 148 * 8);
    if (use_bf16) k_forward<__nv_bfloat16><<<blocks, 128, 0, m->s>>>(m->wb, m->d.x, n, m->d.y);
    else k_forward<float><<<blocks, 128, 0, m->s>>>(m->w, m->d.x, n, m->d.y);
    MLP_CU(cudaGetLastError());
    MLP_CU(cudaMemcpyAsync(y, m->d.y, (size_t)n * OUT * 4, cudaMemcpyDeviceToHost, m->s));
    MLP_CU(cudaStreamSynchronize(m->s));
    return SCOUT_OK;
}

static double mask_sum(const float* mask, int64_t a, int64_t b, const std::vector<int32_t>* order) {
    double s = 0;
    for (int64_t i = a; i < b; i++) {
        const int64_t r = order ? (*order)[i] : i;
        for (int o = 0; o < OUT; o++) s += mask[r * OUT + o];
    }
    return s;
}

int scout_mlp_loss_grad(scout_mlp* m, const float* x, const float* t, const float* mask, int64_t n, float* loss,
                        float* grad) {
    if (!m || n <= 0 || !x || !t || !mask) return host_fail(SCOUT_E_INVALID, "scout_mlp_loss_grad: bad arguments");
    MLP_CU(cudaSetDevice(m->device));
    int rc = ensure_data(m, n);
    if (rc != SCOUT_OK) return rc;
    std::vector<int32_t> idx(n);
    for (int64_t i = 0; i < n; i++) idx[i] = (int32_t)i;
    const double ms = mask_sum(mask, 0, n, nullptr);
    float norms[2] = {ms > 0 ? (float)(1.0 / ms) : 0.f, ms > 0 ? (float)(1.0 / ms) : 0.f};
    MLP_CU(cudaMemcpyAsync(m->d.x, x, (size_t)n * IN * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->d.t, t, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->d.m, mask, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->d.idx, idx.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->loss + 2, norms, 8, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemsetAsync(m->g, 0, NPARAM * 4, m->s));
    MLP_CU(cudaMemsetAsync(m->loss, 0, 8, m->s));
    const int blocks = (int)((n + TILE - 1) / TILE);
    k_grad<<<blocks, THREADS, 0, m->s>>>(m->w, m->g, m->d.x, m->d.t, m->d.m, m->d.idx, 0, (int)n, m->loss + 2, 0,
                                          m->loss);
    MLP_CU(cudaGetLastError());
    float hl[2];
    MLP_CU(cudaMemcpyAsync(hl, m->loss, 8, cudaMemcpyDeviceToHost, m->s));
    if (grad) MLP_CU(cudaMemcpyAsync(grad, m->g, NPARAM * 4, cudaMemcpyDeviceToHost, m->s));
    MLP_CU(cudaStreamSynchronize(m->s));
    if (loss) *loss = hl[0];
    return SCOUT_OK;
}

int scout_mlp_train(scout_mlp* m, const float* x, const float* t, const float* mask, int64_t n, int epochs, int batch,
                    float lr, uint64_t seed, float* loss_per_epoch) {
    if (!m || n <= 0 || !x || !t || !mask || epochs < 0 || batch <= 0 || !(lr > 0.f))
        return host_fail(SCOUT_E_INVALID, "scout_mlp_train: bad arguments");
    if (n > INT32_MAX) return host_fail(SCOUT_E_CAPACITY, "scout_mlp_train: too many samples");
    MLP_CU(cudaSetDevice(m->device));
    int rc = ensure_data(m, n);
    if (rc != SCOUT_OK) return rc;
    MLP_CU(cudaMemcpyAsync(m->d.x, x, (size_t)n * IN * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->d.t, t, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, m->s));
    MLP_CU(cudaMemcpyAsync(m->d.m, mask, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, m->s));
    const int64_t nb = (n + batch - 1) / batch;
    // per-minibatch gradient scales live on the device so one captured epoch serves every
    // permutation: [2 b] = 1 / mask sum of minibatch b, [2 b + 1] = 1 / mask sum of the epoch
    float* d_norms = nullptr;
    MLP_CU(cudaMalloc((void**)&d_norms, (size_t)nb * 2 * 4));
    std::vector<float> norms(nb * 2);
    std::vector<int32_t> order(n);
    uint64_t s = seed;
    const double total = mask_sum(mask, 0, n, nullptr);
    cudaGraph_t gr = nullptr;
    cudaGraphExec_t epoch_graph = nullptr;
    rc = SCOUT_OK;
    MLP_CU(cudaStreamBeginCapture(m->s, cudaStreamCaptureModeThreadLocal));
    for (int64_t b = 0; b < nb; b++) {
        const int64_t b0 = b * batch;
        const int cnt = (int)std::min<int64_t>(batch, n - b0);
        k_zero<<<8, 256, 0, m->s>>>(m->g, m->loss, m->step);
        k_grad<<<(cnt + TILE - 1) / TILE, THREADS, 0, m->s>>>(m->w, m->g, m->d.x, m->d.t, m->d.m, m->d.idx, b0, cnt,
                                                               d_norms, (int)b, m->loss);
        k_adam<<<24, 256, 0, m->s>>>(m->w, m->g, m->am, m->av, m->step, lr);
    }
    cudaError_t ce = cudaStreamEndCapture(m->s, &gr);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&epoch_graph, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (ce != cudaSuccess) { cudaFree(d_norms); return cu(ce, "capture of the training epoch"); }
    for (int e = 0; e < epochs && rc == SCOUT_OK; e++) {
        for (int64_t i = 0; i < n; i++) order[i] = (int32_t)i;
        for (int64_t i = n - 1; i > 0; i--) std::swap(order[i], order[(int64_t)(unif(s) * (double)(i + 1)) % (i + 1)]);
        for (int64_t b = 0; b < nb; b++) {
            const int64_t b0 = b * batch, b1 = std::min<int64_t>(n, b0 + batch);
            const double ms = mask_sum(mask, b0, b1, &order);
            norms[2 * b] = ms > 0 ? (float)(1.0 / ms) : 0.f;
            norms[2 * b + 1] = total > 0 ? (float)(1.0 / total) : 0.f;
        }
        rc = cu(cudaMemcpyAsync(m->d.idx, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->s), "idx");
        if (rc == SCOUT_OK) rc = cu(cudaMemcpyAsync(d_norms, norms.data(), (size_t)nb * 8, cudaMemcpyHostToDevice, m->s), "norms");
        if (rc == SCOUT_OK) rc = cu(cudaMemsetAsync(m->loss + 1, 0, 4, m->s), "loss");
        if (rc == SCOUT_OK) rc = cu(cudaGraphLaunch(epoch_graph, m->s), "cudaGraphLaunch");
        if (rc == SCOUT_OK && loss_per_epoch) {
            rc = cu(cudaMemcpyAsync(loss_per_epoch + e, m->loss + 1, 4, cudaMemcpyDeviceToHost, m->s), "loss");
        }
        // the host buffers (order, norms) are rewritten next epoch: wait for this one
        if (rc == SCOUT_OK) rc = cu(cudaStreamSynchronize(m->s), "epoch");
    }
    cudaGraphExecDestroy(epoch_graph);
    cudaFree(d_norms);
    if (rc != SCOUT_OK) return rc;
    k_to_bf16<<<24, 256, 0, m->s>>>(m->w, m->wb);
    MLP_CU(cudaGetLastError());
    MLP_CU(cudaStreamSynchronize(m->s));
    return SCOUT_OK;
}

}  // extern "C"
