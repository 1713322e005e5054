// Training and evaluation kernels of the learned troubled-cell indicator
// (zk_mlp.h): FP32 forward + backward over mini-batches, an Adam update, and a
// batched forward pass.  Loss: binary cross-entropy on the logit with a
// positive-class weight (troubled cells are rare).
//
// fwd_bwd: one CTA = 64 samples, one thread per sample.  Each thread runs the
// forward pass and backpropagates to the per-layer deltas dz (input gradients
// of the pre-activations); activations and deltas go to shared memory; then
// the threads own parameter entries and reduce sum_s dz[s][o] * act[s][i] over
// the CTA's samples, adding the CTA's partial gradient to the global buffer.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "zk_internal.h"
#include "zk_mlp.h"

namespace zk {
namespace {

constexpr int NS = 64;  // samples per CTA
constexpr int H = MLP_H, IN = MLP_IN, NP = MLP_NPARAM;

// parameter offsets in the flat block
constexpr int OW1 = 0, OB1 = OW1 + H * IN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * H,
              OW4 = OB3 + H, OB4 = OW4 + H;

// d/dx of the tanh-form GELU.
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanhf(GELU_K * (x + GELU_C * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_K * (1.0f + 3.0f * GELU_C * x * x);
}

struct SmemFB {
    float p[NP];
    float x[NS][IN];
    float h1[NS][H], h2[NS][H], h3[NS][H];
    float d1[NS][H], d2[NS][H], d3[NS][H];
    float d4[NS];
};

__global__ void __launch_bounds__(NS) mlp_fwd_bwd_kernel(const float* X, const uint8_t* y, const int64_t* idx,
                                                         int64_t n, const float* params, float* grad, float* loss,
                                                         float pos_weight) {
    extern __shared__ __align__(16) unsigned char raw[];
    SmemFB& S = *reinterpret_cast<SmemFB*>(raw);
    const int t = threadIdx.x;
    for (int i = t; i < NP; i += NS) S.p[i] = params[i];
    const int64_t s = (int64_t)blockIdx.x * NS + t;
    const bool live = s < n;
    const int64_t src = live ? (idx ? idx[s] : s) : 0;
    for (int i = 0; i < IN; ++i) S.x[t][i] = live ? X[src * IN + i] : 0.0f;
    __syncthreads();
    const float* w1 = S.p + OW1;
    const float* w2 = S.p + OW2;
    const float* w3 = S.p + OW3;
    float z1[H], z2[H], z3[H];
    for (int o = 0; o < H; ++o) {
        float a = S.p[OB1 + o];
        for (int i = 0; i < IN; ++i) a = fmaf(w1[o * IN + i], S.x[t][i], a);
        z1[o] = a;
        S.h1[t][o] = gelu(a);
    }
    for (int o = 0; o < H; ++o) {
        float a = S.p[OB2 + o];
        for (int i = 0; i < H; ++i) a = fmaf(w2[o * H + i], S.h1[t][i], a);
        z2[o] = a;
        S.h2[t][o] = gelu(a);
    }
    float z = S.p[OB4];
    for (int o = 0; o < H; ++o) {
        float a = S.p[OB3 + o];
        for (int i = 0; i < H; ++i) a = fmaf(w3[o * H + i], S.h2[t][i], a);
        z3[o] = a;
        const float h = gelu(a);
        S.h3[t][o] = h;
        z = fmaf(S.p[OW4 + o], h, z);
    }
    // BCE with logits, positive weight
    const float yt = live ? (float)y[src] : 0.0f;
    const float sig = 1.0f / (1.0f + expf(-z));
    const float sp_pos = fmaxf(-z, 0.0f) + log1pf(expf(-fabsf(z)));  // softplus(-z)
    const float sp_neg = fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z)));   // softplus(z)
    const float l = live ? pos_weight * yt * sp_pos + (1.0f - yt) * sp_neg : 0.0f;
    const float dz = live ? pos_weight * yt * (sig - 1.0f) + (1.0f - yt) * sig : 0.0f;
    S.d4[t] = dz;
    float d3[H], d2[H];
    for (int o = 0; o < H; ++o) {
        d3[o] = dz * S.p[OW4 + o] * gelu_grad(z3[o]);
        S.d3[t][o] = d3[o];
    }
    for (int i = 0; i < H; ++i) {
        float a = 0.0f;
        for (int o = 0; o < H; ++o) a = fmaf(w3[o * H + i], d3[o], a);
        d2[i] = a * gelu_grad(z2[i]);
        S.d2[t][i] = d2[i];
    }
    for (int i = 0; i < H; ++i) {
        float a = 0.0f;
        for (int o = 0; o < H; ++o) a = fmaf(w2[o * H + i], d2[o], a);
        S.d1[t][i] = a * gelu_grad(z1[i]);
    }
    // block loss
    float lw = l;
    for (int o = 16; o > 0; o >>= 1) lw += __shfl_xor_sync(0xffffffffu, lw, o);
    if ((t & 31) == 0) atomicAdd(loss, lw);
    __syncthreads();
    // parameter gradients: sum over the CTA's samples
    for (int p = t; p < NP; p += NS) {
        float g = 0.0f;
        if (p < OB1) {
            const int o = p / IN, i = p % IN;
            for (int k = 0; k < NS; ++k) g = fmaf(S.d1[k][o], S.x[k][i], g);
        } else if (p < OW2) {
            for (int k = 0; k < NS; ++k) g += S.d1[k][p - OB1];
        } else if (p < OB2) {
            const int o = (p - OW2) / H, i = (p - OW2) % H;
            for (int k = 0; k < NS; ++k) g = fmaf(S.d2[k][o], S.h1[k][i], g);
        } else if (p < OW3) {
            for (int k = 0; k < NS; ++k) g += S.d2[k][p - OB2];
        } else if (p < OB3) {
            const int o = (p - OW3) / H, i = (p - OW3) % H;
            for (int k = 0; k < NS; ++k) g = fmaf(S.d3[k][o], S.h2[k][i], g);
        } else if (p < OW4) {
            for (int k = 0; k < NS; ++k) g += S.d3[k][p - OB3];
        } else if (p < OB4) {
            for (int k = 0; k < NS; ++k) g = fmaf(S.d4[k], S.h3[k][p - OW4], g);
        } else {
            for (int k = 0; k < NS; ++k) g += S.d4[k];
        }
        atomicAdd(&grad[p], g);
    }
}

// Adam on the mean gradient (grad holds the batch sum); grad is cleared.
__global__ void mlp_adam_kernel(float* params, float* grad, float* m, float* v, float inv_batch, float lr, float b1,
                                float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float g = grad[p] * inv_batch;
    grad[p] = 0.0f;
    m[p] = b1 * m[p] + (1.0f - b1) * g;
    v[p] = b2 * v[p] + (1.0f - b2) * g * g;
    params[p] -= lr * (m[p] / c1) / (sqrtf(v[p] / c2) + eps);
}

__global__ void mlp_forward_kernel(const float* X, int64_t n, const MlpWeights* W, float* out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float f[IN];
    for (int i = 0; i < IN; ++i) f[i] = X[s * IN + i];
    out[s] = mlp_logit(*W, f);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

int cuda_fail(cudaError_t e) { return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e)); }

}  // namespace
}  // namespace zk

using namespace zk;

// Mean loss and mean gradient over n samples (the gradient check entry point).
extern "C" int zk_mlp_grad(int device, const float* X, const uint8_t* y, int64_t n, const float* params,
                           float pos_weight, float* grad, float* loss) {
    if (!X || !y || !params || !grad || !loss || n <= 0) return zk_internal_fail(ZK_ERR_ARG, "bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, "cudaSetDevice failed");
    DevBuf dX, dy, dp, dg, dl;
    cudaError_t e = cudaMalloc(&dX.p, sizeof(float) * IN * n);
    if (e == cudaSuccess) e = cudaMalloc(&dy.p, n);
    if (e == cudaSuccess) e = cudaMalloc(&dp.p, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&dg.p, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&dl.p, sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(dX.p, X, sizeof(float) * IN * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dy.p, y, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp.p, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dg.p, 0, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMemset(dl.p, 0, sizeof(float));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(mlp_fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)sizeof(SmemFB));
    if (e != cudaSuccess) return cuda_fail(e);
    mlp_fwd_bwd_kernel<<<(unsigned)((n + NS - 1) / NS), NS, sizeof(SmemFB)>>>(
        (const float*)dX.p, (const uint8_t*)dy.p, nullptr, n, (const float*)dp.p, (float*)dg.p, (float*)dl.p,
        pos_weight);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(grad, dg.p, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e);
    for (int p = 0; p < NP; ++p) grad[p] /= (float)n;
    *loss /= (float)n;
    return ZK_OK;
}

// Mini-batch Adam training on the GPU.  params: in = initial values, out =
// trained values.  epoch_loss[epochs] (may be NULL) gets the mean loss.
extern "C" int zk_mlp_train(int device, const float* X, const uint8_t* y, int64_t n, float* params, int epochs,
                            int batch, float lr, float pos_weight, uint64_t seed, float* epoch_loss) {
    if (!X || !y || !params || n <= 0 || epochs <= 0 || batch <= 0 || batch % NS)
        return zk_internal_fail(ZK_ERR_ARG, "bad argument (batch must be a positive multiple of 64)");
    if (cudaSetDevice(device) != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, "cudaSetDevice failed");
    DevBuf dX, dy, di, dp, dg, dm, dv, dl;
    cudaError_t e = cudaMalloc(&dX.p, sizeof(float) * IN * n);
    if (e == cudaSuccess) e = cudaMalloc(&dy.p, n);
    if (e == cudaSuccess) e = cudaMalloc(&di.p, sizeof(int64_t) * n);
    for (DevBuf* b : {&dp, &dg, &dm, &dv})
        if (e == cudaSuccess) e = cudaMalloc(&b->p, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&dl.p, sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(dX.p, X, sizeof(float) * IN * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dy.p, y, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp.p, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
    for (DevBuf* b : {&dg, &dm, &dv})
        if (e == cudaSuccess) e = cudaMemset(b->p, 0, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(mlp_fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)sizeof(SmemFB));
    if (e != cudaSuccess) return cuda_fail(e);
    std::vector<int64_t> perm(n);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int64_t step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int64_t i = 0; i < n; ++i) perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        e = cudaMemcpy(di.p, perm.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(dl.p, 0, sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e);
        for (int64_t off = 0; off < n; off += batch) {
            const int64_t nb = (n - off < batch) ? n - off : batch;
            mlp_fwd_bwd_kernel<<<(unsigned)((nb + NS - 1) / NS), NS, sizeof(SmemFB)>>>(
                (const float*)dX.p, (const uint8_t*)dy.p, (const int64_t*)di.p + off, nb, (const float*)dp.p,
                (float*)dg.p, (float*)dl.p, pos_weight);
            ++step;
            const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
            mlp_adam_kernel<<<(NP + 255) / 256, 256>>>((float*)dp.p, (float*)dg.p, (float*)dm.p, (float*)dv.p,
                                                       1.0f / (float)nb, lr, b1, b2, eps, c1, c2);
        }
        e = cudaGetLastError();
        float l = 0.0f;
        if (e == cudaSuccess) e = cudaMemcpy(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e);
        if (epoch_loss) epoch_loss[ep] = l / (float)n;
    }
    e = cudaMemcpy(params, dp.p, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// Logits of n samples; bf16 != 0 rounds the weights to BF16 first (the
// inference weights of zk_set_indicator).
extern "C" int zk_mlp_forward(int device, const float* X, int64_t n, const float* params, int bf16, float* logits) {
    if (!X || !params || !logits || n <= 0) return zk_internal_fail(ZK_ERR_ARG, "bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, "cudaSetDevice failed");
    std::vector<float> w(params, params + NP);
    if (bf16)
        for (float& x : w) x = __bfloat162float(__float2bfloat16(x));
    DevBuf dX, dW, dO;
    cudaError_t e = cudaMalloc(&dX.p, sizeof(float) * IN * n);
    if (e == cudaSuccess) e = cudaMalloc(&dW.p, sizeof(MlpWeights));
    if (e == cudaSuccess) e = cudaMalloc(&dO.p, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemcpy(dX.p, X, sizeof(float) * IN * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dW.p, w.data(), sizeof(MlpWeights), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e);
    mlp_forward_kernel<<<(unsigned)((n + 127) / 128), 128>>>((const float*)dX.p, n, (const MlpWeights*)dW.p,
                                                             (float*)dO.p);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(logits, dO.p, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}
