// The learned troubled-cell indicator: a 40 -> 32 -> 32 -> 32 -> 1 MLP with
// GELU activations.  Inputs per cell of an RK stage's output (FP32 values of
// the FP64/FP32 DG states), the "means" being those of the stage's INPUT:
//   f[0..15]   the output's rho modes, slot px*4+py, divided by s_rho = max
//              |rho mean| over the cell and its 4 neighbours, minus 1 in slot
//              0 (the mean), so that a constant state's features are all 0
//   f[16..31]  the output's E modes, same slots, divided by s_E (slot 16 - 1)
//   f[32..35]  (rho mean of neighbour L, R, U, D - own rho mean) / s_rho
//   f[36..39]  the same for E
// Output: a logit; > 0 flags the cell for TVB characteristic limiting.  The
// means of the stage input are in the mixed-precision stage kernel's tile, so
// the indicator runs inside that kernel (dg_mixed.cu, mlp_infer.cuh).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace zk {

constexpr int MLP_IN = 40, MLP_H = 32;
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + 2 * (MLP_H * MLP_H + MLP_H) + MLP_H + 1;

// Parameters in one flat block (row-major weights, out x in).  For inference
// the values are BF16-rounded copies of the FP32 trained parameters.
struct MlpWeights {
    float w1[MLP_H][MLP_IN];
    float b1[MLP_H];
    float w2[MLP_H][MLP_H];
    float b2[MLP_H];
    float w3[MLP_H][MLP_H];
    float b3[MLP_H];
    float w4[MLP_H];
    float b4;
};
static_assert(sizeof(MlpWeights) == sizeof(float) * MLP_NPARAM, "MlpWeights must be a flat float block");

// Inference copy of the weights, packed on the host in the exact shared-memory
// layout of the tensor-core inference (BF16 bits, rows padded for mma
// fragment loads), so a CTA stages it with 16-byte vector copies.
constexpr int MLP_KP1 = 56, MLP_KP2 = 40;
struct MlpPacked {
    uint16_t w1[MLP_H][MLP_KP1];  // [out][in], in 40..55 zero
    uint16_t w2[MLP_H][MLP_KP2];  // [out][in], in 32..39 zero
    uint16_t w3[MLP_H][MLP_KP2];
    float b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_H];
    float b4, pad[3];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked is copied in 16-byte units");

// GELU in its tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
constexpr float GELU_K = 0.7978845608028654f, GELU_C = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + tanhf(GELU_K * (x + GELU_C * x * x * x)));
}
// The same with the hardware tanh approximation (inference).
__device__ __forceinline__ float gelu_fast(float x) {
    float t;
    const float u = GELU_K * (x + GELU_C * x * x * x);
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return 0.5f * x * (1.0f + t);
}

// Plain FP32 forward pass (CUDA cores).
__device__ __forceinline__ float mlp_logit(const MlpWeights& W, const float f[MLP_IN]) {
    float h1[MLP_H], h2[MLP_H];
#pragma unroll 4
    for (int o = 0; o < MLP_H; ++o) {
        float s = W.b1[o];
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) s = fmaf(W.w1[o][i], f[i], s);
        h1[o] = gelu(s);
    }
#pragma unroll 4
    for (int o = 0; o < MLP_H; ++o) {
        float s = W.b2[o];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) s = fmaf(W.w2[o][i], h1[i], s);
        h2[o] = gelu(s);
    }
    float out = W.b4;
#pragma unroll 4
    for (int o = 0; o < MLP_H; ++o) {
        float s = W.b3[o];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) s = fmaf(W.w3[o][i], h2[i], s);
        out = fmaf(W.w4[o], gelu(s), out);
    }
    return out;
}

}  // namespace zk
