// Tensor-core inference of the learned troubled-cell indicator for 16 cells
// per warp, fused into the mixed-precision DG stage kernel (dg_mixed.cu).
//
// One m16 row tile per warp: the 16 cells' 40 features, BF16, in a per-warp
// shared-memory tile; three mma.sync m16n8k16 BF16 layers (K = 48 (40 + zero
// padding), 32, 32; N = 32 hidden units as four n8 tiles) with FP32
// accumulators initialised to the biases; GELU (tanh form) in FP32 on packed
// pairs, rounded to BF16 pairs that are the next layer's A fragments; the
// output unit in FP32.  Weights are packed in fragment order (one 8-byte
// load per lane per mma, the same for every warp) and read through L1.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>
#include <cstring>

#include "f32x2.cuh"
#include "zk_mlp.h"

namespace zk {

// Row stride (BF16 elements) of the per-warp feature tile: 56 = 28 words, so
// the A-fragment loads of the 8 row groups fall in distinct banks.
constexpr int MLP_TILE_KP = 56;

// Weights in mma fragment order.  For layer l, k step kt and n tile nt, lane
// (g = lane / 4, q = lane % 4) holds b0 = W[nt*8+g][kt*16+2q .. +1] and b1 =
// W[nt*8+g][kt*16+8+2q .. +1] as BF16 pairs (low half first); bias and w4
// pairs are the columns nt*8+2q, nt*8+2q+1 of this lane's accumulators.
struct MlpFrag {
    uint2 w1[3][4][32];
    uint2 w2[2][4][32];
    uint2 w3[2][4][32];
    float2 b1[4][32], b2[4][32], b3[4][32];
    float2 w4[4][32];
    float b4, pad[3];
};
static_assert(sizeof(MlpFrag) % 16 == 0, "MlpFrag is copied in 16-byte units");

inline uint16_t bf16_bits_host(float x) {
    const __nv_bfloat16 b = __float2bfloat16(x);
    uint16_t u;
    std::memcpy(&u, &b, 2);
    return u;
}

inline float bf16_round_host(float x) { return __bfloat162float(__float2bfloat16(x)); }

// Host: fragment-order packing of the FP32 parameters, every one rounded to
// BF16 (the inference parameters).
inline void pack_mlp_frag(const MlpWeights& W, MlpFrag* F) {
    std::memset(F, 0, sizeof *F);
    auto pair = [](const float* row, int k, int kin) {
        const uint32_t lo = k < kin ? bf16_bits_host(row[k]) : 0u;
        const uint32_t hi = k + 1 < kin ? bf16_bits_host(row[k + 1]) : 0u;
        return lo | (hi << 16);
    };
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, q = lane & 3;
        for (int nt = 0; nt < 4; ++nt) {
            const int n = nt * 8 + g, c = nt * 8 + 2 * q;
            for (int kt = 0; kt < 3; ++kt)
                F->w1[kt][nt][lane] = make_uint2(pair(W.w1[n], kt * 16 + 2 * q, MLP_IN),
                                                 pair(W.w1[n], kt * 16 + 8 + 2 * q, MLP_IN));
            for (int kt = 0; kt < 2; ++kt) {
                F->w2[kt][nt][lane] = make_uint2(pair(W.w2[n], kt * 16 + 2 * q, MLP_H),
                                                 pair(W.w2[n], kt * 16 + 8 + 2 * q, MLP_H));
                F->w3[kt][nt][lane] = make_uint2(pair(W.w3[n], kt * 16 + 2 * q, MLP_H),
                                                 pair(W.w3[n], kt * 16 + 8 + 2 * q, MLP_H));
            }
            F->b1[nt][lane] = make_float2(bf16_round_host(W.b1[c]), bf16_round_host(W.b1[c + 1]));
            F->b2[nt][lane] = make_float2(bf16_round_host(W.b2[c]), bf16_round_host(W.b2[c + 1]));
            F->b3[nt][lane] = make_float2(bf16_round_host(W.b3[c]), bf16_round_host(W.b3[c + 1]));
            F->w4[nt][lane] = make_float2(bf16_round_host(W.w4[c]), bf16_round_host(W.w4[c + 1]));
        }
    }
    F->b4 = bf16_round_host(W.b4);
}

__device__ __forceinline__ void mma16816_bf16(float (&c)[4], const uint32_t (&a)[4], uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// GELU (tanh form) of two FP32 accumulator values, returned as a BF16 pair
// (low half = x0): u = K (x + C x^3), 0.5 x (1 + tanh u) on packed FP32 pairs
// with the hardware tanh per lane, then one round-to-nearest conversion.  (A
// BF16 tanh would cancel in 1 + tanh u for negative x: the logits drifted by
// about 1 against the FP32 forward pass.)
__device__ __forceinline__ uint32_t gelu_bf16x2(float x0, float x1) {
    const float2 x = make_float2(x0, x1);
    const float2 u = mul2(f2(GELU_K), fma2(mul2(f2(GELU_C), mul2(x, x)), x, x));
    float t0, t1;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(u.x));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(u.y));
    const float2 hx = mul2(f2(0.5f), x);
    const float2 g = fma2(hx, make_float2(t0, t1), hx);
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(g.y), "f"(g.x));
    return r;
}

__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// One hidden layer: acc = bias + A W^T over KSTEPS k steps, then GELU into
// the next layer's A fragments (2 k steps of 16 from the 4 n tiles).
template <int KSTEPS>
__device__ __forceinline__ void mlp_layer16(const uint32_t (&a)[KSTEPS][4], const uint2 (*w)[4][32],
                                            const float2 (*bias)[32], int lane, uint32_t (&out)[2][4]) {
    float c[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const float2 b = __ldg(&bias[nt][lane]);
        c[nt][0] = b.x; c[nt][1] = b.y; c[nt][2] = b.x; c[nt][3] = b.y;
    }
#pragma unroll
    for (int kt = 0; kt < KSTEPS; ++kt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma16816_bf16(c[nt], a[kt], __ldg(&w[kt][nt][lane]));
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
        out[kt][0] = gelu_bf16x2(c[2 * kt][0], c[2 * kt][1]);
        out[kt][1] = gelu_bf16x2(c[2 * kt][2], c[2 * kt][3]);
        out[kt][2] = gelu_bf16x2(c[2 * kt + 1][0], c[2 * kt + 1][1]);
        out[kt][3] = gelu_bf16x2(c[2 * kt + 1][2], c[2 * kt + 1][3]);
    }
}

// Logits of the 16 rows of `tile` (this warp's [16][MLP_TILE_KP] BF16
// features, rows written and __syncwarp'ed by the caller): row g in `lo` and
// row g + 8 in `hi` of every lane of quad g (W in global memory).  Every lane
// of the warp calls it.
__device__ __forceinline__ void mlp_logits16(const MlpFrag* __restrict__ W, const uint16_t* tile, int lane,
                                             float& lo, float& hi) {
    const int g = lane >> 2, q = lane & 3;
    uint32_t a1[3][4];
#pragma unroll
    for (int kt = 0; kt < 3; ++kt) {
        const uint16_t* r0 = tile + g * MLP_TILE_KP + kt * 16 + 2 * q;
        const uint16_t* r1 = r0 + 8 * MLP_TILE_KP;
        a1[kt][0] = *reinterpret_cast<const uint32_t*>(r0);
        a1[kt][1] = *reinterpret_cast<const uint32_t*>(r1);
        a1[kt][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
        a1[kt][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
    }
    uint32_t h1[2][4], h2[2][4], h3[2][4];
    mlp_layer16<3>(a1, W->w1, W->b1, lane, h1);
    mlp_layer16<2>(h1, W->w2, W->b2, lane, h2);
    mlp_layer16<2>(h2, W->w3, W->b3, lane, h3);
    // output unit: this lane's 8 columns of rows g (lo) and g + 8 (hi), then
    // the sum over the quad
    float l = 0.0f, h = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 2; ++kt)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const float2 w4 = __ldg(&W->w4[2 * kt + half][lane]);
            const uint32_t rg = h3[kt][2 * half], rg8 = h3[kt][2 * half + 1];
            l = fmaf(w4.x, bf16_lo(rg), fmaf(w4.y, bf16_hi(rg), l));
            h = fmaf(w4.x, bf16_lo(rg8), fmaf(w4.y, bf16_hi(rg8), h));
        }
    l += __shfl_xor_sync(0xffffffffu, l, 1);
    l += __shfl_xor_sync(0xffffffffu, l, 2);
    h += __shfl_xor_sync(0xffffffffu, h, 1);
    h += __shfl_xor_sync(0xffffffffu, h, 2);
    const float b4 = __ldg(&W->b4);
    lo = l + b4;
    hi = h + b4;
}

}  // namespace zk
