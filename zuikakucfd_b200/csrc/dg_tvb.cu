// TVB limiter pass of the DG path (Cockburn-Shu TVB minmod with characteristic
// decomposition; no reference implementation -- the reference documents this
// design for its DG limiter at src_DG/fluid.h:140-147 but ships a Persson +
// Zhang-Shu limiter instead), the troubled-cell features of the learned
// indicator, and the indicator-gated variant.
//
// One thread per cell, in place on the stage output: a cell reads its own
// linear modes and the MEANS of its four neighbours (through the ghost map);
// means are never modified, so the sweep is race-free in place.  Compiled with
// --fmad=false: the FP64 instantiation is bit-identical to the oracle's C
// restatement (oracle/dg_oracle.c: limit_tvb_all).
//
// The indicator's features (zk_mlp.h) take the cell's modes from the stage
// output and the means from the stage INPUT, the same values the fused
// mixed-precision stage kernel has in its tile (dg_mixed.cu).  List mode
// (tvb_list_kernel) limits only the cells the fused indicator listed.
#include <cuda_bf16.h>

#include "dg_common.cuh"
#include "f32x2.cuh"
#include "zk_internal.h"
#include "zk_mlp.h"

namespace zk {
namespace {

template <typename T>
__device__ __forceinline__ T tmin_(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T tmax_(T a, T b) { return (a < b) ? b : a; }

template <typename T>
__device__ __forceinline__ T tvb_minmod(T a, T b, T c, T mh2) {
    if (fabs(a) <= mh2) return a;
    if (a > T(0) && b > T(0) && c > T(0)) return tmin_(a, tmin_(b, c));
    if (a < T(0) && b < T(0) && c < T(0)) return tmax_(a, tmax_(b, c));
    return T(0);
}

// Euler eigenvectors in direction dir at conserved state u (oracle:
// od_euler_eigen); false for a non-physical state.
template <typename T>
__device__ __forceinline__ bool euler_eigen(const T u[4], T gamma, int dir, T L[4][4], T R[4][4]) {
    const T rho = u[0];
    if (!(rho > T(0))) return false;
    const T vx = u[1] / rho, vy = u[2] / rho;
    const T q2 = vx * vx + vy * vy;
    const T p = (gamma - T(1)) * (u[3] - T(0.5) * rho * q2);
    if (!(p > T(0))) return false;
    const T c = sqrt(gamma * p / rho);
    const T H = (u[3] + p) / rho;
    const T b1 = (gamma - T(1)) / (c * c), b2 = T(0.5) * q2 * b1;
    const T un = dir == 0 ? vx : vy, ut = dir == 0 ? vy : vx;
    const int in = dir == 0 ? 1 : 2, it = dir == 0 ? 2 : 1;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < 4; ++k) L[r][k] = R[r][k] = T(0);
    R[0][0] = T(1); R[in][0] = un - c; R[it][0] = ut; R[3][0] = H - un * c;
    R[0][1] = T(1); R[in][1] = un;     R[it][1] = ut; R[3][1] = T(0.5) * q2;
    R[0][2] = T(0); R[in][2] = T(0);   R[it][2] = T(1); R[3][2] = ut;
    R[0][3] = T(1); R[in][3] = un + c; R[it][3] = ut; R[3][3] = H + un * c;
    L[0][0] = T(0.5) * (b2 + un / c); L[0][in] = -T(0.5) * (b1 * un + T(1) / c); L[0][it] = -T(0.5) * b1 * ut; L[0][3] = T(0.5) * b1;
    L[1][0] = T(1) - b2;              L[1][in] = b1 * un;                        L[1][it] = b1 * ut;             L[1][3] = -b1;
    L[2][0] = -ut;                    L[2][in] = T(0);                           L[2][it] = T(1);                L[2][3] = T(0);
    L[3][0] = T(0.5) * (b2 - un / c); L[3][in] = -T(0.5) * (b1 * un - T(1) / c); L[3][it] = -T(0.5) * b1 * ut; L[3][3] = T(0.5) * b1;
    return true;
}

template <typename T>
__device__ __forceinline__ bool tvb_dir(const T ub[4], T gamma, int dir, T mh2, const T a[4], const T dp[4],
                                        const T dm[4], T out[4]) {
    T L[4][4], R[4][4];
    const bool phys = euler_eigen<T>(ub, gamma, dir, L, R);
    T w[4], wl[4];
    bool changed = false;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T wp, wm;
        if (phys) {
            w[r] = L[r][0] * a[0] + L[r][1] * a[1] + L[r][2] * a[2] + L[r][3] * a[3];
            wp = L[r][0] * dp[0] + L[r][1] * dp[1] + L[r][2] * dp[2] + L[r][3] * dp[3];
            wm = L[r][0] * dm[0] + L[r][1] * dm[1] + L[r][2] * dm[2] + L[r][3] * dm[3];
        } else {
            w[r] = a[r]; wp = dp[r]; wm = dm[r];
        }
        wl[r] = tvb_minmod<T>(w[r], wp, wm, mh2);
        if (wl[r] != w[r]) changed = true;
    }
    if (!changed) return false;
#pragma unroll
    for (int r = 0; r < 4; ++r)
        out[r] = phys ? R[r][0] * wl[0] + R[r][1] * wl[1] + R[r][2] * wl[2] + R[r][3] * wl[3] : wl[r];
    return true;
}

// Mean of the cell at k, gathered through the fill map.
template <typename T>
__device__ __forceinline__ void nb_mean(const T* d, const int8_t* kind, const int32_t* gsrc, size_t k, size_t vs,
                                        T out[4]) {
    const int8_t kd = kind[k] & KIND_MASK;
    size_t s = k;
    int neg = -1;
    if (kd >= KIND_COPY) {
        s = (size_t)gsrc[k];
        neg = kd == KIND_SLIP_X ? 1 : (kd == KIND_SLIP_Y ? 2 : -1);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const T v = d[(size_t)c * vs + s];
        out[c] = (neg == c) ? -v : v;
    }
}

struct TvbArgs {
    void* state;       // T planes [4][NM][ny][pitch]
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double da, gamma, M;
    uint8_t* flags;    // per cell (pitched), may be null
    const MlpPacked* mlp;  // non-null: only cells the indicator flags are limited
    float* features;   // features mode: [ncell][40] output, no limiting
    uint32_t* nflag;   // count of limited cells, may be null
    float* logits;     // with mlp: per-cell logit output [ny*nx], no limiting
    const void* means; // stage input whose means feed the features (null: the state itself)
    int means_fp64;    // means is double (else float)
    const int32_t* list;    // list mode: pitched cell indices to limit ...
    const uint32_t* count;  // ... and their number
    float screen;      // gated: cells within this of a constant state's features are smooth (< 0: none)
};

__device__ __forceinline__ float load_mean(const void* p, int fp64, size_t i) {
    return fp64 ? (float)static_cast<const double*>(p)[i] : static_cast<const float*>(p)[i];
}

// Mean of (rho, E) of the cell at k of the features' means source, through
// the fill map (a slip wall negates only momentum, so rho and E copy).
__device__ __forceinline__ void nb_mean_re(const TvbArgs& a, size_t k, size_t vs, float& rho, float& E) {
    const int8_t kd = a.kind[k] & KIND_MASK;
    const size_t s = kd >= KIND_COPY ? (size_t)a.gsrc[k] : k;
    rho = load_mean(a.means, a.means_fp64, s);
    E = load_mean(a.means, a.means_fp64, 3 * vs + s);
}

// ---- indicator inference on the tensor cores --------------------------------------
// One warp evaluates the MLP for its 32 cells with mma.sync m16n8k16 BF16
// (FP32 accumulation): M = 32 cells (2 tiles), K = 48 (40 features, zero
// padded) then 32, N = 32 hidden units (4 tiles).  A layer's accumulator tiles
// are re-packed in registers as the next layer's A operand.
constexpr int KP = MLP_KP1;  // row stride (bf16) of the per-warp feature tile

struct MlpSmem {
    MlpPacked w;
    uint16_t f[4][32][KP];  // per-warp feature tiles
    float logit[4][32];
};

// Two floats rounded to nearest BF16 and packed, lo in the low half (one
// cvt.rn.bf16x2.f32 instead of two conversions, a shift and an or).
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&p);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ void stage_mlp_weights(MlpSmem& S, const MlpPacked& W) {
    const uint4* src = reinterpret_cast<const uint4*>(&W);
    uint4* dst = reinterpret_cast<uint4*>(&S.w);
    for (int e = threadIdx.x; e < (int)(sizeof(MlpPacked) / 16); e += blockDim.x) dst[e] = src[e];
}

// gelu_fast on the two lanes of a pair (packed .f32x2 arithmetic, explicit
// fused multiply-adds whatever this file's contraction flags; tanh per lane):
// u = K (x + C x^3), 0.5 x (1 + tanh u).
__device__ __forceinline__ float2 gelu2(float2 x) {
    const float2 u = mul2(f2(GELU_K), fma2(mul2(f2(GELU_C), mul2(x, x)), x, x));
    float t0, t1;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(u.x));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(u.y));
    const float2 hx = mul2(f2(0.5f), x);
    return fma2(hx, make_float2(t0, t1), hx);
}

// Hidden layer: acc[mt][nt][4] = A (from a-fragments) x W^T, + bias, GELU.
template <int KSTEPS>
__device__ __forceinline__ void mlp_layer(const uint32_t (&a)[2][KSTEPS][4], const uint16_t* w, int wstride,
                                          const float* bias, float (&h)[2][4][4], int lane) {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) h[mt][nt][e] = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const uint16_t* wr = w + (nt * 8 + g) * wstride;
#pragma unroll
        for (int kt = 0; kt < KSTEPS; ++kt) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + kt * 16 + 2 * q);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + kt * 16 + 8 + 2 * q);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma_bf16(h[mt][nt], a[mt][kt][0], a[mt][kt][1], a[mt][kt][2], a[mt][kt][3], b0, b1);
        }
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const float2 b = make_float2(bias[nt * 8 + 2 * q], bias[nt * 8 + 2 * q + 1]);  // columns 2q, 2q + 1
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const float2 lo = gelu2(add2(make_float2(h[mt][nt][0], h[mt][nt][1]), b));
            const float2 hi = gelu2(add2(make_float2(h[mt][nt][2], h[mt][nt][3]), b));
            h[mt][nt][0] = lo.x;
            h[mt][nt][1] = lo.y;
            h[mt][nt][2] = hi.x;
            h[mt][nt][3] = hi.y;
        }
    }
}

// Accumulator tiles (m16n8, 4 of them along N) -> A fragments (m16k16, 2 k steps).
__device__ __forceinline__ void repack(const float (&h)[2][4][4], uint32_t (&a)[2][2][4]) {
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            a[mt][kt][0] = pack2(h[mt][2 * kt][0], h[mt][2 * kt][1]);
            a[mt][kt][1] = pack2(h[mt][2 * kt][2], h[mt][2 * kt][3]);
            a[mt][kt][2] = pack2(h[mt][2 * kt + 1][0], h[mt][2 * kt + 1][1]);
            a[mt][kt][3] = pack2(h[mt][2 * kt + 1][2], h[mt][2 * kt + 1][3]);
        }
}

// Logit of this lane's cell; every lane of the warp must call it.
__device__ float mlp_logit_mma(MlpSmem& S, int warp, int lane, const float (&f)[MLP_IN]) {
    uint16_t* row = S.f[warp][lane];
#pragma unroll
    for (int i = 0; i < MLP_IN; i += 2) *reinterpret_cast<uint32_t*>(row + i) = pack2(f[i], f[i + 1]);
#pragma unroll
    for (int i = MLP_IN; i < 48; i += 2) *reinterpret_cast<uint32_t*>(row + i) = 0u;
    __syncwarp();
    const int g = lane >> 2, q = lane & 3;
    uint32_t a1[2][3][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kt = 0; kt < 3; ++kt) {
            const uint16_t* r0 = S.f[warp][mt * 16 + g] + kt * 16 + 2 * q;
            const uint16_t* r1 = S.f[warp][mt * 16 + g + 8] + kt * 16 + 2 * q;
            a1[mt][kt][0] = *reinterpret_cast<const uint32_t*>(r0);
            a1[mt][kt][1] = *reinterpret_cast<const uint32_t*>(r1);
            a1[mt][kt][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
            a1[mt][kt][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
        }
    float h[2][4][4];
    uint32_t a[2][2][4];
    mlp_layer<3>(a1, &S.w.w1[0][0], MLP_KP1, S.w.b1, h, lane);
    repack(h, a);
    mlp_layer<2>(a, &S.w.w2[0][0], MLP_KP2, S.w.b2, h, lane);
    repack(h, a);
    mlp_layer<2>(a, &S.w.w3[0][0], MLP_KP2, S.w.b3, h, lane);
    // output unit: per row, sum over this lane's 8 columns, then over the quad
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        float lo = 0.0f, hi = 0.0f;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const float w0 = S.w.w4[nt * 8 + 2 * q], w1 = S.w.w4[nt * 8 + 2 * q + 1];
            lo = fmaf(w0, h[mt][nt][0], fmaf(w1, h[mt][nt][1], lo));
            hi = fmaf(w0, h[mt][nt][2], fmaf(w1, h[mt][nt][3], hi));
        }
        lo += __shfl_xor_sync(0xffffffffu, lo, 1);
        lo += __shfl_xor_sync(0xffffffffu, lo, 2);
        hi += __shfl_xor_sync(0xffffffffu, hi, 1);
        hi += __shfl_xor_sync(0xffffffffu, hi, 2);
        if (q == 0) {
            S.logit[warp][mt * 16 + g] = lo + S.w.b4;
            S.logit[warp][mt * 16 + g + 8] = hi + S.w.b4;
        }
    }
    __syncwarp();
    return S.logit[warp][lane];
}

constexpr int kTvbRows = 1;  // rows per CTA

template <typename T, int P>
__device__ __forceinline__ void tvb_cell(const TvbArgs& a, MlpSmem& S, bool gated, int i, int j);
template <typename T, int P>
__device__ __forceinline__ void tvb_limit(const TvbArgs& a, size_t k, const T (&ub)[4], const T (&uL)[4],
                                          const T (&uR)[4], const T (&uU)[4], const T (&uD)[4]);

// 6 CTAs per SM (80 registers, some spilled): the pass is latency-bound, and
// the extra resident warps beat the 4 CTAs that 110 registers allowed (+1.9%
// on the gated P=3 mixed step; 8 CTAs at 64 registers slowed the FP64 pass).
template <typename T, int P>
__global__ void __launch_bounds__(128, 6) tvb_kernel(TvbArgs a) {
    __shared__ __align__(16) MlpSmem S;
    const bool gated = a.mlp != nullptr;  // uniform over the grid
    if (gated) {
        stage_mlp_weights(S, *a.mlp);
        __syncthreads();
    }
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    for (int r = 0; r < kTvbRows; ++r) tvb_cell<T, P>(a, S, gated, blockIdx.y * kTvbRows + r, j);
}

template <typename T, int P>
__device__ __forceinline__ void tvb_cell(const TvbArgs& a, MlpSmem& S, bool gated, int i, int j) {
    constexpr int NM = (P + 1) * (P + 1);
    const bool inside = j < a.g.nx && i < a.g.ny;
    const size_t k = inside ? (size_t)i * a.g.pitch + j : 0;
    const size_t plane = a.g.plane, vs = (size_t)NM * plane;
    T* d = static_cast<T*>(a.state);
    if (inside && a.flags) a.flags[k] = 0;
    const bool active = inside && (a.kind[k] & KIND_MASK) == KIND_UPDATED;
    if (!gated && !active) return;  // ungated: no warp-wide work follows
    T ub[4] = {T(0), T(0), T(0), T(0)}, uL[4] = {T(0), T(0), T(0), T(0)}, uR[4] = {T(0), T(0), T(0), T(0)},
      uU[4] = {T(0), T(0), T(0), T(0)}, uD[4] = {T(0), T(0), T(0), T(0)};
    if (active) {
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[c] = d[(size_t)c * vs + k];
        nb_mean<T>(d, a.kind, a.gsrc, k - 1, vs, uL);
        nb_mean<T>(d, a.kind, a.gsrc, k + 1, vs, uR);
        nb_mean<T>(d, a.kind, a.gsrc, k - (size_t)a.g.pitch, vs, uU);
        nb_mean<T>(d, a.kind, a.gsrc, k + (size_t)a.g.pitch, vs, uD);
    }
    if (a.features || gated) {
        float f[MLP_IN];
#pragma unroll
        for (int s = 0; s < MLP_IN; ++s) f[s] = 0.0f;
        if (active) {
            // means of the stage input (own, L, R, U, D) for rho and E
            float mr[5], me[5];
            if (a.means) {
                const size_t ks[5] = {k, k - 1, k + 1, k - (size_t)a.g.pitch, k + (size_t)a.g.pitch};
#pragma unroll
                for (int n = 0; n < 5; ++n) nb_mean_re(a, ks[n], vs, mr[n], me[n]);
            } else {
                const T* src[5] = {ub, uL, uR, uU, uD};
#pragma unroll
                for (int n = 0; n < 5; ++n) {
                    mr[n] = (float)src[n][0];
                    me[n] = (float)src[n][3];
                }
            }
            // rho and E modes of the output, slot px*4+py, scaled by the
            // largest |mean| around; neighbour-mean differences
            const float sr = fmaxf(fmaxf(fmaxf(fabsf(mr[0]), fabsf(mr[1])), fmaxf(fabsf(mr[2]), fabsf(mr[3]))),
                                   fabsf(mr[4])) + 1e-12f;
            const float se = fmaxf(fmaxf(fmaxf(fabsf(me[0]), fabsf(me[1])), fmaxf(fabsf(me[2]), fabsf(me[3]))),
                                   fabsf(me[4])) + 1e-12f;
            const float ir = 1.0f / sr, ie = 1.0f / se;
#pragma unroll
            for (int m = 0; m < NM; ++m) {
                const int slot = (m / (P + 1)) * 4 + m % (P + 1);
                f[slot] = (float)d[(size_t)m * plane + k] * ir;
                f[16 + slot] = (float)d[3 * vs + (size_t)m * plane + k] * ie;
            }
            f[0] -= 1.0f;  // the scaled means, centred: a constant state's features are 0
            f[16] -= 1.0f;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                f[32 + n] = (mr[1 + n] - mr[0]) * ir;
                f[36 + n] = (me[1 + n] - me[0]) * ie;
            }
        }
        if (a.features) {
            if (active) {
                const size_t cell = (size_t)i * a.g.nx + j;
#pragma unroll
                for (int s = 0; s < MLP_IN; ++s) a.features[cell * MLP_IN + s] = f[s];
            }
        } else {
            // the screen of the fused indicator (dg_mixed.cu): features within
            // `screen` of a constant state's are smooth; a warp of smooth cells
            // skips the network
            float dev = 0.0f;
#pragma unroll
            for (int s = 0; s < MLP_IN; ++s) dev = fmaxf(dev, fabsf(f[s]));
            const bool cand = active && !(dev <= a.screen);
            float z = -INFINITY;
            if (__any_sync(0xffffffffu, cand)) {
                const float zz = mlp_logit_mma(S, threadIdx.x >> 5, threadIdx.x & 31, f);
                if (cand) z = zz;
            }
            if (a.logits) {
                if (active) a.logits[(size_t)i * a.g.nx + j] = z;
                return;
            }
            if (!(z > 0.0f)) return;  // indicator says smooth: skip the characteristic branch
        }
    }
    if (!active) return;
    tvb_limit<T, P>(a, k, ub, uL, uR, uU, uD);
}

// The TVB test of one updated cell (own mean ub, neighbour means) and, when
// it fires, the characteristic limiting of its modes in place.
template <typename T, int P>
__device__ __forceinline__ void tvb_limit(const TvbArgs& a, size_t k, const T (&ub)[4], const T (&uL)[4],
                                          const T (&uR)[4], const T (&uU)[4], const T (&uD)[4]) {
    constexpr int NM = (P + 1) * (P + 1);
    const size_t plane = a.g.plane, vs = (size_t)NM * plane;
    T* d = static_cast<T*>(a.state);
    const T mh2 = T(a.M) * T(a.da) * T(a.da);
    T ax[4], ay[4], dxp[4], dxm[4], dyp[4], dym[4], lx[4], ly[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        ax[c] = d[(size_t)c * vs + (size_t)(P + 1) * plane + k];
        ay[c] = d[(size_t)c * vs + plane + k];
        dxp[c] = uR[c] - ub[c];
        dxm[c] = ub[c] - uL[c];
        dyp[c] = uD[c] - ub[c];  // eta grows with the row index
        dym[c] = ub[c] - uU[c];
    }
    const bool tx = tvb_dir<T>(ub, T(a.gamma), 0, mh2, ax, dxp, dxm, lx);
    const bool ty = tvb_dir<T>(ub, T(a.gamma), 1, mh2, ay, dyp, dym, ly);
    if (!(tx || ty)) return;
    if (a.flags) a.flags[k] = 1;
    if (a.features) return;  // features mode labels only
    if (a.nflag) atomicAdd(a.nflag, 1u);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (tx) d[(size_t)c * vs + (size_t)(P + 1) * plane + k] = lx[c];
        if (ty) d[(size_t)c * vs + plane + k] = ly[c];
#pragma unroll
        for (int m = 0; m < NM; ++m)
            if (m / (P + 1) + m % (P + 1) > 1) d[(size_t)c * vs + (size_t)m * plane + k] = T(0);
    }
}

// List mode: the cells the fused indicator of the mixed stage kernel flagged
// (pitched indices list[0 .. *count)), each through tvb_limit on the stage
// output; a grid-stride loop over the device-side count.
template <typename T, int P>
__global__ void __launch_bounds__(128) tvb_list_kernel(TvbArgs a) {
    constexpr int NM = (P + 1) * (P + 1);
    const size_t vs = (size_t)NM * a.g.plane;
    const T* d = static_cast<const T*>(a.state);
    const uint32_t n = *a.count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const size_t k = (size_t)a.list[t];
        if (a.flags) a.flags[k] = 0;
        T ub[4], uL[4], uR[4], uU[4], uD[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[c] = d[(size_t)c * vs + k];
        nb_mean<T>(d, a.kind, a.gsrc, k - 1, vs, uL);
        nb_mean<T>(d, a.kind, a.gsrc, k + 1, vs, uR);
        nb_mean<T>(d, a.kind, a.gsrc, k - (size_t)a.g.pitch, vs, uU);
        nb_mean<T>(d, a.kind, a.gsrc, k + (size_t)a.g.pitch, vs, uD);
        tvb_limit<T, P>(a, k, ub, uL, uR, uU, uD);
    }
}

template <typename T>
cudaError_t launch_list_t(int P, const TvbArgs& a, int grid, cudaStream_t s) {
    switch (P) {
        case 1: tvb_list_kernel<T, 1><<<grid, 128, 0, s>>>(a); break;
        case 2: tvb_list_kernel<T, 2><<<grid, 128, 0, s>>>(a); break;
        case 3: tvb_list_kernel<T, 3><<<grid, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_t(int P, const TvbArgs& a, cudaStream_t s) {
    dim3 grid((a.g.nx + 127) / 128, (a.g.ny + kTvbRows - 1) / kTvbRows);
    switch (P) {
        case 1: tvb_kernel<T, 1><<<grid, 128, 0, s>>>(a); break;
        case 2: tvb_kernel<T, 2><<<grid, 128, 0, s>>>(a); break;
        case 3: tvb_kernel<T, 3><<<grid, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dg_tvb(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                          double da, double gamma, double M, uint8_t* flags, const MlpPacked* mlp,
                          float* features, uint32_t* nflag, float* logits, const void* means, bool means_fp64,
                          float screen, cudaStream_t s) {
    TvbArgs a{state, kind, gsrc, g, da, gamma, M, flags, mlp, features, nflag, logits, means, means_fp64 ? 1 : 0,
              nullptr, nullptr, screen};
    return fp64 ? launch_t<double>(P, a, s) : launch_t<float>(P, a, s);
}

// TVB limiting of the listed cells only (list mode), `grid` CTAs of 128 threads.
cudaError_t launch_dg_tvb_list(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                               double da, double gamma, double M, uint8_t* flags, uint32_t* nflag,
                               const int32_t* list, const uint32_t* count, int grid, cudaStream_t s) {
    TvbArgs a{state, kind, gsrc, g, da, gamma, M, flags, nullptr, nullptr, nflag, nullptr, nullptr, 0, list, count,
              -1.0f};
    return fp64 ? launch_list_t<double>(P, a, grid, s) : launch_list_t<float>(P, a, grid, s);
}

}  // namespace zk
