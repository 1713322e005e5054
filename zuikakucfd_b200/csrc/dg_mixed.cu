// DG P=1..3 stage, mixed precision, ONE fused kernel per RK stage.
//
// A CTA owns a 32 x 4 tile of cells.  It gathers the tile plus a 1-cell halo
// of the stage input into shared memory as FP32 (ghosts through the fill
// source map, slip walls negated), computes every interface flux of the tile
// once from the two cells' traces (FP32, in shared memory), then runs each
// cell's volume quadrature and face integrals in FP32 registers, with one
// thread per cell (stage_tile) or two, each owning a pair of the conserved
// variables (stage_tile_pair).  The Shu-Osher combine is FP64 against the
// FP64 U^n; the Persson + Zhang-Shu limiter decides in FP32 and is applied as
// per-mode factors.  Stage states U^(1), U^(2) are stored in FP32; U^(n+1) is
// written in FP64 by the combine, and the limiter rewrites the modes it
// changes.  This file is compiled with --use_fast_math (FP32 division, sqrt,
// log10 and sin use the MUFU approximations); the combine and limiter
// arithmetic is rounded explicitly, so both kernels give the same bits.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>

#include <type_traits>

#include "batch.cuh"
#include "dg_common.cuh"
#include "mlp_infer.cuh"
#include "zk_internal.h"

namespace zk {
namespace {

struct DGTabF {
    float vw[DG_MAXNQ * DG_MAXNQ];
    float vphi[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];
    float vdxi[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];
    float vdet[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];
    float tr[4][DG_MAXNQ][DG_MAXNM];
    float bv[4][DG_MAXNQ][DG_MAXNM];
    float zs[16][DG_MAXNM];
};

__constant__ DGTabF c_tabf[3];

// FP32 one-dimensional basis factors (DGSep) for the sum-factorised
// transforms; WL[n][q] = w_q P_n(x_q).
struct DGSepF {
    float L[DG_MAXNQ][DG_MAXNQ];
    float D[DG_MAXNQ][DG_MAXNQ];
    float W[DG_MAXNQ];
    float WL[DG_MAXNQ][DG_MAXNQ];
    float Z[DG_MAXNQ][4];
};
__constant__ DGSepF c_sepf[3];

// A tile is 32 x MTY cells with one thread per cell; shared memory holds the
// tile plus a 1-cell halo (SX x (MTY + 2) slots).
constexpr int MTX = 32, SX = MTX + 2;
// U^n values a thread loads together in the combine of a stage with an FP64
// output (U^(n+1) written over U^n)
constexpr int kUnChunk = 8;

struct MixArgs {
    const void* cur;  // stage input: double (stage 1: U^n) or float (U^(1), U^(2))
    const double* un;
    void* out;        // float (stages 1, 2) or double (stage 3)
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double dt;
    float inv2h, gamma;
    int stage, limiter, hll;
    float s0;
    uint32_t* status;
    const double* phic;  // basis at the 4 cell corners [NM][4] (LAM kernels only)
    double gamma64;      // gamma in FP64 (LAM kernels only)
    // learned troubled-cell indicator fused into the stage (MLP kernels only):
    // weights, the list the flagged cells are appended to, its count and capacity
    const MlpFrag* mlp;
    int32_t* list;
    uint32_t* count;
    uint32_t cap;
    float* dbg;  // non-null: per updated cell k, dbg[k*41 ..] = the 40 features and the logit
    float screen;  // cells whose features deviate from a constant state's by <= screen skip the network
};

__device__ __forceinline__ float fmaxr(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float fminr(float a, float b) { return (b < a) ? b : a; }

// eulerFluxX/Y (src_DG/fluid.cpp:123-143), FP32
__device__ __forceinline__ void euler_flux_f(const float U[4], float gam, float F[4], float G[4]) {
    const float eps = 1e-3f;
    float rho = fmaxr(U[0], eps);
    float ir = 1.0f / rho;
    float u = U[1] * ir, v = U[2] * ir;
    float p = fmaxr((gam - 1.0f) * (U[3] - 0.5f * rho * (u * u + v * v)), eps);
    F[0] = rho * u; F[1] = rho * u * u + p; F[2] = rho * u * v; F[3] = (U[3] + p) * u;
    G[0] = rho * v; G[1] = rho * u * v; G[2] = rho * v * v + p; G[3] = (U[3] + p) * v;
}

// hllcFlux DG variant (src_DG/fluid.cpp:450-520), FP32
__device__ __forceinline__ void hllc_dg_f(const float L[4], const float R[4], float gamma, float F[4]) {
    const float eps = 1e-5f;
    float rhoL = fmaxr(L[0], eps), irL = 1.0f / rhoL, uL = L[1] * irL, vL = L[2] * irL;
    float pL = fmaxr((gamma - 1.0f) * (L[3] - 0.5f * rhoL * (uL * uL + vL * vL)), eps);
    float aL = sqrtf(fmaxr(gamma * pL * irL, eps));
    float rhoR = fmaxr(R[0], eps), irR = 1.0f / rhoR, uR = R[1] * irR, vR = R[2] * irR;
    float pR = fmaxr((gamma - 1.0f) * (R[3] - 0.5f * rhoR * (uR * uR + vR * vR)), eps);
    float aR = sqrtf(fmaxr(gamma * pR * irR, eps));
    float sqL = sqrtf(rhoL), sqR = sqrtf(rhoR);
    float den = sqL + sqR;
    if (den < eps) den = eps;
    float iden = 1.0f / den;
    float u_roe = (sqL * uL + sqR * uR) * iden;
    float h_roe = (sqL * ((L[3] + pL) * irL) + sqR * ((R[3] + pR) * irR)) * iden;
    float c_roe = sqrtf(fmaxr((gamma - 1.0f) * (h_roe - 0.5f * u_roe * u_roe), eps));
    float SL = fminr(uL - aL, u_roe - c_roe);
    float SR = fmaxr(uR + aR, u_roe + c_roe);
    if (SL >= 0.0f) {
        F[0] = rhoL * uL; F[1] = rhoL * uL * uL + pL; F[2] = rhoL * uL * vL; F[3] = (L[3] + pL) * uL;
        return;
    }
    if (SR <= 0.0f) {
        F[0] = rhoR * uR; F[1] = rhoR * uR * uR + pR; F[2] = rhoR * uR * vR; F[3] = (R[3] + pR) * uR;
        return;
    }
    float num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    float den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabsf(den2) < eps) den2 = (den2 >= 0.0f ? eps : -eps);
    float Ss = num / den2;
    const bool left = Ss >= 0.0f;
    const float rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const float p = left ? pL : pR, S = left ? SL : SR, ir = left ? irL : irR;
    const float* Us = left ? L : R;
    float denom = S - Ss;
    if (fabsf(denom) < eps) denom = (denom >= 0.0f ? eps : -eps);
    float c = rho * (S - u) / denom;
    float term = (Ss - u) * (Ss + p / (rho * (S - u)));
    if (!isfinite(term)) term = 0.0f;
    F[0] = rho * u + S * (c - Us[0]);
    F[1] = rho * u * u + p + S * (c * Ss - Us[1]);
    F[2] = rho * u * v + S * (c * v - Us[2]);
    F[3] = (Us[3] + p) * u + S * (c * (Us[3] * ir + term) - Us[3]);
}

// hlleFlux (src_DG/fluid.cpp:525-580), FP32
__device__ __forceinline__ void hlle_dg_f(const float L[4], const float R[4], float gamma, float F[4]) {
    const float eps = 1e-6f;
    float rhoL = fmaxr(L[0], eps), irL = 1.0f / rhoL, uL = L[1] * irL, vL = L[2] * irL, EL = L[3];
    float pL = fmaxr((gamma - 1.0f) * (EL - 0.5f * rhoL * (uL * uL + vL * vL)), eps);
    float aL = sqrtf(fmaxr(gamma * pL * irL, eps));
    float rhoR = fmaxr(R[0], eps), irR = 1.0f / rhoR, uR = R[1] * irR, vR = R[2] * irR, ER = R[3];
    float pR = fmaxr((gamma - 1.0f) * (ER - 0.5f * rhoR * (uR * uR + vR * vR)), eps);
    float aR = sqrtf(fmaxr(gamma * pR * irR, eps));
    float sqL = sqrtf(rhoL), sqR = sqrtf(rhoR);
    float invDen = 1.0f / fmaxr(sqL + sqR, eps);
    float u_roe = (sqL * uL + sqR * uR) * invDen, v_roe = (sqL * vL + sqR * vR) * invDen;
    float h_roe = (sqL * ((EL + pL) * irL) + sqR * ((ER + pR) * irR)) * invDen;
    float c_roe = sqrtf(fmaxr((gamma - 1.0f) * (h_roe - 0.5f * (u_roe * u_roe + v_roe * v_roe)), eps));
    float SL = fminr(uL - aL, u_roe - c_roe), SR = fmaxr(uR + aR, u_roe + c_roe);
    float FL[4] = {rhoL * uL, rhoL * uL * uL + pL, rhoL * uL * vL, (EL + pL) * uL};
    float FR[4] = {rhoR * uR, rhoR * uR * uR + pR, rhoR * uR * vR, (ER + pR) * uR};
    if (SL >= 0.0f) {
        for (int c = 0; c < 4; ++c) F[c] = FL[c];
    } else if (SR <= 0.0f) {
        for (int c = 0; c < 4; ++c) F[c] = FR[c];
    } else {
        float invDiff = 1.0f / fmaxr(SR - SL, eps);
        for (int c = 0; c < 4; ++c) F[c] = (SR * FL[c] - SL * FR[c] + SL * SR * (R[c] - L[c])) * invDiff;
    }
}

// Combine and limiter arithmetic of the mixed stage, shared by the one- and
// two-thread-per-cell kernels.  Every operation is rounded explicitly (fused
// multiply-adds written as such, nothing left to the compiler's contraction),
// so both kernels produce the same bits.
// Shu-Osher stages 2 and 3 in FP64: 3/4 un + 1/4 w, 1/3 un + 2/3 w (one
// fused multiply-add each).
__device__ __forceinline__ double so_combine(int stage, double un, double w) {
    return stage == 2 ? __fma_rn(0.75, un, __dmul_rn(0.25, w)) : __fma_rn(1.0 / 3.0, un, __dmul_rn(2.0 / 3.0, w));
}
// |m|^2 / 2 rho
__device__ __forceinline__ float half_m2_over_rho(float rho, float mx, float my) {
    return __fdividef(__fmul_rn(0.5f, __fmaf_rn(mx, mx, __fmul_rn(my, my))), rho);
}
// (gamma - 1)(E - |m|^2 / 2 rho)
__device__ __forceinline__ float pressure_f(float g1, float rho, float mx, float my, float E) {
    return __fmul_rn(g1, __fsub_rn(E, half_m2_over_rho(rho, mx, my)));
}
// Zhang-Shu ratio (avg - lo) / (avg - x + eps)
__device__ __forceinline__ float zs_ratio(float avg, float lo, float x, float eps) {
    return __fdividef(__fsub_rn(avg, lo), __fadd_rn(__fsub_rn(avg, x), eps));
}
// Persson indicator of one variable's modes (src_DG/fluid.cpp:824-870): the
// factor for its highest modes, 1 when the variable is not limited.
template <int P, int NM>
__device__ __forceinline__ float persson_factor(const float (&d)[NM], float s0) {
    constexpr int NQ = P + 1;
    float Et = 0.0f, Ep = 0.0f;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        Et = __fmaf_rn(d[m], d[m], Et);
        if (m / NQ == P || m % NQ == P) Ep = __fmaf_rn(d[m], d[m], Ep);
    }
    const float s = __log10f(__fdividef(Ep, __fadd_rn(Et, 1e-5f)));
    if (!(s > s0)) return 1.0f;
    const float eps = (s > s0 + 1.0f)
                          ? 1.0f
                          : __fmul_rn(0.5f, __fadd_rn(1.0f, __sinf(__fmul_rn(3.14159265f, __fsub_rn(__fsub_rn(s, s0), 0.5f)))));
    return __fsub_rn(1.0f, eps);
}

// Zhang-Shu point values use the modes with px, py < NZ = min(P + 1, 3), and
// every factor is a Legendre value (|P_n| <= 1 on [-1, 1]), so a variable's
// point values stay within its mean +- zs_spread.  A pass whose every point
// provably stays above its floor returns exactly 1 and is skipped.
template <int P, int NM>
__device__ __forceinline__ float zs_spread(const float (&d)[NM]) {
    constexpr int NQ = P + 1, NZ = NQ < 3 ? NQ : 3;
    float s = 0.0f;
#pragma unroll
    for (int px = 0; px < NZ; ++px)
#pragma unroll
        for (int py = 0; py < NZ; ++py)
            if (px || py) s += fabsf(d[px * NQ + py]);
    return s;
}
// every point value of a variable with mean a and spread sp exceeds lo (with a
// 1e-5 relative margin for the rounding of the bound and of the point values)
__device__ __forceinline__ bool zs_above(float a, float sp, float lo) {
    return a - sp - 1e-5f * (fabsf(a) + sp) > lo;
}
// every point pressure exceeds p_min: lower bound (gamma-1)(E_lo - |m|_hi^2 /
// 2 rho_lo) from the four means and spreads, with the same margin
__device__ __forceinline__ bool zs_p_above(const float (&mean)[4], const float (&sp)[4], float g1, float rho_min,
                                           float p_min) {
    const float rlo = mean[0] - sp[0] - 1e-5f * (fabsf(mean[0]) + sp[0]);
    if (!(rlo > rho_min)) return false;
    const float mx = fabsf(mean[1]) + sp[1], my = fabsf(mean[2]) + sp[2];
    const float ke = 0.5f * (mx * mx + my * my) / rlo;
    const float plo = g1 * (mean[3] - sp[3] - ke) - 1e-5f * g1 * (fabsf(mean[3]) + sp[3] + ke);
    return plo > p_min;
}

// Floats per cell slot in shared memory: 4*NM rounded so that (stride/4) is
// odd, which puts 8 consecutive cells' 16-byte loads in 8 distinct bank groups.
__host__ __device__ constexpr int vpitch(int nm) { return ((4 * nm / 4) % 2 == 1) ? 4 * nm : 4 * nm + 4; }

// Plane strides (words) of the interface-flux arrays: x faces MTY rows of
// MTX + 1, y faces MTY + 1 rows of MTX, each padded to 8 (mod 16).  In the
// two-threads-per-cell face integrals a warp reads one plane per half, 2
// planes apart, for 16 consecutive cells: offsets 0, 8 (cells 8-15) and
// 2 stride, 2 stride + 8 (the other half) then fall on 4 distinct groups of 8
// banks (unpadded, 132 and 160 words, two groups shared their banks).
__host__ __device__ constexpr int pad8mod16(int n) { return n + ((8 - n % 16) + 16) % 16; }
__host__ __device__ constexpr int fx_stride(int mty, int tx = MTX) { return pad8mod16(mty * (tx + 1)); }
__host__ __device__ constexpr int fy_stride(int mty, int tx = MTX) { return pad8mod16((mty + 1) * tx); }

template <typename T>
__device__ __forceinline__ float load_f(const void* p, size_t i) {
    return (float)static_cast<const T*>(p)[i];
}

// Every interface flux of a tile once, from the two cells' traces (FP32, in
// shared memory): faces dealt to the NTHREAD threads in turn, each thread the
// whole face (all four variables).  Shared by the one- and two-thread-per-cell
// stages.
template <int P, int MTY, int NTHREAD, int TX = MTX>
__device__ __forceinline__ void tile_face_fluxes(const MixArgs& a, const float* sd, float* sfx, float* sfy,
                                                 const uint8_t* sk, int tid) {
    constexpr int NQ = P + 1, NM = NQ * NQ;
    constexpr int VP = vpitch(NM);
    const DGSepF& S = c_sepf[P - 1];
    constexpr int SXT = TX + 2, NXF = MTY * (TX + 1), NYF = (MTY + 1) * TX;
    for (int f = tid; f < NXF + NYF; f += NTHREAD) {
        int sl, sr, side_l, side_r;
        float* dst;
        int dstride;
        bool ydir;
        if (f < NXF) {
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            sl = (r + 1) * SXT + c;          // left cell slot
            sr = sl + 1;                     // right cell slot
            side_l = 0; side_r = 1;          // xi=+1 of left, xi=-1 of right
            dst = sfx + r * (TX + 1) + c;
            dstride = fx_stride(MTY, TX);
            ydir = false;
        } else {
            const int g = f - NXF, r = g / TX, c = g - r * TX;
            sl = r * SXT + c + 1;             // cell above
            sr = sl + SXT;                    // cell below
            side_l = 2; side_r = 3;          // eta=+1 of upper, eta=-1 of lower
            dst = sfy + r * TX + c;
            dstride = fy_stride(MTY, TX);
            ydir = true;
        }
        if (sk[sl] != KIND_UPDATED && sk[sr] != KIND_UPDATED) continue;
        // Traces by sum factorisation: contract the face-normal index with
        // P_n(+1) = 1 (left/upper cell) and P_n(-1) = (-1)^n (right/lower
        // cell), then evaluate along the face at the NQ Gauss points.
        float el[4][NQ], er[4][NQ];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int n = 0; n < NQ; ++n) el[c][n] = er[c][n] = 0.0f;
        const float* pl = sd + sl * VP;
        const float* pr = sd + sr * VP;
        if (ydir) {
#pragma unroll
            for (int v4 = 0; v4 < 4 * NM; v4 += 4) {
                const float4 l4 = *reinterpret_cast<const float4*>(pl + v4);
                const float4 r4 = *reinterpret_cast<const float4*>(pr + v4);
                const float lv[4] = {l4.x, l4.y, l4.z, l4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int c = (v4 + e) / NM, m = (v4 + e) % NM, px = m / NQ, py = m % NQ;
                    el[c][px] += lv[e];
                    er[c][px] += (py & 1) ? -rv[e] : rv[e];
                }
            }
        } else {
#pragma unroll
            for (int v4 = 0; v4 < 4 * NM; v4 += 4) {
                const float4 l4 = *reinterpret_cast<const float4*>(pl + v4);
                const float4 r4 = *reinterpret_cast<const float4*>(pr + v4);
                const float lv[4] = {l4.x, l4.y, l4.z, l4.w}, rv[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int c = (v4 + e) / NM, m = (v4 + e) % NM, px = m / NQ, py = m % NQ;
                    el[c][py] += lv[e];
                    er[c][py] += (px & 1) ? -rv[e] : rv[e];
                }
            }
        }
        float UL[NQ][4], UR[NQ][4];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float ul = 0.0f, ur = 0.0f;
#pragma unroll
                for (int n = 0; n < NQ; ++n) {
                    ul = fmaf(el[c][n], S.L[n][q], ul);
                    ur = fmaf(er[c][n], S.L[n][q], ur);
                }
                UL[q][c] = ul;
                UR[q][c] = ur;
            }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            float Fq[4];
            if (ydir) {
                float l[4] = {UL[q][0], UL[q][2], UL[q][1], UL[q][3]};
                float r[4] = {UR[q][0], UR[q][2], UR[q][1], UR[q][3]};
                float g[4];
                if (a.hll) hlle_dg_f(l, r, a.gamma, g);
                else hllc_dg_f(l, r, a.gamma, g);
                Fq[0] = g[0]; Fq[1] = g[2]; Fq[2] = g[1]; Fq[3] = g[3];
            } else {
                if (a.hll) hlle_dg_f(UL[q], UR[q], a.gamma, Fq);
                else hllc_dg_f(UL[q], UR[q], a.gamma, Fq);
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) dst[(q * 4 + c) * dstride] = Fq[c];
        }
    }
}

// The tile (top-left cell (i0, j0)) and its 1-cell halo into shared memory,
// ghosts taken from their source cells (slip walls negate the normal
// momentum), slots outside the grid zero; the kind of every slot into sk.
// One slot per thread; the input (FP64 or FP32) goes through registers, all
// of a slot's loads in flight at once (up to 64), four planes per 16-byte
// shared store (a quarter warp's stores, VP words per slot apart, fill
// distinct bank groups).  For FP32 input this takes the P = 3 step from 5.60
// to 5.41 ms against 4-byte asynchronous copies (one slot per thread put 4
// lanes on every bank; 8 slots x 4 planes per warp instruction is
// conflict-free but makes four dependent passes per warp: 5.87 ms), and 16
// loads per batch instead of 8 another 0.05 ms.  The caller synchronises
// after it.
template <int P, typename TIn, int MTY, int NTHREAD, int TX = MTX>
__device__ __forceinline__ void gather_tile(const MixArgs& a, int j0, int i0, float* sd, uint8_t* sk, int tid) {
    constexpr int SXT = TX + 2, NQ = P + 1, NM = NQ * NQ, VP = vpitch(NM), SD = SXT * (MTY + 2);
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;
    for (int slot = tid; slot < SD; slot += NTHREAD) {
        const int r = slot / SXT, c = slot - r * SXT;
        const int gi = i0 - 1 + r, gj = j0 - 1 + c;
        uint8_t kd = KIND_PASSIVE;
        if (gi >= 0 && gi < ny && gj >= 0 && gj < nx) {
            const size_t k = (size_t)gi * pitch + gj;
            kd = a.kind[k] & KIND_MASK;
            size_t ks = k;
            int neg = -1;
            if (kd >= KIND_COPY) {
                ks = (size_t)a.gsrc[k];
                neg = (kd == KIND_SLIP_X) ? 1 : (kd == KIND_SLIP_Y ? 2 : -1);
            }
#pragma unroll 16
            for (int v = 0; v < 4 * NM; v += 4) {
                float4 x;
                x.x = load_f<TIn>(a.cur, (size_t)(v + 0) * plane + ks);
                x.y = load_f<TIn>(a.cur, (size_t)(v + 1) * plane + ks);
                x.z = load_f<TIn>(a.cur, (size_t)(v + 2) * plane + ks);
                x.w = load_f<TIn>(a.cur, (size_t)(v + 3) * plane + ks);
                if (neg == (v + 0) / NM) x.x = -x.x;
                if (neg == (v + 1) / NM) x.y = -x.y;
                if (neg == (v + 2) / NM) x.z = -x.z;
                if (neg == (v + 3) / NM) x.w = -x.w;
                *reinterpret_cast<float4*>(&sd[slot * VP + v]) = x;
            }
        } else {
            for (int v = 0; v < 4 * NM; v += 4)
                *reinterpret_cast<float4*>(&sd[slot * VP + v]) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        sk[slot] = kd;
    }
}

// One tile whose top-left cell is (i0, j0), shared memory at `smem`
// (smem_bytes<P, MTY>()).  Per-thread returns leave only this function: every
// barrier of the tile precedes them.  LAM (FP64 output only): returns the max
// corner wave speed of the thread's cell if it is fluid (computeMaxSpeedDG_omp
// on the FP64 values written), else 0.
template <int P, typename TIn, typename TOut, int MTY, bool LAM = false>
__device__ __forceinline__ double stage_tile(const MixArgs& a, int j0, int i0, float* smem) {
    constexpr int MNT = MTX * MTY, SY = MTY + 2;
    constexpr int NQ = P + 1, NM = NQ * NQ;
    constexpr int SD = SX * SY;  // cell slots of the tile + halo
    constexpr int VP = vpitch(NM);  // floats per slot: 4*NM padded so 16-byte loads are conflict-free
    const DGSepF& S = c_sepf[P - 1];
    float* sd = smem;                       // [SD][VP] gathered stage input, cell-major
    float* sfx = sd + VP * SD;              // [NQ*4][MTY][MTX+1]
    float* sfy = sfx + NQ * 4 * fx_stride(MTY);  // [NQ*4][MTY+1][MTX] at fy_stride per plane
    uint8_t* sk = reinterpret_cast<uint8_t*>(sfy + NQ * 4 * fy_stride(MTY));  // [SY][SX]

    const int tid = threadIdx.x;
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;

    // U^n of this thread's cell is read again only by the combine: start
    // bringing it into L2 now so those loads overlap the flux work
    {
        const int pr = tid / MTX, pc = tid - pr * MTX;
        if (i0 + pr < ny && j0 + pc < nx) {
            const double* u0 = a.un + (size_t)(i0 + pr) * pitch + (j0 + pc);
#pragma unroll 8
            for (int v = 0; v < 4 * NM; ++v)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(u0 + (size_t)v * plane));
        }
    }

    // 0. gather tile + halo (corners unused)
    gather_tile<P, TIn, MTY, MNT>(a, j0, i0, sd, sk, tid);
    __syncthreads();

    // 1. interface fluxes of the tile, once each
    tile_face_fluxes<P, MTY, MNT>(a, sd, sfx, sfy, sk, tid);
    // no barrier yet: the volume quadrature reads only the gathered state, so
    // threads without a last-round face start on it while the last faces finish

    // 2. one thread per cell
    const int r = tid / MTX, c = tid - r * MTX;
    const int gi = i0 + r, gj = j0 + c;
    const bool inside = gi < ny && gj < nx;
    const int slot = (r + 1) * SX + c + 1;
    const size_t k = inside ? (size_t)gi * pitch + gj : 0;
    const uint8_t kd = inside ? sk[slot] : (uint8_t)KIND_PASSIVE;
    float acc[4][NM];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[q][m] = 0.0f;
    if (kd == KIND_UPDATED) {
        const float* pc = sd + slot * VP;
        // volume integral by sum factorisation over the tensor Gauss grid:
        // for each xi-row qa, e = d contracted with P_px(x_qa), U at the NQ
        // points of the row, fluxes, then f = sum_qb w F P_py, g = sum_qb w G P_py',
        // acc += P_px'(x_qa) f + P_px(x_qa) g
#pragma unroll 1
        for (int qa = 0; qa < NQ; ++qa) {
            float e[4][NQ];
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int n = 0; n < NQ; ++n) e[c][n] = 0.0f;
#pragma unroll
            for (int v4 = 0; v4 < 4 * NM; v4 += 4) {
                const float4 d4 = *reinterpret_cast<const float4*>(pc + v4);
                const float dv[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int c = (v4 + u) / NM, m = (v4 + u) % NM;
                    e[c][m % NQ] = fmaf(dv[u], S.L[m / NQ][qa], e[c][m % NQ]);
                }
            }
            float f[4][NQ], g[4][NQ];
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int n = 0; n < NQ; ++n) f[c][n] = g[c][n] = 0.0f;
#pragma unroll
            for (int qb = 0; qb < NQ; ++qb) {
                float U[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    float x = 0.0f;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) x = fmaf(e[c][n], S.L[n][qb], x);
                    U[c] = x;
                }
                float F[4], G[4];
                euler_flux_f(U, a.gamma, F, G);
                const float w = S.W[qa] * S.W[qb];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float Fw = F[c] * w, Gw = G[c] * w;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) {
                        f[c][n] = fmaf(Fw, S.L[n][qb], f[c][n]);
                        g[c][n] = fmaf(Gw, S.D[n][qb], g[c][n]);
                    }
                }
            }
#pragma unroll
            for (int px = 0; px < NQ; ++px) {
                const float dx = S.D[px][qa], lx = S.L[px][qa];
#pragma unroll
                for (int py = 0; py < NQ; ++py)
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        acc[c][px * NQ + py] = fmaf(dx, f[c][py], fmaf(lx, g[c][py], acc[c][px * NQ + py]));
            }
        }
    }
    __syncthreads();  // every interface flux is in shared memory
    if (!inside) return 0.0;
    if (kd == KIND_UPDATED) {
        // face integrals (src_DG/fluid.cpp:731-796): right (-) and left (+) x
        // faces weigh the face-normal factor P_px(+1) = 1 and P_px(-1) =
        // (-1)^px; bottom (-) and top (+) y faces P_py(+-1).  h = sum_q w_q
        // P_n(x_q) F_q along the face.
        {
            const float* Fr = sfx + r * (MTX + 1) + c + 1;
            const float* Fl = sfx + r * (MTX + 1) + c;
            const float* Fd = sfy + (r + 1) * MTX + c;
            const float* Fu = sfy + r * MTX + c;
            constexpr int fsx = fx_stride(MTY), fsy = fy_stride(MTY);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                float hr[NQ], hl[NQ], hd[NQ], hu[NQ];
#pragma unroll
                for (int n = 0; n < NQ; ++n) hr[n] = hl[n] = hd[n] = hu[n] = 0.0f;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const float xr = Fr[(q * 4 + u) * fsx], xl = Fl[(q * 4 + u) * fsx];
                    const float xd = Fd[(q * 4 + u) * fsy], xu = Fu[(q * 4 + u) * fsy];
#pragma unroll
                    for (int n = 0; n < NQ; ++n) {
                        const float wl = S.WL[n][q];
                        hr[n] = fmaf(wl, xr, hr[n]);
                        hl[n] = fmaf(wl, xl, hl[n]);
                        hd[n] = fmaf(wl, xd, hd[n]);
                        hu[n] = fmaf(wl, xu, hu[n]);
                    }
                }
#pragma unroll
                for (int px = 0; px < NQ; ++px)
#pragma unroll
                    for (int py = 0; py < NQ; ++py) {
                        float t = acc[u][px * NQ + py] - hr[py] - hd[px];
                        t += (px & 1) ? -hl[py] : hl[py];
                        t += (py & 1) ? -hu[px] : hu[px];
                        acc[u][px * NQ + py] = t;
                    }
            }
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const float scale = (float)((2 * (m / NQ) + 1) * (2 * (m % NQ) + 1)) * a.inv2h;
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q][m] *= scale;
        }
    }

    if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 4 * NM; ++v) static_cast<TOut*>(a.out)[(size_t)v * plane + k] = (TOut)acc[v / NM][v % NM];
        return 0.0;
    }
    // combine in FP64 (w = cur + dt dU at stages 2, 3); an FP64 output is
    // written here, and the limiter later rewrites only the modes it changes
    const double dt = a.dt;
    const float* pw = sd + slot * VP;
    TOut* out = static_cast<TOut*>(a.out);
    constexpr bool OUT64 = sizeof(TOut) == 8;
    // U^n in chunks loaded before any is combined (as stage_tile_pair: an
    // FP64 output is U^n itself, and each store orders the loads after it);
    // FP32-output chunks of 16 (64 values at once spill at 168 registers)
    constexpr int UC = OUT64 ? kUnChunk : 16;
#pragma unroll
    for (int v0 = 0; v0 < 4 * NM; v0 += UC) {
        double unc[UC];
#pragma unroll
        for (int e = 0; e < UC; ++e)
            if (v0 + e < 4 * NM) unc[e] = a.un[(size_t)(v0 + e) * plane + k];
#pragma unroll
        for (int v4 = v0; v4 < v0 + UC && v4 < 4 * NM; v4 += 4) {
            const float4 c4 = *reinterpret_cast<const float4*>(pw + v4);
            const float cv[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int v = v4 + e, q = v / NM, m = v % NM;
                const double un = unc[v - v0];
                const double du = (double)acc[q][m];
                const double o =
                    a.stage == 1 ? __fma_rn(dt, du, un) : so_combine(a.stage, un, __fma_rn(dt, du, (double)cv[e]));
                acc[q][m] = (float)o;
                if (OUT64) out[(size_t)v * plane + k] = (TOut)o;
            }
        }
    }

    // limiter decisions in FP32 (src_DG/fluid.cpp:824-992), as factors
    float pf[4] = {1.0f, 1.0f, 1.0f, 1.0f};
    float theta = 1.0f;
    bool rho_clamp = false, e_fix = false;
    const bool in_range = gi >= 3 && gi < ny - 3 && gj >= 3 && gj < nx - 3;
    if (a.limiter == ZK_LIMITER_REFERENCE && in_range) {
        if (kd == KIND_UPDATED) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                pf[q] = persson_factor<P, NM>(acc[q], a.s0);
                if (pf[q] != 1.0f) {
#pragma unroll
                    for (int m = 0; m < NM; ++m)
                        if (m / NQ == P || m % NQ == P) acc[q][m] = __fmul_rn(acc[q][m], pf[q]);
                }
            }
        }
        const float RHO_MIN = 1e-5f, P_MIN = 1e-5f, EPS = 1e-5f, g1 = a.gamma - 1.0f;
        if (acc[0][0] < RHO_MIN) { acc[0][0] = RHO_MIN; rho_clamp = true; }
        const float rho0 = acc[0][0], mx0 = acc[1][0], my0 = acc[2][0];
        const float ke0 = half_m2_over_rho(rho0, mx0, my0);
        if (__fmul_rn(g1, __fsub_rn(acc[3][0], ke0)) < P_MIN) { acc[3][0] = __fadd_rn(__fdividef(P_MIN, g1), ke0); e_fix = true; }
        // Zhang-Shu points (4 x 4 Gauss grid, cubic factors zero): separable
        // evaluation, first over px at node a, then over py at node b
        constexpr int NZ = NQ < 3 ? NQ : 3;
        float th = 1.0f;
        const bool rho_pass = !zs_above(rho0, zs_spread<P, NM>(acc[0]), RHO_MIN);
#pragma unroll 1
        for (int za = 0; za < (rho_pass ? 4 : 0); ++za) {
            float t[NZ];
#pragma unroll
            for (int py = 0; py < NZ; ++py) {
                float x = 0.0f;
#pragma unroll
                for (int px = 0; px < NZ; ++px) x = fmaf(acc[0][px * NQ + py], S.Z[px][za], x);
                t[py] = x;
            }
#pragma unroll
            for (int zb = 0; zb < 4; ++zb) {
                float rho = 0.0f;
#pragma unroll
                for (int py = 0; py < NZ; ++py) rho = fmaf(t[py], S.Z[py][zb], rho);
                if (rho < RHO_MIN) th = fminr(th, zs_ratio(rho0, RHO_MIN, rho, EPS));
            }
        }
        if (th < 1.0f) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q][m] = __fmul_rn(acc[q][m], th);
        }
        const float p_avg = pressure_f(g1, acc[0][0], acc[1][0], acc[2][0], acc[3][0]);
        float tp = 1.0f;
        bool p_pass;
        {
            const float mean[4] = {acc[0][0], acc[1][0], acc[2][0], acc[3][0]};
            const float sp[4] = {zs_spread<P, NM>(acc[0]), zs_spread<P, NM>(acc[1]), zs_spread<P, NM>(acc[2]),
                                 zs_spread<P, NM>(acc[3])};
            p_pass = !zs_p_above(mean, sp, g1, RHO_MIN, P_MIN);
        }
#pragma unroll 1
        for (int za = 0; za < (p_pass ? 4 : 0); ++za) {
            float t[4][NZ];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int py = 0; py < NZ; ++py) {
                    float x = 0.0f;
#pragma unroll
                    for (int px = 0; px < NZ; ++px) x = fmaf(acc[q][px * NQ + py], S.Z[px][za], x);
                    t[q][py] = x;
                }
#pragma unroll
            for (int zb = 0; zb < 4; ++zb) {
                float U[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float x = 0.0f;
#pragma unroll
                    for (int py = 0; py < NZ; ++py) x = fmaf(t[q][py], S.Z[py][zb], x);
                    U[q] = x;
                }
                if (U[0] <= RHO_MIN) continue;
                const float p = pressure_f(g1, U[0], U[1], U[2], U[3]);
                if (p < P_MIN) tp = fminr(tp, zs_ratio(p_avg, P_MIN, p, EPS));
            }
        }
        if (tp < 1.0f) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q][m] = __fmul_rn(acc[q][m], tp);
        }
        theta = th * tp;
    }

    uint32_t flags = 0;
    double umax = 0.0;
    if (kd == KIND_UPDATED) {
        if (!isfinite(acc[0][0]) || !isfinite(acc[3][0])) flags |= STATUS_NAN;
        if (!(acc[0][0] > 0.0f)) flags |= STATUS_RHO;
    }
    if (!OUT64) {
#pragma unroll
        for (int v = 0; v < 4 * NM; ++v) out[(size_t)v * plane + k] = (TOut)acc[v / NM][v % NM];
    } else {
        // U^(n+1) in FP64 is in place: apply the limiter's factors to the modes
        // they change, on the values the combine wrote
        if (rho_clamp || e_fix || theta != 1.0f || pf[0] != 1.0f || pf[1] != 1.0f || pf[2] != 1.0f ||
            pf[3] != 1.0f) {
            double e0 = 0.0;
            if (e_fix) {
                const double rho0 = rho_clamp ? 1e-5 : (double)out[k];
                const double mx0 = out[(size_t)NM * plane + k], my0 = out[(size_t)2 * NM * plane + k];
                e0 = __dadd_rn(__ddiv_rn(1e-5, (double)(a.gamma - 1.0f)),
                               __ddiv_rn(__dmul_rn(0.5, __dadd_rn(__dmul_rn(mx0, mx0), __dmul_rn(my0, my0))), rho0));
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const size_t idx = (size_t)(q * NM + m) * plane + k;
                    if (m == 0) {
                        if (q == 0 && rho_clamp) out[idx] = 1e-5;
                        if (q == 3 && e_fix) out[idx] = e0;
                    } else {
                        const bool border = m / NQ == P || m % NQ == P;
                        if ((border && pf[q] != 1.0f) || theta != 1.0f) {
                            double o = out[idx];
                            if (border) o = __dmul_rn(o, (double)pf[q]);
                            out[idx] = __dmul_rn(o, (double)theta);
                        }
                    }
                }
        }
        if (LAM) {
            // corner values of the state written, accumulated over the modes in
            // increasing order (read back: nothing extra stays live in registers)
            double cs[4][4];
#pragma unroll 1
            for (int q = 0; q < 4; ++q) {  // one variable at a time: bounded live loads
                double cq[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const double o = out[(size_t)(q * NM + m) * plane + k];
#pragma unroll
                    for (int e = 0; e < 4; ++e) cq[e] = __dadd_rn(cq[e], __dmul_rn(o, __ldg(a.phic + m * 4 + e)));
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) cs[e][q] = cq[e];
            }
            if (a.kind[k] & KIND_FLUID) umax = dg_cell_speed(cs, a.gamma64, 0.0);
        }
        if (kd == KIND_UPDATED) {
            const double rho = out[k], mx = out[(size_t)NM * plane + k], my = out[(size_t)2 * NM * plane + k];
            const double p = (double)(a.gamma - 1.0f) * (out[(size_t)3 * NM * plane + k] - 0.5 * (mx * mx + my * my) / rho);
            if (!(p > 0.0)) flags |= STATUS_P;
        }
    }
    if (flags) atomicOr(a.status, flags);
    return umax;
}

// Lanes of a cell in the two-threads-per-cell kernels: lane l (bit 3 clear)
// holds half 0 and lane l + 8 half 1 of the warp's cell (l >> 4) * 8 + (l & 7).
// Eight consecutive lanes thus read one half of 8 consecutive cells, whose
// slots lie VP words apart: their float4 loads fall in 8 distinct bank groups
// (with the partners one lane apart, both halves of a cell, 2 NM words apart,
// shared their banks: every volume load was a 2-way conflict).
constexpr int kPairLane = 8;
__device__ __forceinline__ int pair_half(int t) { return (t >> 3) & 1; }
__device__ __forceinline__ int pair_cell(int t) { return ((t >> 4) << 3) | (t & 7); }

// Shared memory of the fused indicator: one [16][MLP_TILE_KP] BF16 feature
// tile per warp (8 warps).  It reuses the interface-flux region, free once
// every cell has taken its face integrals, where that region is large enough
// (P = 3), else it follows the stage's own shared memory.  The weights are
// read through L1 (staging them in shared memory left L1 too small for the
// stage: measured slower).
constexpr size_t kMlpTileBytes = 8 * 16 * MLP_TILE_KP * sizeof(uint16_t);
__host__ __device__ constexpr size_t align16(size_t n) { return (n + 15) & ~size_t(15); }
template <int P, int MTY, int TX = MTX>
constexpr bool mlp_tiles_in_flux() {
    return sizeof(float) * (P + 1) * 4 * (fx_stride(MTY, TX) + fy_stride(MTY, TX)) >= kMlpTileBytes;
}

// Round-to-nearest BF16 pair, lo in the low half.
__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// The learned indicator fused into the two-threads-per-cell stage (every
// thread of the CTA calls it, once, after the cell phase).  Features
// (zk_mlp.h) of the cell a lane pair just wrote: half 0 the rho modes, half 1
// the E modes (FP32 values of the combine, acc[h]), scaled by the largest
// |mean| of the cell and its four neighbours in the stage INPUT (the tile's
// shared memory, ghosts already filled), and the neighbour-mean differences of
// that input.  Screen: a cell whose features all lie within `screen` of a
// constant state's (all 0) is smooth; a warp
// whose 16 cells are all smooth skips the network.  Otherwise the warp's 16
// cells go through the MLP on the tensor cores (mlp_logits16), and half 0 of
// every updated, unscreened cell with a positive logit appends the cell to the
// list, which the TVB list pass then limits.
template <int P, int TX = MTX>
__device__ __forceinline__ void indicator_epilogue(const MixArgs& a, const float* sd, uint16_t* ftiles, int slot,
                                                   int h, bool upd, const float (&acc)[2][(P + 1) * (P + 1)],
                                                   size_t k) {
    constexpr int NQ = P + 1, NM = NQ * NQ, VP = vpitch(NM);
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, row = pair_cell(lane);
    float f[20];
#pragma unroll
    for (int i = 0; i < 20; ++i) f[i] = 0.0f;
    float dev = 0.0f;  // largest |feature| of this half: the deviation from a constant state
    if (upd) {
        const int var = h ? 3 : 0;
        const float m0 = sd[slot * VP + var * NM];
        const float mL = sd[(slot - 1) * VP + var * NM], mR = sd[(slot + 1) * VP + var * NM];
        const float mU = sd[(slot - (TX + 2)) * VP + var * NM], mD = sd[(slot + (TX + 2)) * VP + var * NM];
        const float sc = fmaxf(fmaxf(fmaxf(fabsf(m0), fabsf(mL)), fmaxf(fabsf(mR), fabsf(mU))), fabsf(mD)) + 1e-12f;
        const float is = 1.0f / sc;
#pragma unroll
        for (int px = 0; px < NQ; ++px)
#pragma unroll
            for (int py = 0; py < NQ; ++py) f[px * 4 + py] = (h ? acc[1][px * NQ + py] : acc[0][px * NQ + py]) * is;
        f[0] = __fsub_rn(f[0], 1.0f);
        f[16] = (mL - m0) * is;
        f[17] = (mR - m0) * is;
        f[18] = (mU - m0) * is;
        f[19] = (mD - m0) * is;
#pragma unroll
        for (int i = 0; i < 20; ++i) dev = fmaxf(dev, fabsf(f[i]));
    }
    dev = fmaxf(dev, __shfl_xor_sync(FULL, dev, kPairLane));
    const bool cand = upd && !(dev <= a.screen);
    __syncthreads();  // every face integral is taken: the flux region may hold the feature tiles
    const bool warp_runs = __any_sync(FULL, cand);
    float z = -INFINITY;
    if (warp_runs) {
        uint16_t* tile = ftiles + (threadIdx.x >> 5) * 16 * MLP_TILE_KP;
        uint32_t* trow = reinterpret_cast<uint32_t*>(tile + row * MLP_TILE_KP);
        // row layout (words of BF16 pairs): rho modes 0..7, E modes 8..15, rho
        // differences 16..17, E differences 18..19, zero padding 20..23
#pragma unroll
        for (int w = 0; w < 8; ++w) trow[8 * h + w] = bf16x2(f[2 * w], f[2 * w + 1]);
        trow[16 + 2 * h] = bf16x2(f[16], f[17]);
        trow[17 + 2 * h] = bf16x2(f[18], f[19]);
        trow[20 + 2 * h] = 0u;
        trow[21 + 2 * h] = 0u;
        __syncwarp();
        float lo, hi;
        mlp_logits16(a.mlp, tile, lane, lo, hi);
        const int src = 4 * (row & 7);
        const float zl = __shfl_sync(FULL, lo, src), zh = __shfl_sync(FULL, hi, src);
        if (cand) z = row < 8 ? zl : zh;
    }
    if (a.dbg && upd) {
        float* o = a.dbg + k * 41;
#pragma unroll
        for (int i = 0; i < 16; ++i) o[16 * h + i] = f[i];
#pragma unroll
        for (int i = 0; i < 4; ++i) o[32 + 4 * h + i] = f[16 + i];
        if (h == 0) o[40] = z;
    }
    const bool app = h == 0 && z > 0.0f;
    const unsigned m = __ballot_sync(FULL, app);
    if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(a.count, (uint32_t)__popc(m));
        base = __shfl_sync(FULL, base, leader);
        if (app) {
            const uint32_t idx = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
            if (idx < a.cap) a.list[idx] = (int32_t)k;
        }
    }
}

// Own half (two variables, 2 NM floats, contiguous in a cell-major slot) as
// vectors of VW floats.
template <int NM>
struct HalfVec {
    static constexpr int VW = (2 * NM) % 4 == 0 ? 4 : 2;
};
template <int VW>
__device__ __forceinline__ void load_vec(const float* p, float (&x)[VW]) {
    if constexpr (VW == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
    } else {
        const float2 v = *reinterpret_cast<const float2*>(p);
        x[0] = v.x; x[1] = v.y;
    }
}
template <int VW>
__device__ __forceinline__ void store_vec(float* p, const float (&x)[VW]) {
    if constexpr (VW == 4) *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
    else *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
}

// The four variables from this half's pair (a0, a1) and the partner's
// (o0, o1): half 0 owns variables 0, 1, half 1 owns 2, 3.
__device__ __forceinline__ void join_pair(int h, float a0, float a1, float o0, float o1, float (&U)[4]) {
    U[0] = h ? o0 : a0;
    U[1] = h ? o1 : a1;
    U[2] = h ? a0 : o0;
    U[3] = h ? a1 : o1;
}

// stage_tile with two threads per cell: lanes 2i and 2i + 1 share cell i of
// the tile and half h = lane & 1 owns variables 2h, 2h + 1 (traces,
// transforms, accumulators, Persson factor, combine, output).  What needs all
// four variables at a point -- the fluxes at every quadrature point and face
// point, the Zhang-Shu pressure, the positivity check -- swaps the pair with
// the partner lane and is evaluated by both halves.  Every value is formed
// with the operations, in the order, of stage_tile, so the two give the same
// bits.  Shuffles run under masks taken by ballot over lanes that are all
// present: the face loop has a warp-uniform trip count and the cell phase
// returns only after its last shuffle.
template <int P, typename TIn, typename TOut, int MTY, bool LAM = false, bool MLP = false, int TX = MTX>
__device__ __forceinline__ double stage_tile_pair(const MixArgs& a, int j0, int i0, float* smem) {
    constexpr int SXT = TX + 2, MNT = TX * MTY, NT = 2 * MNT, SY = MTY + 2;
    constexpr int NQ = P + 1, NM = NQ * NQ;
    constexpr int SD = SXT * SY;
    constexpr int VP = vpitch(NM);
    constexpr int VW = HalfVec<NM>::VW;
    constexpr unsigned FULL = 0xffffffffu;
    const DGSepF& S = c_sepf[P - 1];
    float* sd = smem;
    float* sfx = sd + VP * SD;
    float* sfy = sfx + NQ * 4 * fx_stride(MTY, TX);
    uint8_t* sk = reinterpret_cast<uint8_t*>(sfy + NQ * 4 * fy_stride(MTY, TX));

    const int tid = threadIdx.x, h = pair_half(tid), ci = pair_cell(tid);
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;

    // U^n of this half's variables, towards L2 (read again only by the combine)
    {
        const int pr = ci / TX, pc = ci - pr * TX;
        if (i0 + pr < ny && j0 + pc < nx) {
            const double* u0 = a.un + (size_t)(2 * h * NM) * plane + (size_t)(i0 + pr) * pitch + (j0 + pc);
#pragma unroll 8
            for (int v = 0; v < 2 * NM; ++v)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(u0 + (size_t)v * plane));
        }
    }

    // 0. gather tile + halo over all NT threads
    gather_tile<P, TIn, MTY, NT, TX>(a, j0, i0, sd, sk, tid);
    __syncthreads();

    // 1. interface fluxes: one thread per face (all four variables), so no
    //    flux is evaluated twice and the 256 threads cover the faces in two rounds
    tile_face_fluxes<P, MTY, NT, TX>(a, sd, sfx, sfy, sk, tid);
    // no barrier yet: the volume quadrature reads only the gathered state, so
    // warps without a second face start on it while the last faces finish

    // 2. one lane pair per cell
    const int r = ci / TX, c = ci - r * TX;
    const int gi = i0 + r, gj = j0 + c;
    const bool inside = gi < ny && gj < nx;
    const unsigned pm = __ballot_sync(FULL, inside);  // lanes of cells in the grid (whole pairs)
    const int slot = (r + 1) * SXT + c + 1;
    const size_t k = inside ? (size_t)gi * pitch + gj : 0;
    const uint8_t kd = inside ? sk[slot] : (uint8_t)KIND_PASSIVE;
    const unsigned um = __ballot_sync(FULL, kd == KIND_UPDATED);
    float acc[2][NM];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc)
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[cc][m] = 0.0f;
    if (kd == KIND_UPDATED) {
        const float* pc = sd + slot * VP + 2 * h * NM;
#pragma unroll 1
        for (int qa = 0; qa < NQ; ++qa) {
            float e[2][NQ];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int n = 0; n < NQ; ++n) e[cc][n] = 0.0f;
#pragma unroll
            for (int v = 0; v < 2 * NM; v += VW) {
                float dv[VW];
                load_vec<VW>(pc + v, dv);
#pragma unroll
                for (int u = 0; u < VW; ++u) {
                    const int cc = (v + u) / NM, m = (v + u) % NM;
                    e[cc][m % NQ] = fmaf(dv[u], S.L[m / NQ][qa], e[cc][m % NQ]);
                }
            }
            float f[2][NQ], g[2][NQ];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int n = 0; n < NQ; ++n) f[cc][n] = g[cc][n] = 0.0f;
#pragma unroll
            for (int qb = 0; qb < NQ; ++qb) {
                float uo[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    float x = 0.0f;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) x = fmaf(e[cc][n], S.L[n][qb], x);
                    uo[cc] = x;
                }
                float U[4];
                join_pair(h, uo[0], uo[1], __shfl_xor_sync(um, uo[0], kPairLane), __shfl_xor_sync(um, uo[1], kPairLane), U);
                float F[4], G[4];
                euler_flux_f(U, a.gamma, F, G);
                const float w = S.W[qa] * S.W[qb];
                const float Fo[2] = {h ? F[2] : F[0], h ? F[3] : F[1]};
                const float Go[2] = {h ? G[2] : G[0], h ? G[3] : G[1]};
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const float Fw = Fo[cc] * w, Gw = Go[cc] * w;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) {
                        f[cc][n] = fmaf(Fw, S.L[n][qb], f[cc][n]);
                        g[cc][n] = fmaf(Gw, S.D[n][qb], g[cc][n]);
                    }
                }
            }
#pragma unroll
            for (int px = 0; px < NQ; ++px) {
                const float dx = S.D[px][qa], lx = S.L[px][qa];
#pragma unroll
                for (int py = 0; py < NQ; ++py)
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc)
                        acc[cc][px * NQ + py] = fmaf(dx, f[cc][py], fmaf(lx, g[cc][py], acc[cc][px * NQ + py]));
            }
        }
    }
    __syncthreads();  // every interface flux is in shared memory
    // the cell phase of lanes whose cell is in the grid; the fused indicator
    // after it is entered by every lane of the warp
    const auto cell_phase = [&]() -> double {
    if (!inside) return 0.0;
    if (kd == KIND_UPDATED) {
        // face integrals of this half's variables (order of stage_tile)
        {
            const float* Fr = sfx + r * (TX + 1) + c + 1;
            const float* Fl = sfx + r * (TX + 1) + c;
            const float* Fd = sfy + (r + 1) * TX + c;
            const float* Fu = sfy + r * TX + c;
            constexpr int fsx = fx_stride(MTY, TX), fsy = fy_stride(MTY, TX);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int u = 2 * h + cc;
                float hr[NQ], hl[NQ], hd[NQ], hu[NQ];
#pragma unroll
                for (int n = 0; n < NQ; ++n) hr[n] = hl[n] = hd[n] = hu[n] = 0.0f;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const float xr = Fr[(q * 4 + u) * fsx], xl = Fl[(q * 4 + u) * fsx];
                    const float xd = Fd[(q * 4 + u) * fsy], xu = Fu[(q * 4 + u) * fsy];
#pragma unroll
                    for (int n = 0; n < NQ; ++n) {
                        const float wl = S.WL[n][q];
                        hr[n] = fmaf(wl, xr, hr[n]);
                        hl[n] = fmaf(wl, xl, hl[n]);
                        hd[n] = fmaf(wl, xd, hd[n]);
                        hu[n] = fmaf(wl, xu, hu[n]);
                    }
                }
#pragma unroll
                for (int px = 0; px < NQ; ++px)
#pragma unroll
                    for (int py = 0; py < NQ; ++py) {
                        float t = acc[cc][px * NQ + py] - hr[py] - hd[px];
                        t += (px & 1) ? -hl[py] : hl[py];
                        t += (py & 1) ? -hu[px] : hu[px];
                        acc[cc][px * NQ + py] = t;
                    }
            }
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const float scale = (float)((2 * (m / NQ) + 1) * (2 * (m % NQ) + 1)) * a.inv2h;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) acc[cc][m] *= scale;
        }
    }

    if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 2 * NM; ++v)
            static_cast<TOut*>(a.out)[(size_t)(2 * h * NM + v) * plane + k] = (TOut)acc[v / NM][v % NM];
        return 0.0;
    }
    // combine in FP64 (w = cur + dt dU at stages 2, 3); an FP64 output is
    // written here, and the limiter later rewrites only the modes it changes
    const double dt = a.dt;
    const float* pw = sd + slot * VP + 2 * h * NM;
    TOut* out = static_cast<TOut*>(a.out);
    constexpr bool OUT64 = sizeof(TOut) == 8;
    double om[2] = {0.0, 0.0};  // this half's written cell means
    // U^n in chunks of UC values loaded before any is combined: an FP64
    // output is U^n itself, so each store orders the loads after it and a
    // load per store is one L2 round trip per value (stage 3 at 2048^2, P = 3:
    // 2.66 -> 1.93 ms).  With an FP32 output all of this half's values are
    // loaded first (the P = 3 step: 5.75 -> 5.62 ms against a vector at a time)
    constexpr int NV = 2 * NM, UC = OUT64 ? kUnChunk : NV;
    static_assert(UC % VW == 0, "chunks of whole vectors");
#pragma unroll
    for (int v0 = 0; v0 < NV; v0 += UC) {
        double unc[UC];
#pragma unroll
        for (int e = 0; e < UC; ++e)
            if (v0 + e < NV) unc[e] = a.un[(size_t)(2 * h * NM + v0 + e) * plane + k];
#pragma unroll
        for (int v = v0; v < v0 + UC && v < NV; v += VW) {
            float cv[VW];
            load_vec<VW>(pw + v, cv);
#pragma unroll
            for (int e = 0; e < VW; ++e) {
                const int vv = v + e, cc = vv / NM, m = vv % NM;
                const double un = unc[vv - v0];
                const double du = (double)acc[cc][m];
                const double o =
                    a.stage == 1 ? __fma_rn(dt, du, un) : so_combine(a.stage, un, __fma_rn(dt, du, (double)cv[e]));
                acc[cc][m] = (float)o;
                if (OUT64) {
                    out[(size_t)(2 * h * NM + vv) * plane + k] = (TOut)o;
                    if (m == 0) om[cc] = o;
                }
            }
        }
    }
    __syncwarp(pm);  // the partner's written cell means are read below

    // limiter decisions in FP32 (src_DG/fluid.cpp:824-992), as factors
    float pf[2] = {1.0f, 1.0f};
    float theta = 1.0f;
    bool rho_clamp = false, e_fix = false;
    const bool in_range = gi >= 3 && gi < ny - 3 && gj >= 3 && gj < nx - 3;
    const bool lim = a.limiter == ZK_LIMITER_REFERENCE && in_range;
    const unsigned lm = __ballot_sync(pm, lim);
    if (lim) {
        if (kd == KIND_UPDATED) {
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                pf[cc] = persson_factor<P, NM>(acc[cc], a.s0);
                if (pf[cc] != 1.0f) {
#pragma unroll
                    for (int m = 0; m < NM; ++m)
                        if (m / NQ == P || m % NQ == P) acc[cc][m] = __fmul_rn(acc[cc][m], pf[cc]);
                }
            }
        }
        const float RHO_MIN = 1e-5f, P_MIN = 1e-5f, EPS = 1e-5f, g1 = a.gamma - 1.0f;
        float m0[4];  // the cell means of all four variables
        join_pair(h, acc[0][0], acc[1][0], __shfl_xor_sync(lm, acc[0][0], kPairLane), __shfl_xor_sync(lm, acc[1][0], kPairLane), m0);
        if (m0[0] < RHO_MIN) { m0[0] = RHO_MIN; rho_clamp = true; }
        const float rho0 = m0[0], mx0 = m0[1], my0 = m0[2];
        const float ke0 = half_m2_over_rho(rho0, mx0, my0);
        if (__fmul_rn(g1, __fsub_rn(m0[3], ke0)) < P_MIN) { m0[3] = __fadd_rn(__fdividef(P_MIN, g1), ke0); e_fix = true; }
        acc[0][0] = h ? m0[2] : m0[0];
        acc[1][0] = h ? m0[3] : m0[1];
        // Zhang-Shu points (4 x 4 Gauss grid, cubic factors zero), separable;
        // the density pass runs on half 0's variable 0 and is shared
        constexpr int NZ = NQ < 3 ? NQ : 3;
        float th = 1.0f;
        float spo[2] = {zs_spread<P, NM>(acc[0]), zs_spread<P, NM>(acc[1])};  // this half's spreads
        float sp[4];
        join_pair(h, spo[0], spo[1], __shfl_xor_sync(lm, spo[0], kPairLane), __shfl_xor_sync(lm, spo[1], kPairLane), sp);
        const bool rho_pass = !zs_above(rho0, sp[0], RHO_MIN);  // the same decision in both halves
#pragma unroll 1
        for (int za = 0; za < (rho_pass ? 4 : 0); ++za) {
            float t[NZ];
#pragma unroll
            for (int py = 0; py < NZ; ++py) {
                float x = 0.0f;
#pragma unroll
                for (int px = 0; px < NZ; ++px) x = fmaf(acc[0][px * NQ + py], S.Z[px][za], x);
                t[py] = x;
            }
#pragma unroll
            for (int zb = 0; zb < 4; ++zb) {
                float rho = 0.0f;
#pragma unroll
                for (int py = 0; py < NZ; ++py) rho = fmaf(t[py], S.Z[py][zb], rho);
                if (rho < RHO_MIN) th = fminr(th, zs_ratio(rho0, RHO_MIN, rho, EPS));
            }
        }
        {
            const float tho = __shfl_xor_sync(lm, th, kPairLane);
            th = h ? tho : th;
        }
        if (th < 1.0f) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) acc[cc][m] = __fmul_rn(acc[cc][m], th);
        }
        const float p_avg = pressure_f(g1, m0[0], m0[1], m0[2], m0[3]);
        float tp = 1.0f;
        // the spreads after the density factor (every lane of lm shuffles)
        spo[0] = zs_spread<P, NM>(acc[0]);
        spo[1] = zs_spread<P, NM>(acc[1]);
        join_pair(h, spo[0], spo[1], __shfl_xor_sync(lm, spo[0], kPairLane), __shfl_xor_sync(lm, spo[1], kPairLane), sp);
        const bool p_pass = !zs_p_above(m0, sp, g1, RHO_MIN, P_MIN);  // the same in both halves
        const unsigned zm = __ballot_sync(lm, p_pass);                 // lanes that run the pressure pass
#pragma unroll 1
        for (int za = 0; za < (p_pass ? 4 : 0); ++za) {
            float t[2][NZ];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int py = 0; py < NZ; ++py) {
                    float x = 0.0f;
#pragma unroll
                    for (int px = 0; px < NZ; ++px) x = fmaf(acc[cc][px * NQ + py], S.Z[px][za], x);
                    t[cc][py] = x;
                }
#pragma unroll
            for (int zb = 0; zb < 4; ++zb) {
                float uo[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    float x = 0.0f;
#pragma unroll
                    for (int py = 0; py < NZ; ++py) x = fmaf(t[cc][py], S.Z[py][zb], x);
                    uo[cc] = x;
                }
                float U[4];
                join_pair(h, uo[0], uo[1], __shfl_xor_sync(zm, uo[0], kPairLane), __shfl_xor_sync(zm, uo[1], kPairLane), U);
                if (U[0] <= RHO_MIN) continue;
                const float p = pressure_f(g1, U[0], U[1], U[2], U[3]);
                if (p < P_MIN) tp = fminr(tp, zs_ratio(p_avg, P_MIN, p, EPS));
            }
        }
        if (tp < 1.0f) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) acc[cc][m] = __fmul_rn(acc[cc][m], tp);
        }
        theta = th * tp;
    }

    uint32_t flags = 0;
    double umax = 0.0;
    if (kd == KIND_UPDATED) {
        if (!isfinite(h ? acc[1][0] : acc[0][0])) flags |= STATUS_NAN;  // rho (half 0) or E (half 1)
        if (h == 0 && !(acc[0][0] > 0.0f)) flags |= STATUS_RHO;
    }
    if (!OUT64) {
#pragma unroll
        for (int v = 0; v < 2 * NM; ++v) out[(size_t)(2 * h * NM + v) * plane + k] = (TOut)acc[v / NM][v % NM];
    } else {
        // U^(n+1) in FP64 is in place: apply the limiter's factors to the modes
        // of this half they change, on the values the combine wrote
        if (rho_clamp || e_fix || theta != 1.0f || pf[0] != 1.0f || pf[1] != 1.0f) {
            double e0 = 0.0;
            if (e_fix && h == 1) {  // rho and m_x means: the partner's, written before the syncwarp
                const double rho0 = rho_clamp ? 1e-5 : (double)out[k];
                const double mx0 = out[(size_t)NM * plane + k], my0 = om[0];
                e0 = __dadd_rn(__ddiv_rn(1e-5, (double)(a.gamma - 1.0f)),
                               __ddiv_rn(__dmul_rn(0.5, __dadd_rn(__dmul_rn(mx0, mx0), __dmul_rn(my0, my0))), rho0));
            }
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const int q = 2 * h + cc;
                    const size_t idx = (size_t)(q * NM + m) * plane + k;
                    if (m == 0) {
                        if (q == 0 && rho_clamp) out[idx] = om[cc] = 1e-5;
                        if (q == 3 && e_fix) out[idx] = om[cc] = e0;
                    } else {
                        const bool border = m / NQ == P || m % NQ == P;
                        if ((border && pf[cc] != 1.0f) || theta != 1.0f) {
                            double o = out[idx];
                            if (border) o = __dmul_rn(o, (double)pf[cc]);
                            out[idx] = __dmul_rn(o, (double)theta);
                        }
                    }
                }
        }
        if (LAM) {
            // corner values of this half's variables in the state written (read back)
            double cs[4][2] = {};
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const double o = out[(size_t)((2 * h + cc) * NM + m) * plane + k];
#pragma unroll
                    for (int e = 0; e < 4; ++e) cs[e][cc] = __dadd_rn(cs[e][cc], __dmul_rn(o, __ldg(a.phic + m * 4 + e)));
                }
            double full[4][4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double o0 = __shfl_xor_sync(pm, cs[e][0], kPairLane), o1 = __shfl_xor_sync(pm, cs[e][1], kPairLane);
                full[e][0] = h ? o0 : cs[e][0];
                full[e][1] = h ? o1 : cs[e][1];
                full[e][2] = h ? cs[e][0] : o0;
                full[e][3] = h ? cs[e][1] : o1;
            }
            if (a.kind[k] & KIND_FLUID) umax = dg_cell_speed(full, a.gamma64, 0.0);
        }
        const double p0 = __shfl_xor_sync(pm, om[0], kPairLane), p1 = __shfl_xor_sync(pm, om[1], kPairLane);
        if (kd == KIND_UPDATED && h == 0) {
            const double rho = om[0], mx = om[1], my = p0, E = p1;
            const double p = (double)(a.gamma - 1.0f) * (E - 0.5 * (mx * mx + my * my) / rho);
            if (!(p > 0.0)) flags |= STATUS_P;
        }
    }
    if (flags) atomicOr(a.status, flags);
    return umax;
    };
    const double umax_cell = cell_phase();
    if constexpr (MLP) {
        // feature tiles: the flux region, or after the stage's shared memory
        constexpr size_t own = sizeof(float) * (VP * SD + NQ * 4 * fx_stride(MTY, TX) + NQ * 4 * fy_stride(MTY, TX)) + SD;
        uint16_t* tiles = mlp_tiles_in_flux<P, MTY, TX>() ? reinterpret_cast<uint16_t*>(sfx)
                                                     : reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(smem) +
                                                                                   align16(own));
        if (a.stage > 0) indicator_epilogue<P, TX>(a, sd, tiles, slot, h, inside && kd == KIND_UPDATED, acc, k);
    }
    return umax_cell;
}

template <int P, int MTY, int TX = MTX>
constexpr size_t smem_bytes() {
    constexpr int NQ = P + 1, NM = NQ * NQ, SY = MTY + 2, SXT = TX + 2;
    return sizeof(float) * (vpitch(NM) * SXT * SY + NQ * 4 * fx_stride(MTY, TX) + NQ * 4 * fy_stride(MTY, TX)) +
           SXT * SY;
}

// resident CTAs per SM: 8 for P=1 (+5% over 3), 3 for P=2 (4 and 5 were
// slower) and P=3 (bounded by shared memory)
template <int P, typename TIn, typename TOut>
__global__ void __launch_bounds__(MTX * 4, P == 1 ? 8 : 3) dg_stage_mixed_kernel(MixArgs a) {
    extern __shared__ __align__(16) float smem[];
    stage_tile<P, TIn, TOut, 4>(a, blockIdx.x * MTX, blockIdx.y * 4, smem);
}

// The same stage with two threads per cell (stage_tile_pair).  Register
// shares: 1024 threads per SM for P = 1, 768 for P = 2 (80 registers, no
// spills; 512 ran 15% slower), 512 for P = 3 (2 CTAs of 8 warps at 128
// registers; 768 spilled and ran 17% slower).
constexpr int pair_thread_budget(int P) { return P == 1 ? 1024 : P == 3 ? 512 : 768; }
// Tile of the single-problem two-threads-per-cell kernel (columns x rows).
// 16 x 8 gathers 1.41 halo slots per cell and leaves 24 of its 280 faces for
// a second round of the 256 threads; 32 x 4: 1.59 and 36 of 292.  P = 3 step
// with the fused indicator at 2048^2: 5.355 vs 5.394 ms, P = 2 2.605 vs 2.656
// ms (P = 3 with the reference limiter 5.237 vs 5.199).  32 x 2 (4 CTAs of
// 128 threads, the same 16 warps per SM, halo 2.1x) ran 9% slower than 32 x 4.
constexpr int kPairCols = 16, kPairRows = 8;
// Shared memory of the single-problem pair kernel, with the indicator's
// feature tiles when MLP.
template <int P, bool MLP>
constexpr size_t pair_smem_bytes() {
    return MLP && !mlp_tiles_in_flux<P, kPairRows, kPairCols>()
               ? align16(smem_bytes<P, kPairRows, kPairCols>()) + kMlpTileBytes
               : smem_bytes<P, kPairRows, kPairCols>();
}
template <int P, bool MLP = false>
constexpr int pair_min_blocks() {
    return batch_min_blocks(kPairCols * 2 * kPairRows, pair_thread_budget(P), pair_smem_bytes<P, MLP>());
}
template <int P, typename TIn, typename TOut, bool MLP>
__global__ void __launch_bounds__(kPairCols * 2 * kPairRows, pair_min_blocks<P, MLP>())
    dg_stage_mixed_pair_kernel(MixArgs a) {
    extern __shared__ __align__(16) float smem[];
    stage_tile_pair<P, TIn, TOut, kPairRows, false, MLP, kPairCols>(a, blockIdx.x * kPairCols, blockIdx.y * kPairRows,
                                                                    smem);
}

// Default threads per cell of the single-problem stage kernel, per P, when
// the autotuner does not run (measured at 2048^2, four-quadrant, GDOF/s, one
// vs two threads per cell): P = 1 38.4 vs 35.9, P = 2 39.0 vs 42.5, P = 3 33.8
// vs 39.0.  The context's autotuner times both on its own grid (dg_driver.cu).
constexpr int kSingleTpc[4] = {0, 1, 2, 2};

// Persistent stage STAGE over every listed problem of a batch group, tile
// variant V (dg_variant_rows(V) rows, dg_variant_tpc(V) threads per cell):
// stage 1 reads U^n (FP64) and writes F[0], stage 2 reads F[0] and writes
// F[1], stage 3 reads F[1] and writes U^n and leaves the new state's max wave
// speed in the problem's control block.  Register shares: one thread per
// cell, 1024 (P = 1) or 384 threads per SM; two, pair_thread_budget(P).
template <int P, int V>
constexpr int batch_blocks() {
    constexpr int MTY = dg_variant_rows(V);
    return dg_variant_tpc(V) == 1 ? (P == 1 ? 32 : 12) / MTY
                                  : batch_min_blocks(MTX * MTY * 2, pair_thread_budget(P), smem_bytes<P, MTY>());
}
template <int P, int STAGE, int V>
__global__ void __launch_bounds__(MTX * dg_variant_rows(V) * dg_variant_tpc(V), batch_blocks<P, V>())
    dg_stage_mixed_batch_kernel(const DgItem* __restrict__ items, const int* __restrict__ dir, int cap) {
    constexpr int MTY = dg_variant_rows(V);
    using TIn = typename std::conditional<STAGE == 1, double, float>::type;
    using TOut = typename std::conditional<STAGE == 3, double, float>::type;
    extern __shared__ __align__(16) float smem[];
    __shared__ MixArgs sa;  // the current tile's problem, kept out of registers
    __shared__ int s_org[3];
    __shared__ unsigned long long* s_lam;
    const int total = __ldg(dir + 1);
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        if (threadIdx.x == 0) {
            const DirHit h = dir_lookup(dir, cap, t);
            const DgItem& it = items[h.item];
            BatchCtl* ctl = it.ctl;
            s_org[2] = ctl->stepping;
            if (s_org[2]) {
                const int tiles_x = (it.g.nx + MTX - 1) / MTX;
                const int ty = h.local / tiles_x;
                s_org[0] = (h.local - ty * tiles_x) * MTX;
                s_org[1] = ty * MTY;
                const void* cur = STAGE == 1 ? (const void*)it.U[0] : (const void*)it.F[STAGE - 2];
                void* out = STAGE == 3 ? (void*)it.U[0] : (void*)it.F[STAGE - 1];
                sa = MixArgs{cur, it.U[0], out, it.kind, it.gsrc, it.g, ctl->dt, (float)it.inv2h, (float)it.gamma,
                             STAGE, it.limiter, it.hll, (float)it.s0, &ctl->status, it.phic, it.gamma};
                s_lam = &ctl->lam;
            }
        }
        __syncthreads();
        if (s_org[2]) {
            double m;
            if constexpr (dg_variant_tpc(V) == 1) m = stage_tile<P, TIn, TOut, MTY, STAGE == 3>(sa, s_org[0], s_org[1], smem);
            else m = stage_tile_pair<P, TIn, TOut, MTY, STAGE == 3>(sa, s_org[0], s_org[1], smem);
            if (STAGE == 3) block_max_commit_to(m, s_lam);  // the next step's wave speed
        }
        __syncthreads();
    }
}

template <int P, int STAGE, int V>
cudaError_t batch_one(const DgItem* items, const int* dir, int cap, int grid, cudaStream_t s, int* occ) {
    constexpr size_t sm = smem_bytes<P, dg_variant_rows(V)>();
    constexpr int nt = MTX * dg_variant_rows(V) * dg_variant_tpc(V);
    static std::atomic<bool> attr_set[64];  // per device; any host thread may launch
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(dg_stage_mixed_batch_kernel<P, STAGE, V>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr_set[dev].store(true, std::memory_order_release);
    }
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, dg_stage_mixed_batch_kernel<P, STAGE, V>, nt, sm);
    dg_stage_mixed_batch_kernel<P, STAGE, V><<<grid, nt, sm, s>>>(items, dir, cap);
    return cudaGetLastError();
}

template <int P, int V>
cudaError_t batch_pv(int stage, const DgItem* items, const int* dir, int cap, int grid, cudaStream_t s, int* occ) {
    switch (stage) {
        case 1: return batch_one<P, 1, V>(items, dir, cap, grid, s, occ);
        case 2: return batch_one<P, 2, V>(items, dir, cap, grid, s, occ);
        case 3: return batch_one<P, 3, V>(items, dir, cap, grid, s, occ);
        default: return cudaErrorInvalidValue;
    }
}

template <int P>
cudaError_t batch_p(int variant, int stage, const DgItem* items, const int* dir, int cap, int grid, cudaStream_t s,
                    int* occ) {
    static_assert(kDgVariants == 4, "one case per tile variant");
    switch (variant) {
        case 0: return batch_pv<P, 0>(stage, items, dir, cap, grid, s, occ);
        case 1: return batch_pv<P, 1>(stage, items, dir, cap, grid, s, occ);
        case 2: return batch_pv<P, 2>(stage, items, dir, cap, grid, s, occ);
        case 3: return batch_pv<P, 3>(stage, items, dir, cap, grid, s, occ);
        default: return cudaErrorInvalidValue;
    }
}

template <int P, typename TIn, typename TOut, int TPC, bool MLP>
cudaError_t launch_one(const MixArgs& a, cudaStream_t s) {
    constexpr bool pair = TPC == 2;
    static_assert(pair || !MLP, "the fused indicator runs in the two-threads-per-cell kernel");
    constexpr int rows = pair ? kPairRows : 4, cols = pair ? kPairCols : MTX;
    constexpr size_t sm = pair ? pair_smem_bytes<P, MLP>() : smem_bytes<P, rows>();
    auto* kern = pair ? dg_stage_mixed_pair_kernel<P, TIn, TOut, MLP> : dg_stage_mixed_kernel<P, TIn, TOut>;
    static std::atomic<bool> attr_set[64];  // per device; any host thread may launch
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr_set[dev].store(true, std::memory_order_release);
    }
    dim3 grid((a.g.nx + cols - 1) / cols, (a.g.ny + rows - 1) / rows);
    kern<<<grid, cols * rows * TPC, sm, s>>>(a);
    return cudaGetLastError();
}

template <int P, typename TIn, typename TOut>
cudaError_t launch_io(const MixArgs& a, int tpc, cudaStream_t s) {
    if constexpr (P >= 2)
        if (a.mlp) return launch_one<P, TIn, TOut, 2, true>(a, s);
    return tpc == 2 ? launch_one<P, TIn, TOut, 2, false>(a, s) : launch_one<P, TIn, TOut, 1, false>(a, s);
}

template <int P>
cudaError_t launch_p(const MixArgs& a, int in_fp64, int out_fp64, int tpc, cudaStream_t s) {
    if (in_fp64 && !out_fp64) return launch_io<P, double, float>(a, tpc, s);
    if (!in_fp64 && !out_fp64) return launch_io<P, float, float>(a, tpc, s);
    if (!in_fp64 && out_fp64) return launch_io<P, float, double>(a, tpc, s);
    return launch_io<P, double, double>(a, tpc, s);
}

}  // namespace

// FP32 copy of P's basis tables in this file's constant bank (once per device, P).
int dg_upload_tables_f32(int P) {
    static std::mutex mu;
    static uint64_t done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ZK_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev] & (1ull << P)) return ZK_OK;
    DGTab T;
    double phic[DG_MAXNM * 4];
    dg_make_tables(P, &T, phic);
    DGTabF F;
    std::memset(&F, 0, sizeof F);
    const double* src = reinterpret_cast<const double*>(&T);
    float* dst = reinterpret_cast<float*>(&F);
    static_assert(sizeof(DGTab) / sizeof(double) == sizeof(DGTabF) / sizeof(float), "table layouts differ");
    for (size_t i = 0; i < sizeof(DGTab) / sizeof(double); ++i) dst[i] = (float)src[i];
    if (cudaMemcpyToSymbol(c_tabf, &F, sizeof F, sizeof F * (P - 1)) != cudaSuccess) return ZK_ERR_CUDA;
    DGSep S;
    dg_make_sep(P, &S);
    DGSepF SF;
    std::memset(&SF, 0, sizeof SF);
    for (int n = 0; n < DG_MAXNQ; ++n) {
        for (int q = 0; q < DG_MAXNQ; ++q) {
            SF.L[n][q] = (float)S.L[n][q];
            SF.D[n][q] = (float)S.D[n][q];
            SF.WL[n][q] = (float)(S.W[q] * S.L[n][q]);
        }
        SF.W[n] = (float)S.W[n];
        for (int a = 0; a < 4; ++a) SF.Z[n][a] = (float)S.Z[n][a];
    }
    if (cudaMemcpyToSymbol(c_sepf, &SF, sizeof SF, sizeof SF * (P - 1)) != cudaSuccess) return ZK_ERR_CUDA;
    done[dev] |= (1ull << P);
    return ZK_OK;
}

// One mixed-precision DG stage of a batch group (grid persistent CTAs).
cudaError_t launch_dg_stage_mixed_batch(int P, int variant, int stage, const DgItem* items, const int* dir, int cap,
                                        int grid, cudaStream_t s) {
    switch (P) {
        case 1: return batch_p<1>(variant, stage, items, dir, cap, grid, s, nullptr);
        case 2: return batch_p<2>(variant, stage, items, dir, cap, grid, s, nullptr);
        case 3: return batch_p<3>(variant, stage, items, dir, cap, grid, s, nullptr);
        default: return cudaErrorInvalidValue;
    }
}

// Resident CTAs per SM of the batch stage kernel (0 on error).
int dg_mixed_batch_occupancy(int P, int variant, int stage) {
    int n = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (P) {
        case 1: e = batch_p<1>(variant, stage, nullptr, nullptr, 0, 0, nullptr, &n); break;
        case 2: e = batch_p<2>(variant, stage, nullptr, nullptr, 0, 0, nullptr, &n); break;
        case 3: e = batch_p<3>(variant, stage, nullptr, nullptr, 0, 0, nullptr, &n); break;
        default: break;
    }
    return e == cudaSuccess ? n : 0;
}

// Tiles of one problem for tile variant v.
int dg_mixed_batch_tiles(int variant, int ny, int nx) {
    return ((nx + MTX - 1) / MTX) * ((ny + dg_variant_rows(variant) - 1) / dg_variant_rows(variant));
}

// One mixed-precision DG stage: cur (double if in_fp64 else float) -> out
// (double if out_fp64 else float).

// Whether the single-problem stage of order P runs the indicator fused (the
// two-threads-per-cell kernel, P = 2, 3), and its default threads per cell.
bool dg_mixed_fuses_indicator(int P) { return P >= 2 && P <= 3; }
int dg_mixed_default_tpc(int P) { return P >= 1 && P <= 3 ? kSingleTpc[P] : 1; }
// With `ind` (P = 2, 3: the two-threads-per-cell kernels) the learned
// indicator runs fused in the stage and appends the cells it flags to
// ind->list; the caller then runs the TVB list pass.
cudaError_t launch_dg_stage_mixed(int P, const void* cur, int in_fp64, const double* un, void* out, int out_fp64,
                                  const int8_t* kind, const int32_t* gsrc, const Grid& g, double dt, double da,
                                  double gamma, int stage, int limiter, int hll, double s0, uint32_t* status,
                                  const FusedIndicator* ind, int tpc, cudaStream_t s) {
    MixArgs a{cur, un, out, kind, gsrc, g, dt, (float)(0.5 / da), (float)gamma, stage, limiter, hll, (float)s0,
              status};
    if (tpc != 1 && tpc != 2) tpc = dg_mixed_default_tpc(P);
    if (ind) {
        if (!dg_mixed_fuses_indicator(P)) return cudaErrorInvalidValue;
        a.mlp = static_cast<const MlpFrag*>(ind->mlp);
        a.list = ind->list;
        a.count = ind->count;
        a.cap = ind->cap;
        a.dbg = ind->dbg;
        a.screen = ind->screen;
    }
    switch (P) {
        case 1: return launch_p<1>(a, in_fp64, out_fp64, tpc, s);
        case 2: return launch_p<2>(a, in_fp64, out_fp64, tpc, s);
        case 3: return launch_p<3>(a, in_fp64, out_fp64, tpc, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zk
