// WENO5 + HLLC + SSP-RK3 stage, mixed precision (the fast path).
//
// Precision split:
//   * reconstruction and HLLC fluxes in FP32 (this file is compiled with
//     --use_fast_math: FP32 division and square root map to the MUFU
//     approximations; FP64 arithmetic is unaffected);
//   * faces whose 6-cell stencil touches an FP64 cell are evaluated in FP64.
//     A cell is FP64 when it is high-Mach -- E > 100 p, where recovering
//     p = (gamma-1)(E - |m|^2 / 2 rho) from FP32 values would lose more than
//     two of its digits to cancellation -- or when a conserved value reaches
//     kFp32Max, beyond which the FP32 smoothness indicators (t ~ 33 |U|^2)
//     square past the range of the reciprocal and the weights turn to 0/0;
//   * interface fluxes are kept in FP64 in shared memory, and dU and the
//     Shu-Osher combine are FP64: the conserved state is accumulated in FP64;
//   * the positivity check recovers p from the FP64 result.
//
// Data movement: one 3D TMA tensor load (cp.async.bulk.tensor, no multicast)
// brings the CTA's 40 x 14 x 4 FP64 box (tile + 3-cell halo, x start rounded
// down to a 16-byte boundary) into shared memory; the completion wait is
// bounded and reports STATUS_TIMEOUT instead of hanging.
#include "batch.cuh"
#include "f32x2.cuh"
#include "tma.cuh"
#include "tma_host.h"
#include "zk_common.cuh"
#include "zk_internal.h"

namespace zk {
namespace {

// A tile is 32 x TY cells; NW warps (TY + 1 by default) take the 2 TY + 2
// face-row tasks in turn.
constexpr int TX = 32, HX = TX + 6;
constexpr int SX = TX + 8;  // staged columns: x from j0-4 (16-byte aligned) to j0+35
template <int TY, int NW = TY + 1>
struct Tile {
    static constexpr int HY = TY + 6, NWARP = NW, NTHREAD = NW * 32;
};
constexpr uint8_t FP64_CELL = 0x10;
constexpr double kFp32Max = 1e8;  // t^2 <= (33.4 kFp32Max^2)^2 ~ 1e35 < 2^126

// weno5_reconstruct (src_WENO/fluid.cpp:230-263), any precision.
template <typename T>
__device__ __forceinline__ void weno5(T UL2, T UL1, T UP, T UR1, T UR2, T UR3, T& UL, T& UR) {
    const T eps = T(1e-6), C1 = T(13.0 / 12.0), C2 = T(0.25);
    const T c13 = T(1.0 / 3.0), c76 = T(7.0 / 6.0), c116 = T(11.0 / 6.0), c16 = T(1.0 / 6.0), c56 = T(5.0 / 6.0);
    T qL0 = c13 * UL2 - c76 * UL1 + c116 * UP;
    T qL1 = -c16 * UL1 + c56 * UP + c13 * UR1;
    T qL2 = c13 * UP + c56 * UR1 - c16 * UR2;
    T d0 = UL2 - T(2) * UL1 + UP, d1 = UL2 - T(4) * UL1 + T(3) * UP;
    T d2 = UL1 - T(2) * UP + UR1, d3 = UL1 - UR1;
    T d4 = UP - T(2) * UR1 + UR2, d5 = T(3) * UP - T(4) * UR1 + UR2;
    T t0 = eps + (C1 * d0 * d0 + C2 * d1 * d1);
    T t1 = eps + (C1 * d2 * d2 + C2 * d3 * d3);
    T t2 = eps + (C1 * d4 * d4 + C2 * d5 * d5);
    T a0 = T(0.1) / (t0 * t0), a1 = T(0.6) / (t1 * t1), a2 = T(0.3) / (t2 * t2);
    UL = (a0 * qL0 + a1 * qL1 + a2 * qL2) / (a0 + a1 + a2);

    T qR0 = c116 * UR1 - c76 * UR2 + c13 * UR3;
    T qR1 = qL2;  // same combination of the same cells
    T qR2 = qL1;
    T r0 = UR1 - T(2) * UR2 + UR3, r1 = T(3) * UR1 - T(4) * UR2 + UR3;
    T r3 = UP - UR2, r5 = UL1 - T(4) * UP + T(3) * UR1;
    T s0 = eps + (C1 * r0 * r0 + C2 * r1 * r1);
    T s1 = eps + (C1 * d4 * d4 + C2 * r3 * r3);  // r2 == d4
    T s2 = eps + (C1 * d2 * d2 + C2 * r5 * r5);  // r4 == d2
    T e0 = T(0.1) / (s0 * s0), e1 = T(0.6) / (s1 * s1), e2 = T(0.3) / (s2 * s2);
    UR = (e0 * qR0 + e1 * qR1 + e2 * qR2) / (e0 + e1 + e2);
}

// Reciprocals of packed pairs stay per lane (MUFU has no pair form).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }

// weno5 above for two variables at once.  The ideal weights are scaled by 10
// (1, 6, 3), which the normalisation divides out.
__device__ __forceinline__ void weno5x2(float2 UL2, float2 UL1, float2 UP, float2 UR1, float2 UR2, float2 UR3,
                                        float2& UL, float2& UR) {
    const float2 eps = f2(1e-6f), C1 = f2(13.0f / 12.0f), C2 = f2(0.25f);
    const float2 c13 = f2(1.0f / 3.0f), m76 = f2(-7.0f / 6.0f), c116 = f2(11.0f / 6.0f), m16 = f2(-1.0f / 6.0f),
                 c56 = f2(5.0f / 6.0f);
    const float2 m1 = f2(-1.0f), m2 = f2(-2.0f), m4 = f2(-4.0f), c3 = f2(3.0f), c6 = f2(6.0f);
    const float2 qL0 = fma2(c116, UP, fma2(m76, UL1, mul2(c13, UL2)));
    const float2 qL1 = fma2(c13, UR1, fma2(c56, UP, mul2(m16, UL1)));
    const float2 qL2 = fma2(m16, UR2, fma2(c56, UR1, mul2(c13, UP)));
    const float2 d0 = add2(fma2(m2, UL1, UL2), UP), d1 = fma2(c3, UP, fma2(m4, UL1, UL2));
    const float2 d2 = add2(fma2(m2, UP, UL1), UR1), d3 = fma2(m1, UR1, UL1);
    const float2 d4 = add2(fma2(m2, UR1, UP), UR2), d5 = add2(fma2(m4, UR1, mul2(c3, UP)), UR2);
    const float2 t0 = add2(eps, fma2(mul2(C1, d0), d0, mul2(mul2(C2, d1), d1)));
    const float2 t1 = add2(eps, fma2(mul2(C1, d2), d2, mul2(mul2(C2, d3), d3)));
    const float2 t2 = add2(eps, fma2(mul2(C1, d4), d4, mul2(mul2(C2, d5), d5)));
    {
        const float2 a0 = rcp2(mul2(t0, t0)), a1 = mul2(c6, rcp2(mul2(t1, t1))), a2 = mul2(c3, rcp2(mul2(t2, t2)));
        const float2 num = fma2(a2, qL2, fma2(a1, qL1, mul2(a0, qL0)));
        UL = mul2(num, rcp2(add2(add2(a0, a1), a2)));
    }
    const float2 qR0 = fma2(c13, UR3, fma2(m76, UR2, mul2(c116, UR1)));
    const float2 r0 = add2(fma2(m2, UR2, UR1), UR3), r1 = fma2(c3, UR1, fma2(m4, UR2, UR3));
    const float2 r3 = fma2(m1, UR2, UP), r5 = fma2(c3, UR1, fma2(m4, UP, UL1));
    const float2 s0 = add2(eps, fma2(mul2(C1, r0), r0, mul2(mul2(C2, r1), r1)));
    const float2 s1 = add2(eps, fma2(mul2(C1, d4), d4, mul2(mul2(C2, r3), r3)));  // r2 == d4
    const float2 s2 = add2(eps, fma2(mul2(C1, d2), d2, mul2(mul2(C2, r5), r5)));  // r4 == d2
    const float2 e0 = rcp2(mul2(s0, s0)), e1 = mul2(c6, rcp2(mul2(s1, s1))), e2 = mul2(c3, rcp2(mul2(s2, s2)));
    const float2 num = fma2(e2, qL1, fma2(e1, qL2, mul2(e0, qR0)));  // qR1 == qL2, qR2 == qL1
    UR = mul2(num, rcp2(add2(add2(e0, e1), e2)));
}

// std::min / std::max argument order of the reference, for either precision.
template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }

// hllcFlux (WENO variant, src_WENO/fluid.cpp:268-317), any precision.
template <typename T>
__device__ __forceinline__ void hllc(const T L[4], const T R[4], T gamma, T F[4]) {
    const T eps = T(1e-12);
    const T gm1 = gamma - T(1);
    T rhoL = (L[0] < eps) ? eps : L[0];
    T irL = T(1) / rhoL;
    T uL = L[1] * irL, vL = L[2] * irL;
    T pL = gm1 * (L[3] - T(0.5) * rhoL * (uL * uL + vL * vL));
    pL = (pL < eps) ? eps : pL;
    T rhoR = (R[0] < eps) ? eps : R[0];
    T irR = T(1) / rhoR;
    T uR = R[1] * irR, vR = R[2] * irR;
    T pR = gm1 * (R[3] - T(0.5) * rhoR * (uR * uR + vR * vR));
    pR = (pR < eps) ? eps : pR;
    T aL = sqrt(gamma * pL * irL), aR = sqrt(gamma * pR * irR);
    T sqL = sqrt(rhoL), sqR = sqrt(rhoR), iden = T(1) / (sqL + sqR);
    T u_roe = (sqL * uL + sqR * uR) * iden;
    T h_roe = (sqL * ((L[3] + pL) * irL) + sqR * ((R[3] + pR) * irR)) * iden;
    T c2 = gm1 * (h_roe - T(0.5) * u_roe * u_roe);
    T c_roe = sqrt(c2 < eps ? eps : c2);
    T SL = tmin(uL - aL, u_roe - c_roe);
    T SR = tmax(uR + aR, u_roe + c_roe);
    if (SL >= T(0)) {
        F[0] = rhoL * uL; F[1] = rhoL * uL * uL + pL; F[2] = rhoL * uL * vL; F[3] = (L[3] + pL) * uL;
        return;
    }
    if (SR <= T(0)) {
        F[0] = rhoR * uR; F[1] = rhoR * uR * uR + pR; F[2] = rhoR * uR * vR; F[3] = (R[3] + pR) * uR;
        return;
    }
    T num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    T den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabs(den2) < eps) den2 = (den2 >= T(0)) ? eps : -eps;
    T Ss = num / den2;
    const bool left = Ss >= T(0);
    const T rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const T p = left ? pL : pR, S = left ? SL : SR, ir = left ? irL : irR;
    const T* Us = left ? L : R;
    T Su = S - u;
    T c = rho * Su / (S - Ss);
    T E = Us[3] * ir;
    T s3 = c * (E + (Ss - u) * (Ss + p / (rho * Su)));
    F[0] = rho * u + S * (c - Us[0]);
    F[1] = rho * u * u + p + S * (c * Ss - Us[1]);
    F[2] = rho * u * v + S * (c * v - Us[2]);
    F[3] = (Us[3] + p) * u + S * (s3 - Us[3]);
}

struct MixedArgs {
    const double* Ucur;  // stage input (ghosts unfilled); the tensor map covers it
    const double* Un;
    double* Uout;  // may alias Un at stage 3 (read-before-write per cell)
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double dtdx, dtdy, gamma;
    int stage;
    uint32_t* status;
    int want_lam;  // 1: report the max wave speed of the cells written
    // failure self-test only (0 in every step): the barrier expects extra_tx
    // bytes more than the copy delivers, and the wait gives up after `spin`
    // polls (0: kSpinLimit)
    uint32_t extra_tx, spin;
};

template <int TY>
struct Smem {
    double stg[4][TY + 6][SX];  // TMA destination, FP64, ghosts fixed up in place (offset 0: 128-byte aligned)
    float2 sU[2][TY + 6][HX];   // FP32 copy of the tile + halo, pairs (rho, m_x) and (m_y, E)
    double sFx[4][TY][TX + 1];
    double sFy[4][TY + 1][TX];
    uint8_t sK[TY + 6][HX];     // kind | FP64_CELL
};

// Flux of one face: XDIR, the x face left of tile cell (r, c) (stencil cells
// (r, c-3 .. c+2)); else the y face above it (cells (r-3 .. r+2, c), normal
// momentum swapped into slot 1).  FP32 unless a stencil cell is FP64_CELL.
template <bool XDIR, int TY>
__device__ __forceinline__ void face_flux(Smem<TY>& S, int r, int c, double gamma, float gf) {
    constexpr int SU = XDIR ? 1 : HX;  // stride between stencil cells in sU / sK
    constexpr int SG = XDIR ? 1 : SX;  // and in stg
    const float2* u0 = XDIR ? &S.sU[0][r + 3][c] : &S.sU[0][r][c + 3];
    const uint8_t* k0 = XDIR ? &S.sK[r + 3][c] : &S.sK[r][c + 3];
    constexpr int PU = (TY + 6) * HX;  // plane stride of sU
    uint8_t hm = 0;
#pragma unroll
    for (int n = 0; n < 6; ++n) hm |= k0[n * SU];
    double F[4];
    if (hm & FP64_CELL) {
        const double* g0 = XDIR ? &S.stg[0][r + 3][c + 1] : &S.stg[0][r][c + 4];
        constexpr int PG = (TY + 6) * SX;
        double QL[4], QR[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double* g = g0 + q * PG;
            weno5<double>(g[0], g[SG], g[2 * SG], g[3 * SG], g[4 * SG], g[5 * SG], QL[q], QR[q]);
        }
        if (!XDIR) {
            double t = QL[1]; QL[1] = QL[2]; QL[2] = t;
            t = QR[1]; QR[1] = QR[2]; QR[2] = t;
        }
        hllc<double>(QL, QR, gamma, F);
    } else {
        float2 L[2], R[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float2* u = u0 + h * PU;
            weno5x2(u[0], u[SU], u[2 * SU], u[3 * SU], u[4 * SU], u[5 * SU], L[h], R[h]);
        }
        // normal momentum into slot 1
        float QL[4] = {L[0].x, XDIR ? L[0].y : L[1].x, XDIR ? L[1].x : L[0].y, L[1].y};
        float QR[4] = {R[0].x, XDIR ? R[0].y : R[1].x, XDIR ? R[1].x : R[0].y, R[1].y};
        float Ff[4];
        hllc<float>(QL, QR, gf, Ff);
#pragma unroll
        for (int q = 0; q < 4; ++q) F[q] = (double)Ff[q];
    }
    if (XDIR) {
#pragma unroll
        for (int q = 0; q < 4; ++q) S.sFx[q][r][c] = F[q];
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) S.sFy[q][r][c] = F[q];
    }
}

// One tile whose top-left cell is (i0, j0); `bar` is an initialised mbarrier
// whose current phase has parity `phase`.  Returns false (after recording
// STATUS_TIMEOUT) when the TMA copy did not land within the spin limit.
// Every thread is past its last shared-memory access on return.  umax: the
// thread's max wave speed of the cells it wrote (want_lam), else 0.
template <int TY, int NW = TY + 1>
__device__ __forceinline__ bool stage_tile(const CUtensorMap* tmap, const MixedArgs& a, int j0, int i0, Smem<TY>& S,
                                           uint64_t* bar, uint32_t phase, double& umax) {
    umax = 0.0;
    constexpr int HY = Tile<TY, NW>::HY, NWARP = Tile<TY, NW>::NWARP, NTHREAD = Tile<TY, NW>::NTHREAD;
    auto& stg = S.stg;
    auto& sU = S.sU;
    auto& sFx = S.sFx;
    auto& sFy = S.sFy;
    auto& sK = S.sK;
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;

    // 1. TMA: the 40 x (TY+6) x 4 box starting at (j0-4, i0-3, 0); out-of-range
    //    elements arrive as zeros
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)sizeof(stg) + a.extra_tx);
        tma_load_3d(&stg[0][0][0], tmap, bar, j0 - 4, i0 - 3, 0);
    }
    const bool ok = mbar_wait_bounded(bar, phase, a.spin ? a.spin : kSpinLimit);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            atomicOr(a.status, STATUS_TIMEOUT);
            if (a.extra_tx) mbar_complete_tx(bar, a.extra_tx);  // self-test: settle the bytes never sent
            mbar_wait_bounded(bar, phase);  // give a late copy a second bounded chance to land
        }
        __syncthreads();  // no thread leaves before the copy into this CTA's shared memory has landed
        return false;
    }

    // U^n of the tile is read again only by the combine; at stages 2 and 3 it
    // is not the TMA'd buffer, so start it towards L2 now (each 32-cell row
    // segment of a plane is two 128-byte lines; pitch is a multiple of 32)
    if (a.stage >= 2 && threadIdx.x < 8 * TY) {
        const int q = threadIdx.x / (2 * TY), rr = (threadIdx.x >> 1) - q * TY, half = threadIdx.x & 1;
        if (i0 + rr < ny)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a.Un + q * plane + (size_t)(i0 + rr) * pitch + j0 +
                                                          16 * half));
    }

    // 2. ghost fill from the source map, FP32 copy, FP64_CELL flags
    const double gm1 = a.gamma - 1.0;
    for (int t = threadIdx.x; t < HY * HX; t += NTHREAD) {
        const int r = t / HX, c = t - r * HX;
        const int gi = i0 - 3 + r, gj = j0 - 3 + c;
        uint8_t kd = KIND_PASSIVE;
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = stg[q][r][c + 1];
        if (gi >= 0 && gi < ny && gj >= 0 && gj < nx) {
            const size_t k = (size_t)gi * pitch + gj;
            kd = a.kind[k] & KIND_MASK;
            if (kd >= KIND_COPY) {
                const size_t s = (size_t)a.gsrc[k];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    v[q] = a.Ucur[q * plane + s];
                    stg[q][r][c + 1] = v[q];
                }
            }
            // high-Mach test E > 100 p, p = (gamma-1)(E - |m|^2 / 2 rho), with
            // both sides multiplied by rho > 0 (no division)
            const double prho = gm1 * (v[3] * v[0] - 0.5 * (v[1] * v[1] + v[2] * v[2]));
            // with rho > 0 and p > 0, |m| <= sqrt(2 rho E) <= rho + E bounds every component
            if (!(v[0] > 0.0) || !(prho > 0.0) || v[3] * v[0] > 100.0 * prho || !(v[0] + v[3] < kFp32Max))
                kd |= FP64_CELL;
        }
        sU[0][r][c] = make_float2((float)v[0], (float)v[1]);
        sU[1][r][c] = make_float2((float)v[2], (float)v[3]);
        sK[r][c] = kd;
    }
    __syncthreads();

    // 3. interface fluxes, once per face (warp tasks as in the FP64 kernel)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float gf = (float)a.gamma;
    for (int task = warp; task < 2 * TY + 2; task += NWARP) {
        // a task is one row of x faces or of y faces, so the direction is
        // uniform across the warp and the stencil addressing is compile-time
        if (task <= TY) {
            int r, c;
            if (task < TY) { r = task; c = lane; }
            else { if (lane >= TY) continue; r = lane; c = TX; }
            if ((sK[r + 3][c + 2] & KIND_MASK) != KIND_UPDATED && (sK[r + 3][c + 3] & KIND_MASK) != KIND_UPDATED)
                continue;
            face_flux<true, TY>(S, r, c, a.gamma, gf);
        } else {
            const int r = task - TY - 1, c = lane;
            if ((sK[r + 2][c + 3] & KIND_MASK) != KIND_UPDATED && (sK[r + 3][c + 3] & KIND_MASK) != KIND_UPDATED)
                continue;
            face_flux<false, TY>(S, r, c, a.gamma, gf);
        }
    }
    __syncthreads();

    // 4. dU (FP64) and the Shu-Osher combine (FP64) for every cell of the tile
    uint32_t flags = 0;
    for (int t = threadIdx.x; t < TY * TX; t += NTHREAD) {
        const int r = t / TX, c = t - r * TX;
        const int gi = i0 + r, gj = j0 + c;
        if (gi >= ny || gj >= nx) continue;
        const size_t k = (size_t)gi * pitch + gj;
        const bool upd = (sK[r + 3][c + 3] & KIND_MASK) == KIND_UPDATED;
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        if (upd) {
            // y fluxes carry the normal momentum in slot 1 (src_WENO/fluid.cpp:457-460)
            d[0] = -(a.dtdx * (sFx[0][r][c + 1] - sFx[0][r][c]) + a.dtdy * (sFy[0][r + 1][c] - sFy[0][r][c]));
            d[1] = -(a.dtdx * (sFx[1][r][c + 1] - sFx[1][r][c]) + a.dtdy * (sFy[2][r + 1][c] - sFy[2][r][c]));
            d[2] = -(a.dtdx * (sFx[2][r][c + 1] - sFx[2][r][c]) + a.dtdy * (sFy[1][r + 1][c] - sFy[1][r][c]));
            d[3] = -(a.dtdx * (sFx[3][r][c + 1] - sFx[3][r][c]) + a.dtdy * (sFy[3][r + 1][c] - sFy[3][r][c]));
        }
        double o[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double un = a.Un[q * plane + k];
            const double v = stg[q][r + 3][c + 4];
            if (a.stage == 1) o[q] = un + d[q];
            else if (a.stage == 2) o[q] = 0.75 * un + 0.25 * (v + d[q]);
            else o[q] = (1.0 / 3.0) * un + (2.0 / 3.0) * (v + d[q]);
        }
        if (upd) {
            if (isnan(o[0]) || isnan(o[1]) || isnan(o[2]) || isnan(o[3])) flags |= STATUS_NAN;
            if (!(o[0] > 0.0)) flags |= STATUS_RHO;  // then p > 0 <=> rho E > |m|^2 / 2
            else if (!(o[3] * o[0] - 0.5 * (o[1] * o[1] + o[2] * o[2]) > 0.0)) flags |= STATUS_P;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) a.Uout[q * plane + k] = o[q];
        if (a.want_lam) {
            const double spd = weno_cell_speed(o[0], o[1], o[2], o[3], a.gamma);
            if (spd > umax) umax = spd;
        }
    }
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (flags && lane == 0) atomicOr(a.status, flags);
    // the next TMA copy overwrites stg, which this tile wrote through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    return true;
}

// 5 CTAs per SM (40 registers, 384 bytes spilled; 223 KB of shared memory):
// the extra resident warps hide more latency than the spills cost.  Per step
// at 2048^2, same bits: 0.618 ms at 5 CTAs, 0.669 ms at 4 (56 registers, 148
// bytes spilled), 0.765 ms at 3 (72 registers).
__global__ void __launch_bounds__(Tile<8>::NTHREAD, 5)
    weno_stage_mixed_kernel(const __grid_constant__ CUtensorMap tmap, MixedArgs a) {
    __shared__ __align__(128) Smem<8> S;
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tma_prefetch_desc(&tmap);
        mbar_init(&bar, 1);
    }
    __syncthreads();
    double umax;
    stage_tile<8>(&tmap, a, blockIdx.x * TX, blockIdx.y * 8, S, &bar, 0, umax);
}

// Persistent stage over every listed problem of a batch group (tile variant
// V of batch.cuh; the register share is that of 1440 threads per SM, 40
// registers).  The tensor maps live in the item array in global memory,
// written by the host before the launch.
template <int V, int TY = weno_variant_rows(V), int NW = weno_variant_warps(V)>
__global__ void __launch_bounds__(NW * 32, batch_min_blocks(NW * 32, 1440, sizeof(Smem<TY>)))
    weno_stage_mixed_batch_kernel(const WenoItem* __restrict__ items, const int* __restrict__ dir, int cap,
                                  int stage) {
    __shared__ __align__(128) Smem<TY> S;
    __shared__ __align__(8) uint64_t bar;
    __shared__ MixedArgs sa;  // the current tile's problem, kept out of registers
    __shared__ int s_org[3];  // tile origin x, y; 0 when the problem is not stepping
    __shared__ const CUtensorMap* s_map;
    __shared__ unsigned long long* s_lam;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    const int total = __ldg(dir + 1);
    uint32_t phase = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        if (threadIdx.x == 0) {
            const DirHit h = dir_lookup(dir, cap, t);
            const WenoItem& it = items[h.item];
            BatchCtl* ctl = it.ctl;
            s_org[2] = ctl->stepping;
            if (s_org[2]) {
                const int tiles_x = (it.g.nx + TX - 1) / TX;
                const int ty = h.local / tiles_x;
                s_org[0] = (h.local - ty * tiles_x) * TX;
                s_org[1] = ty * TY;
                sa = MixedArgs{it.U[stage - 1], it.U[0], it.U[stage % 3], it.kind, it.gsrc, it.g,
                               ctl->dtdx, ctl->dtdy, it.gamma, stage, &ctl->status, stage == 3};
                s_lam = &ctl->lam;
                s_map = &it.tmap[V / 3][stage - 1];
                asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(
                                 reinterpret_cast<uint64_t>(s_map))
                             : "memory");
            }
        }
        __syncthreads();
        if (s_org[2]) {
            double umax;
            if (!stage_tile<TY, NW>(s_map, sa, s_org[0], s_org[1], S, &bar, phase, umax)) return;
            phase ^= 1u;
            if (stage == 3) block_max_commit_to(umax, s_lam);  // the next step's wave speed
        }
        __syncthreads();
    }
}

}  // namespace

namespace {
template <int V>
cudaError_t launch_batch_v(const WenoItem* items, const int* dir, int cap, int stage, int grid, cudaStream_t s) {
    weno_stage_mixed_batch_kernel<V><<<grid, weno_variant_warps(V) * 32, 0, s>>>(items, dir, cap, stage);
    return cudaGetLastError();
}
template <int V>
int occupancy_v() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, weno_stage_mixed_batch_kernel<V>, weno_variant_warps(V) * 32, 0);
    return n;
}
}  // namespace

cudaError_t launch_weno_stage_mixed_batch(int variant, const WenoItem* items, const int* dir, int cap, int stage,
                                          int grid, cudaStream_t s) {
    static_assert(kWenoVariants == 6, "one case per tile variant");
    switch (variant) {
        case 0: return launch_batch_v<0>(items, dir, cap, stage, grid, s);
        case 1: return launch_batch_v<1>(items, dir, cap, stage, grid, s);
        case 2: return launch_batch_v<2>(items, dir, cap, stage, grid, s);
        case 3: return launch_batch_v<3>(items, dir, cap, stage, grid, s);
        case 4: return launch_batch_v<4>(items, dir, cap, stage, grid, s);
        case 5: return launch_batch_v<5>(items, dir, cap, stage, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

int weno_mixed_batch_occupancy(int variant) {
    switch (variant) {
        case 0: return occupancy_v<0>();
        case 1: return occupancy_v<1>();
        case 2: return occupancy_v<2>();
        case 3: return occupancy_v<3>();
        case 4: return occupancy_v<4>();
        case 5: return occupancy_v<5>();
        default: return 0;
    }
}

cudaError_t launch_weno_stage_mixed(const CUtensorMap& tmap, const double* Ucur, const double* Un, double* Uout,
                                    const int8_t* kind, const int32_t* gsrc, const Grid& g, double dtdx,
                                    double dtdy, double gamma, int stage, uint32_t* status, cudaStream_t s) {
    MixedArgs a{Ucur, Un, Uout, kind, gsrc, g, dtdx, dtdy, gamma, stage, status};
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + 7) / 8);
    weno_stage_mixed_kernel<<<grid, Tile<8>::NTHREAD, 0, s>>>(tmap, a);
    return cudaGetLastError();
}

// Stage 1 of the mixed WENO step with a barrier that expects 16 bytes more
// than the TMA copy delivers and a wait limited to `spin` polls: every CTA
// runs out of its wait, records STATUS_TIMEOUT, settles the missing bytes,
// waits for its copy to land and leaves without writing its tile.
cudaError_t launch_weno_timeout_selftest(const CUtensorMap& tmap, const double* Un, double* Uout, const int8_t* kind,
                                         const int32_t* gsrc, const Grid& g, double dtdx, double dtdy, double gamma,
                                         uint32_t spin, uint32_t* status, cudaStream_t s) {
    MixedArgs a{Un, Un, Uout, kind, gsrc, g, dtdx, dtdy, gamma, 1, status, 0, 16u, spin ? spin : 1u};
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + 7) / 8);
    weno_stage_mixed_kernel<<<grid, Tile<8>::NTHREAD, 0, s>>>(tmap, a);
    return cudaGetLastError();
}

// Tensor map over one FP64 WENO state: dims (x = nx, y = ny, field = 4),
// strides pitch*8 and plane*8 bytes, box 40 x (rows + 6) x 4.
bool encode_weno_state_map(CUtensorMap* m, const double* base, const Grid& g, const char** err, int rows) {
    const uint64_t dims[3] = {(uint64_t)g.nx, (uint64_t)g.ny, 4};
    const uint64_t strides[2] = {(uint64_t)g.pitch * 8, (uint64_t)g.plane * 8};
    const uint32_t box[3] = {SX, (uint32_t)rows + 6, 4};
    return encode_tmap(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, err);
}

}  // namespace zk

// ---- driver: the mixed-precision WENO step ---------------------------------------
int zk_weno_mixed_setup(zk_ctx* c) {
    const char* err = nullptr;
    double* bufs[3] = {c->Un, c->S1, c->S2};
    for (int b = 0; b < 3; ++b)
        if (!zk::encode_weno_state_map(&c->tmap[b], bufs[b], c->g, &err, 8)) return zk_internal_fail(ZK_ERR_CUDA, err);
    return ZK_OK;
}

int zk_weno_mixed_step(zk_ctx* c, double dt) {
    const double dtdx = dt / c->da, dtdy = dt / c->da;
    cudaError_t e;
    e = zk::launch_weno_stage_mixed(c->tmap[0], c->Un, c->Un, c->S1, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma, 1,
                                    c->d_status, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_weno_stage_mixed(c->tmap[1], c->S1, c->Un, c->S2, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma,
                                        2, c->d_status, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_weno_stage_mixed(c->tmap[2], c->S2, c->Un, c->Un, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma,
                                        3, c->d_status, c->stream);
    if (e != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e));
    return ZK_OK;
}

extern "C" int zk_selftest_tma_timeout(zk_ctx* c, uint32_t spin_limit, uint32_t* status_out) {
    if (!c || !c->Un || !status_out) return zk_internal_fail(ZK_ERR_ARG, "needs a context with a mesh and status_out");
    if (c->opt.method != ZK_METHOD_WENO || c->opt.precision != ZK_PREC_MIXED)
        return zk_internal_fail(ZK_ERR_UNSUPPORTED, "needs a mixed-precision WENO context");
    cudaError_t e = cudaSetDevice(c->opt.device);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess)
        e = zk::launch_weno_timeout_selftest(c->tmap[0], c->Un, c->S1, c->kind, c->gsrc, c->g, 1e-6 / c->da,
                                             1e-6 / c->da, c->gamma, spin_limit, c->d_status, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(status_out, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? ZK_OK : zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e));
}

// Stage `stage` (1..3) of zk_weno_mixed_step alone: the same launch with the
// same buffers (U^n -> S1 -> S2 -> U^n).
int zk_weno_mixed_stage(zk_ctx* c, double dt, int stage) {
    const double dtdx = dt / c->da, dtdy = dt / c->da;
    double* in[3] = {c->Un, c->S1, c->S2};
    double* out[3] = {c->S1, c->S2, c->Un};
    const cudaError_t e = zk::launch_weno_stage_mixed(c->tmap[stage - 1], in[stage - 1], c->Un, out[stage - 1], c->kind,
                                                      c->gsrc, c->g, dtdx, dtdy, c->gamma, stage, c->d_status,
                                                      c->stream);
    return e == cudaSuccess ? ZK_OK : zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e));
}
