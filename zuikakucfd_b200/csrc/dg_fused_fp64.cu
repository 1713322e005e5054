// DG P=1..3 stage in FP64, ONE fused kernel per RK stage (ZK_PREC_FP64_FMA).
//
// The plain-FP64 counterpart of the mixed-precision stage (dg_mixed.cu): the
// same tile structure and sum-factorised transforms, every value in FP64 and
// multiply-adds contracted, as the reference's own Makefile build contracts
// them.  It is the fastest plain-FP64 DG stage of this library and the
// denominator the mixed path's speed-up is quoted against; it is not
// bit-identical to the reference (the reference-arithmetic path, dg_fp64.cu,
// is), and holds the FP64 path's 1e-10 against the reference's faithful build.
//
// A CTA owns a 32 x 4 tile with two threads per cell (lanes 2i, 2i + 1 share
// cell i; half h owns variables 2h, 2h + 1).  It gathers tile + 1-cell halo of
// the FP64 stage input into shared memory (ghosts through the fill source map,
// slip walls negated), computes every interface flux of the tile once (one
// thread per face, all four variables), then each lane pair runs its cell's
// volume quadrature and face integrals by sum factorisation, the Shu-Osher
// combine and the Persson + Zhang-Shu limiter (src_DG/fluid.cpp:824-992),
// exchanging what needs all four variables at a point with the partner lane.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>

#include "dg_common.cuh"
#include "zk_internal.h"

namespace zk {
namespace {

// One-dimensional basis factors in FP64 (DGSep), plus WL[n][q] = w_q P_n(x_q).
struct DGSepD {
    double L[DG_MAXNQ][DG_MAXNQ];
    double D[DG_MAXNQ][DG_MAXNQ];
    double W[DG_MAXNQ];
    double WL[DG_MAXNQ][DG_MAXNQ];
    double Z[DG_MAXNQ][4];
};
__constant__ DGSepD c_sepd[3];

constexpr int TX = 32, TY = 4, SXD = TX + 2, SYD = TY + 2, SDD = SXD * SYD;
constexpr int NTHREAD = 2 * TX * TY;

struct F64Args {
    const double* cur;  // stage input (U^n at stage 1)
    const double* un;
    double* out;        // may alias un at stage 3 (each cell reads U^n before writing it)
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double dt, inv2h, gamma;
    int stage, limiter, hll;
    double s0;
    uint32_t* status;
};

// Doubles per cell slot in shared memory: 4 NM, or 4 NM + 2, so that a slot
// is an odd number of 16-byte units (conflict-free double2 loads across cells).
__host__ __device__ constexpr int vpitch_d(int nm) { return ((4 * nm / 2) % 2 == 1) ? 4 * nm : 4 * nm + 2; }

template <int P>
constexpr size_t smem_bytes_d() {
    constexpr int NQ = P + 1, NM = NQ * NQ;
    return sizeof(double) * ((size_t)vpitch_d(NM) * SDD + NQ * 4 * TY * (TX + 1) + NQ * 4 * (TY + 1) * TX) + SDD;
}

// eulerFluxX/Y (src_DG/fluid.cpp:123-143)
__device__ __forceinline__ void euler_flux_d(const double U[4], double gam, double F[4], double G[4]) {
    const double eps = 1e-3;
    const double rho = ref_max(U[0], eps);
    const double u = U[1] / rho, v = U[2] / rho;
    const double p = ref_max((gam - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
    F[0] = rho * u; F[1] = rho * u * u + p; F[2] = rho * u * v; F[3] = (U[3] + p) * u;
    G[0] = rho * v; G[1] = rho * u * v; G[2] = rho * v * v + p; G[3] = (U[3] + p) * v;
}

// hllcFlux, DG variant (src_DG/fluid.cpp:450-520)
__device__ __forceinline__ void hllc_dg_d(const double L[4], const double R[4], double gamma, double F[4]) {
    const double eps = 1e-5;
    const double rhoL = ref_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL;
    const double pL = ref_max((gamma - 1.0) * (L[3] - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    const double aL = sqrt(ref_max(gamma * pL / rhoL, eps));
    const double rhoR = ref_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR;
    const double pR = ref_max((gamma - 1.0) * (R[3] - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    const double aR = sqrt(ref_max(gamma * pR / rhoR, eps));
    const double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    double den = sqL + sqR;
    if (den < eps) den = eps;
    const double u_roe = (sqL * uL + sqR * uR) / den;
    const double h_roe = (sqL * ((L[3] + pL) / rhoL) + sqR * ((R[3] + pR) / rhoR)) / den;
    const double c_roe = sqrt(ref_max((gamma - 1.0) * (h_roe - 0.5 * u_roe * u_roe), eps));
    const double SL = ref_min(uL - aL, u_roe - c_roe);
    const double SR = ref_max(uR + aR, u_roe + c_roe);
    if (SL >= 0.0) {
        F[0] = rhoL * uL; F[1] = rhoL * uL * uL + pL; F[2] = rhoL * uL * vL; F[3] = (L[3] + pL) * uL;
        return;
    }
    if (SR <= 0.0) {
        F[0] = rhoR * uR; F[1] = rhoR * uR * uR + pR; F[2] = rhoR * uR * vR; F[3] = (R[3] + pR) * uR;
        return;
    }
    const double num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    double den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabs(den2) < eps) den2 = (den2 >= 0.0 ? eps : -eps);
    const double Ss = num / den2;
    const bool left = Ss >= 0.0;
    const double rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const double p = left ? pL : pR, S = left ? SL : SR;
    // the upwind side's conserved state (values selected, no pointer into the arrays)
    const double U0 = left ? L[0] : R[0], U1 = left ? L[1] : R[1], U2 = left ? L[2] : R[2], U3 = left ? L[3] : R[3];
    double denom = S - Ss;
    if (fabs(denom) < eps) denom = (denom >= 0.0 ? eps : -eps);
    const double c = rho * (S - u) / denom;
    double term = (Ss - u) * (Ss + p / (rho * (S - u)));
    if (!isfinite(term)) term = 0.0;
    F[0] = rho * u + S * (c - U0);
    F[1] = rho * u * u + p + S * (c * Ss - U1);
    F[2] = rho * u * v + S * (c * v - U2);
    F[3] = (U3 + p) * u + S * (c * (U3 / rho + term) - U3);
}

// hlleFlux (src_DG/fluid.cpp:525-580)
__device__ __forceinline__ void hlle_dg_d(const double L[4], const double R[4], double gamma, double F[4]) {
    const double eps = 1e-6;
    const double rhoL = ref_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3];
    const double pL = ref_max((gamma - 1.0) * (EL - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    const double aL = sqrt(ref_max(gamma * pL / rhoL, eps));
    const double rhoR = ref_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3];
    const double pR = ref_max((gamma - 1.0) * (ER - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    const double aR = sqrt(ref_max(gamma * pR / rhoR, eps));
    const double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    const double den = ref_max(sqL + sqR, eps);
    const double u_roe = (sqL * uL + sqR * uR) / den, v_roe = (sqL * vL + sqR * vR) / den;
    const double h_roe = (sqL * ((EL + pL) / rhoL) + sqR * ((ER + pR) / rhoR)) / den;
    const double c_roe = sqrt(ref_max((gamma - 1.0) * (h_roe - 0.5 * (u_roe * u_roe + v_roe * v_roe)), eps));
    const double SL = ref_min(uL - aL, u_roe - c_roe), SR = ref_max(uR + aR, u_roe + c_roe);
    const double FL[4] = {rhoL * uL, rhoL * uL * uL + pL, rhoL * uL * vL, (EL + pL) * uL};
    const double FR[4] = {rhoR * uR, rhoR * uR * uR + pR, rhoR * uR * vR, (ER + pR) * uR};
    if (SL >= 0.0) {
        for (int c = 0; c < 4; ++c) F[c] = FL[c];
    } else if (SR <= 0.0) {
        for (int c = 0; c < 4; ++c) F[c] = FR[c];
    } else {
        const double d = ref_max(SR - SL, eps);
        for (int c = 0; c < 4; ++c) F[c] = (SR * FL[c] - SL * FR[c] + SL * SR * (R[c] - L[c])) / d;
    }
}

// Every interface flux of the tile once, one thread per face (all four
// variables): traces by sum factorisation (the face-normal index contracted
// with P_n(+1) = 1 and P_n(-1) = (-1)^n), then HLLC / HLL at the NQ face points.
template <int P>
__device__ __forceinline__ void face_fluxes_d(const F64Args& a, const double* sd, double* sfx, double* sfy,
                                              const uint8_t* sk, int tid) {
    constexpr int NQ = P + 1, NM = NQ * NQ, VP = vpitch_d(NM);
    const DGSepD& S = c_sepd[P - 1];
    constexpr int NXF = TY * (TX + 1), NYF = (TY + 1) * TX;
    for (int f = tid; f < NXF + NYF; f += NTHREAD) {
        int sl, sr;
        double* dst;
        int dstride;
        bool ydir;
        if (f < NXF) {
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            sl = (r + 1) * SXD + c;
            sr = sl + 1;
            dst = sfx + r * (TX + 1) + c;
            dstride = TY * (TX + 1);
            ydir = false;
        } else {
            const int g = f - NXF, r = g / TX, c = g - r * TX;
            sl = r * SXD + c + 1;
            sr = sl + SXD;
            dst = sfy + r * TX + c;
            dstride = (TY + 1) * TX;
            ydir = true;
        }
        if (sk[sl] != KIND_UPDATED && sk[sr] != KIND_UPDATED) continue;
        double el[4][NQ], er[4][NQ];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int n = 0; n < NQ; ++n) el[c][n] = er[c][n] = 0.0;
        const double* pl = sd + sl * VP;
        const double* pr = sd + sr * VP;
#pragma unroll
        for (int v2 = 0; v2 < 4 * NM; v2 += 2) {
            const double2 l2 = *reinterpret_cast<const double2*>(pl + v2);
            const double2 r2 = *reinterpret_cast<const double2*>(pr + v2);
            const double lv[2] = {l2.x, l2.y}, rv[2] = {r2.x, r2.y};
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = (v2 + e) / NM, m = (v2 + e) % NM, px = m / NQ, py = m % NQ;
                if (ydir) {
                    el[c][px] += lv[e];
                    er[c][px] += (py & 1) ? -rv[e] : rv[e];
                } else {
                    el[c][py] += lv[e];
                    er[c][py] += (px & 1) ? -rv[e] : rv[e];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double UL[4], UR[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                double ul = 0.0, ur = 0.0;
#pragma unroll
                for (int n = 0; n < NQ; ++n) {
                    ul += el[c][n] * S.L[n][q];
                    ur += er[c][n] * S.L[n][q];
                }
                UL[c] = ul;
                UR[c] = ur;
            }
            double Fq[4];
            if (ydir) {
                const double l[4] = {UL[0], UL[2], UL[1], UL[3]}, r[4] = {UR[0], UR[2], UR[1], UR[3]};
                double g[4];
                if (a.hll) hlle_dg_d(l, r, a.gamma, g);
                else hllc_dg_d(l, r, a.gamma, g);
                Fq[0] = g[0]; Fq[1] = g[2]; Fq[2] = g[1]; Fq[3] = g[3];
            } else {
                if (a.hll) hlle_dg_d(UL, UR, a.gamma, Fq);
                else hllc_dg_d(UL, UR, a.gamma, Fq);
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) dst[(q * 4 + c) * dstride] = Fq[c];
        }
    }
}

__device__ __forceinline__ void join_pair_d(int h, double a0, double a1, double o0, double o1, double (&U)[4]) {
    U[0] = h ? o0 : a0;
    U[1] = h ? o1 : a1;
    U[2] = h ? a0 : o0;
    U[3] = h ? a1 : o1;
}

// One stage of one tile (i0, j0).  Shuffles run under masks taken by ballot
// over lanes that are all present: the cell phase returns only after its last
// shuffle.
template <int P>
__global__ void __launch_bounds__(NTHREAD, P == 3 ? 1 : 2) dg_stage_fused_fp64_kernel(F64Args a) {
    constexpr int NQ = P + 1, NM = NQ * NQ, VP = vpitch_d(NM);
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) double smd[];
    double* sd = smd;                              // [SDD][VP] stage input, cell-major
    double* sfx = sd + VP * SDD;                   // [NQ*4][TY][TX+1]
    double* sfy = sfx + NQ * 4 * TY * (TX + 1);    // [NQ*4][TY+1][TX]
    uint8_t* sk = reinterpret_cast<uint8_t*>(sfy + NQ * 4 * (TY + 1) * TX);  // [SYD][SXD]
    const DGSepD& S = c_sepd[P - 1];

    const int tid = threadIdx.x, h = tid & 1, ci = tid >> 1;
    const int j0 = blockIdx.x * TX, i0 = blockIdx.y * TY;
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;

    // U^n of this half's variables towards L2 (read again only by the combine)
    {
        const int pr = ci / TX, pc = ci - pr * TX;
        if (i0 + pr < ny && j0 + pc < nx) {
            const double* u0 = a.un + (size_t)(2 * h * NM) * plane + (size_t)(i0 + pr) * pitch + (j0 + pc);
#pragma unroll 8
            for (int v = 0; v < 2 * NM; ++v) asm volatile("prefetch.global.L2 [%0];" ::"l"(u0 + (size_t)v * plane));
        }
    }

    // 0. gather tile + halo: asynchronous 8-byte copies, ghosts through the
    //    fill source map, then the slip-wall negation
    for (int slot = tid; slot < SDD; slot += NTHREAD) {
        const int r = slot / SXD, c = slot - r * SXD;
        const int gi = i0 - 1 + r, gj = j0 - 1 + c;
        uint8_t kd = KIND_PASSIVE;
        double* dst = sd + (size_t)slot * VP;
        if (gi >= 0 && gi < ny && gj >= 0 && gj < nx) {
            const size_t k = (size_t)gi * pitch + gj;
            kd = a.kind[k] & KIND_MASK;
            size_t ks = k;
            int neg = -1;
            if (kd >= KIND_COPY) {
                ks = (size_t)a.gsrc[k];
                neg = (kd == KIND_SLIP_X) ? 1 : (kd == KIND_SLIP_Y ? 2 : -1);
            }
            const double* src = a.cur + ks;
#pragma unroll 8
            for (int v = 0; v < 4 * NM; ++v)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst + v)),
                             "l"(src + (size_t)v * plane)
                             : "memory");
            asm volatile("cp.async.wait_all;" ::: "memory");
            if (neg >= 0)
                for (int m = 0; m < NM; ++m) dst[neg * NM + m] = -dst[neg * NM + m];
        } else {
            for (int v = 0; v < 4 * NM; ++v) dst[v] = 0.0;
        }
        sk[slot] = kd;
    }
    __syncthreads();

    // 1. interface fluxes, once each
    face_fluxes_d<P>(a, sd, sfx, sfy, sk, tid);

    // 2. one lane pair per cell: volume quadrature by rows (the gathered state only)
    const int r = ci / TX, c = ci - r * TX;
    const int gi = i0 + r, gj = j0 + c;
    const bool inside = gi < ny && gj < nx;
    const unsigned pm = __ballot_sync(FULL, inside);
    const int slot = (r + 1) * SXD + c + 1;
    const size_t k = inside ? (size_t)gi * pitch + gj : 0;
    const uint8_t kd = inside ? sk[slot] : (uint8_t)KIND_PASSIVE;
    const unsigned um = __ballot_sync(FULL, kd == KIND_UPDATED);
    double acc[2][NM];
#pragma unroll
    for (int cc = 0; cc < 2; ++cc)
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[cc][m] = 0.0;
    if (kd == KIND_UPDATED) {
        const double* pc = sd + slot * VP + 2 * h * NM;
#pragma unroll 1
        for (int qa = 0; qa < NQ; ++qa) {
            double e[2][NQ];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int n = 0; n < NQ; ++n) e[cc][n] = 0.0;
#pragma unroll
            for (int v = 0; v < 2 * NM; v += 2) {
                const double2 d2 = *reinterpret_cast<const double2*>(pc + v);
                const double dv[2] = {d2.x, d2.y};
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int cc = (v + u) / NM, m = (v + u) % NM;
                    e[cc][m % NQ] += dv[u] * S.L[m / NQ][qa];
                }
            }
            double f[2][NQ], g[2][NQ];
#pragma unroll
            for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                for (int n = 0; n < NQ; ++n) f[cc][n] = g[cc][n] = 0.0;
#pragma unroll
            for (int qb = 0; qb < NQ; ++qb) {
                double uo[2];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    double x = 0.0;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) x += e[cc][n] * S.L[n][qb];
                    uo[cc] = x;
                }
                double U[4];
                join_pair_d(h, uo[0], uo[1], __shfl_xor_sync(um, uo[0], 1), __shfl_xor_sync(um, uo[1], 1), U);
                double F[4], G[4];
                euler_flux_d(U, a.gamma, F, G);
                const double w = S.W[qa] * S.W[qb];
                const double Fo[2] = {h ? F[2] : F[0], h ? F[3] : F[1]};
                const double Go[2] = {h ? G[2] : G[0], h ? G[3] : G[1]};
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const double Fw = Fo[cc] * w, Gw = Go[cc] * w;
#pragma unroll
                    for (int n = 0; n < NQ; ++n) {
                        f[cc][n] += Fw * S.L[n][qb];
                        g[cc][n] += Gw * S.D[n][qb];
                    }
                }
            }
#pragma unroll
            for (int px = 0; px < NQ; ++px) {
                const double dx = S.D[px][qa], lx = S.L[px][qa];
#pragma unroll
                for (int py = 0; py < NQ; ++py)
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc)
                        acc[cc][px * NQ + py] += dx * f[cc][py] + lx * g[cc][py];
            }
        }
    }
    __syncthreads();  // every interface flux is in shared memory
    if (!inside) return;
    if (kd == KIND_UPDATED) {
        // face integrals (src_DG/fluid.cpp:731-796): right (-), left (+),
        // bottom (-), top (+), weighing P_n(+1) = 1 and P_n(-1) = (-1)^n
        const double* Fr = sfx + r * (TX + 1) + c + 1;
        const double* Fl = sfx + r * (TX + 1) + c;
        const double* Fd = sfy + (r + 1) * TX + c;
        const double* Fu = sfy + r * TX + c;
        constexpr int fsx = TY * (TX + 1), fsy = (TY + 1) * TX;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int u = 2 * h + cc;
            double hr[NQ], hl[NQ], hd[NQ], hu[NQ];
#pragma unroll
            for (int n = 0; n < NQ; ++n) hr[n] = hl[n] = hd[n] = hu[n] = 0.0;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const double xr = Fr[(q * 4 + u) * fsx], xl = Fl[(q * 4 + u) * fsx];
                const double xd = Fd[(q * 4 + u) * fsy], xu = Fu[(q * 4 + u) * fsy];
#pragma unroll
                for (int n = 0; n < NQ; ++n) {
                    const double wl = S.WL[n][q];
                    hr[n] += wl * xr;
                    hl[n] += wl * xl;
                    hd[n] += wl * xd;
                    hu[n] += wl * xu;
                }
            }
#pragma unroll
            for (int px = 0; px < NQ; ++px)
#pragma unroll
                for (int py = 0; py < NQ; ++py) {
                    double t = acc[cc][px * NQ + py] - hr[py] - hd[px];
                    t += (px & 1) ? -hl[py] : hl[py];
                    t += (py & 1) ? -hu[px] : hu[px];
                    acc[cc][px * NQ + py] = t;
                }
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const double scale = (double)((2 * (m / NQ) + 1) * (2 * (m % NQ) + 1)) * a.inv2h;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) acc[cc][m] *= scale;
        }
    }

    // 3. combine (src_DG/fluid.cpp:1005-1054), every cell of the tile, ghosts
    //    with their filled values as the whole-array reference does
    const double dt = a.dt;
    const double* pw = sd + slot * VP + 2 * h * NM;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc)
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const double un = a.un[(size_t)((2 * h + cc) * NM + m) * plane + k];
            const double w = pw[cc * NM + m] + dt * acc[cc][m];
            acc[cc][m] = a.stage == 1 ? un + dt * acc[cc][m]
                                      : (a.stage == 2 ? 0.75 * un + 0.25 * w : (1.0 / 3.0) * un + (2.0 / 3.0) * w);
        }

    // 4. limiter (src_DG/fluid.cpp:824-992): Persson on updated cells, then
    //    Zhang-Shu on every cell of [3, n-3)^2
    const bool in_range = gi >= 3 && gi < ny - 3 && gj >= 3 && gj < nx - 3;
    const bool lim = a.limiter == ZK_LIMITER_REFERENCE && in_range;
    const unsigned lm = __ballot_sync(pm, lim);
    if (lim) {
        const double RHO_MIN = 1e-5, P_MIN = 1e-5, EPS = 1e-5, g1 = a.gamma - 1.0;
        if (kd == KIND_UPDATED) {
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                double Et = 0.0, Ep = 0.0;
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const double x = acc[cc][m];
                    Et += x * x;
                    if (m / NQ == P || m % NQ == P) Ep += x * x;
                }
                const double s = log10(Ep / (Et + EPS));
                if (s > a.s0) {
                    const double eps = (s > a.s0 + 1.0) ? 1.0 : 0.5 * (1.0 + sin(M_PI * ((s - a.s0) - 0.5)));
#pragma unroll
                    for (int m = 0; m < NM; ++m)
                        if (m / NQ == P || m % NQ == P) acc[cc][m] *= (1.0 - eps);
                }
            }
        }
        double m0[4];
        join_pair_d(h, acc[0][0], acc[1][0], __shfl_xor_sync(lm, acc[0][0], 1), __shfl_xor_sync(lm, acc[1][0], 1), m0);
        m0[0] = ref_max(m0[0], RHO_MIN);
        const double ke0 = 0.5 * (m0[1] * m0[1] + m0[2] * m0[2]) / m0[0];
        if (g1 * (m0[3] - ke0) < P_MIN) m0[3] = P_MIN / g1 + ke0;
        acc[0][0] = h ? m0[2] : m0[0];
        acc[1][0] = h ? m0[3] : m0[1];
        // Zhang-Shu point values: separable over the 4 x 4 Gauss nodes with the
        // cubic factors dropped (modes px, py < NZ); a variable's point values
        // lie within mean +- sum |modes| (|factor| <= 1), so a pass whose lower
        // bound clears the floor is skipped (it would return exactly 1)
        constexpr int NZ = NQ < 3 ? NQ : 3;
        double spo[2] = {0.0, 0.0};
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
#pragma unroll
            for (int px = 0; px < NZ; ++px)
#pragma unroll
                for (int py = 0; py < NZ; ++py)
                    if (px || py) spo[cc] += fabs(acc[cc][px * NQ + py]);
        double sp[4];
        join_pair_d(h, spo[0], spo[1], __shfl_xor_sync(lm, spo[0], 1), __shfl_xor_sync(lm, spo[1], 1), sp);
        const double rho0 = m0[0];
        double th = 1.0;
        const bool rho_pass = !(rho0 - sp[0] - 1e-12 * (fabs(rho0) + sp[0]) > RHO_MIN);
        if (h == 0 && rho_pass) {
#pragma unroll 1
            for (int za = 0; za < 4; ++za) {
                double t[NZ];
#pragma unroll
                for (int py = 0; py < NZ; ++py) {
                    double x = 0.0;
#pragma unroll
                    for (int px = 0; px < NZ; ++px) x += acc[0][px * NQ + py] * S.Z[px][za];
                    t[py] = x;
                }
#pragma unroll
                for (int zb = 0; zb < 4; ++zb) {
                    double rho = 0.0;
#pragma unroll
                    for (int py = 0; py < NZ; ++py) rho += t[py] * S.Z[py][zb];
                    if (rho < RHO_MIN) th = ref_min(th, (rho0 - RHO_MIN) / (rho0 - rho + EPS));
                }
            }
        }
        {
            const double tho = __shfl_xor_sync(lm, th, 1);
            if (h) th = tho;
        }
        if (th < 1.0) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) acc[cc][m] *= th;
        }
        // the spreads after the density factor (every lane of lm shuffles)
        spo[0] *= th;
        spo[1] *= th;
        join_pair_d(h, spo[0], spo[1], __shfl_xor_sync(lm, spo[0], 1), __shfl_xor_sync(lm, spo[1], 1), sp);
        const double p_avg = g1 * (m0[3] - 0.5 * (m0[1] * m0[1] + m0[2] * m0[2]) / m0[0]);
        // pressure lower bound from the means and spreads (the same decision in both halves)
        bool p_pass = true;
        {
            const double rlo = m0[0] - sp[0] - 1e-12 * (fabs(m0[0]) + sp[0]);
            if (rlo > RHO_MIN) {
                const double mx = fabs(m0[1]) + sp[1], my = fabs(m0[2]) + sp[2];
                const double ke = 0.5 * (mx * mx + my * my) / rlo;
                const double plo = g1 * (m0[3] - sp[3] - ke) - 1e-12 * g1 * (fabs(m0[3]) + sp[3] + ke);
                p_pass = !(plo > P_MIN);
            }
        }
        double tp = 1.0;
        const unsigned zm = __ballot_sync(lm, p_pass);
        if (p_pass) {
#pragma unroll 1
            for (int za = 0; za < 4; ++za) {
                double t[2][NZ];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc)
#pragma unroll
                    for (int py = 0; py < NZ; ++py) {
                        double x = 0.0;
#pragma unroll
                        for (int px = 0; px < NZ; ++px) x += acc[cc][px * NQ + py] * S.Z[px][za];
                        t[cc][py] = x;
                    }
#pragma unroll
                for (int zb = 0; zb < 4; ++zb) {
                    double uo[2];
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        double x = 0.0;
#pragma unroll
                        for (int py = 0; py < NZ; ++py) x += t[cc][py] * S.Z[py][zb];
                        uo[cc] = x;
                    }
                    double U[4];
                    join_pair_d(h, uo[0], uo[1], __shfl_xor_sync(zm, uo[0], 1), __shfl_xor_sync(zm, uo[1], 1), U);
                    if (U[0] <= RHO_MIN) continue;
                    const double u = U[1] / U[0], v = U[2] / U[0];
                    const double p = g1 * (U[3] - 0.5 * U[0] * (u * u + v * v));
                    if (p < P_MIN) tp = ref_min(tp, (p_avg - P_MIN) / (p_avg - p + EPS));
                }
            }
        }
        if (tp < 1.0) {
#pragma unroll
            for (int m = 1; m < NM; ++m)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) acc[cc][m] *= tp;
        }
    }

    // 5. output (this half's variables) and the status word
#pragma unroll
    for (int cc = 0; cc < 2; ++cc)
#pragma unroll
        for (int m = 0; m < NM; ++m) a.out[(size_t)((2 * h + cc) * NM + m) * plane + k] = acc[cc][m];
    uint32_t flags = 0;
    const double o0 = __shfl_xor_sync(pm, acc[0][0], 1), o1 = __shfl_xor_sync(pm, acc[1][0], 1);
    if (kd == KIND_UPDATED && h == 0) {
        const double rho = acc[0][0], mx = acc[1][0], my = o0, E = o1;
        if (!isfinite(rho) || !isfinite(E)) flags |= STATUS_NAN;
        if (!(rho > 0.0)) flags |= STATUS_RHO;
        const double p = (a.gamma - 1.0) * (E - 0.5 * (mx * mx + my * my) / rho);
        if (!(p > 0.0)) flags |= STATUS_P;
    }
    if (flags) atomicOr(a.status, flags);
}

template <int P>
cudaError_t launch_p(const F64Args& a, cudaStream_t s) {
    constexpr size_t sm = smem_bytes_d<P>();
    static std::atomic<bool> attr_set[64];  // per device; any host thread may launch
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev].load(std::memory_order_acquire)) {
        const cudaError_t e =
            cudaFuncSetAttribute(dg_stage_fused_fp64_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr_set[dev].store(true, std::memory_order_release);
    }
    const dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY);
    dg_stage_fused_fp64_kernel<P><<<grid, NTHREAD, sm, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

// FP64 one-dimensional basis factors of P in this file's constant bank (once
// per device and P).
int dg_upload_sep_f64(int P) {
    static std::mutex mu;
    static uint64_t done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ZK_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev] & (1ull << P)) return ZK_OK;
    DGSep S;
    dg_make_sep(P, &S);
    DGSepD D;
    std::memset(&D, 0, sizeof D);
    for (int n = 0; n < DG_MAXNQ; ++n) {
        for (int q = 0; q < DG_MAXNQ; ++q) {
            D.L[n][q] = S.L[n][q];
            D.D[n][q] = S.D[n][q];
            D.WL[n][q] = S.W[q] * S.L[n][q];
        }
        D.W[n] = S.W[n];
        for (int z = 0; z < 4; ++z) D.Z[n][z] = S.Z[n][z];
    }
    if (cudaMemcpyToSymbol(c_sepd, &D, sizeof D, sizeof D * (P - 1)) != cudaSuccess) return ZK_ERR_CUDA;
    done[dev] |= (1ull << P);
    return ZK_OK;
}

// One fused FP64 DG stage (1..3): cur -> out, U^n = un.
cudaError_t launch_dg_stage_fused_fp64(int P, const double* cur, const double* un, double* out, const int8_t* kind,
                                       const int32_t* gsrc, const Grid& g, double dt, double da, double gamma,
                                       int stage, int limiter, int hll, double s0, uint32_t* status, cudaStream_t s) {
    if (stage < 1 || stage > 3) return cudaErrorInvalidValue;
    const F64Args a{cur, un, out, kind, gsrc, g, dt, 0.5 / da, gamma, stage, limiter, hll, s0, status};
    switch (P) {
        case 1: return launch_p<1>(a, s);
        case 2: return launch_p<2>(a, s);
        case 3: return launch_p<3>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zk
