// Discontinuous Galerkin P=1..3 stage, FP64, the reference's arithmetic op
// for op (compiled with --fmad=false, like weno_fp64.cu).
//
// Per RK stage two kernels:
//   dg_face_kernel<P, DIR>  every x (DIR=0) / y (DIR=1) interface flux ONCE:
//                           traces of both cells at the NQ Gauss points of the
//                           face (ghost neighbours gathered through the fill
//                           source map), HLLC or HLL; the reference computes
//                           each face twice from identical inputs.
//   dg_cell_kernel<P>       per cell: volume quadrature, the four face
//                           integrals in the reference's order (right, left,
//                           bottom, top), inverse-mass scaling, the Shu-Osher
//                           combine and the Persson + Zhang-Shu limiter, all in
//                           registers; ghosts get the combine of their filled
//                           value, exactly as the whole-array reference does.
// Basis values are tabulated on the host (no FMA contraction) with the
// reference's own expressions and kept in __constant__ memory, one table set
// per P.
#include <cmath>
#include <cstring>
#include <mutex>

#include "batch.cuh"
#include "dg_common.cuh"
#include "zk_internal.h"

// Built twice: with --fmad=false as the reference-arithmetic path (namespace
// zk), and with -DZK_FP64_FMA, fused multiply-adds contracted, as the
// ZK_PREC_FP64_FMA path (namespace zk_fma).
#ifdef ZK_FP64_FMA
#define ZK_FP64_NS zk_fma
#else
#define ZK_FP64_NS zk
#endif

namespace ZK_FP64_NS {
using namespace zk;

__constant__ DGTab c_dgtab[3];

namespace {

// legP / legD, src_DG/fluid.cpp:34-55 (host; this translation unit's host code
// is compiled without FMA contraction)
double legP_h(int n, double x) {
    switch (n) {
        case 0: return 1.0;
        case 1: return x;
        case 2: return 0.5 * (3.0 * x * x - 1.0);
        case 3: return 0.5 * (5.0 * x * x * x - 3.0 * x);
        case 4: return 0.125 * (35.0 * x * x * x * x - 30.0 * x * x + 3.0);
        default: return 0.0;
    }
}
double legD_h(int n, double x) {
    switch (n) {
        case 0: return 0.0;
        case 1: return 1.0;
        case 2: return 3.0 * x;
        case 3: return 0.5 * (15.0 * x * x - 3.0);
        case 4: return 0.5 * (35.0 * x * x * x - 15.0 * x);
        default: return 0.0;
    }
}

// Gauss-Legendre nodes and weights, the decimal literals of
// src_DG/fluid.cpp:94-111 for NQ = 2..4.
const double kGLPt[5][4] = {{0}, {0},
                            {-0.5773502691896257, 0.5773502691896257, 0, 0},
                            {-0.7745966692414834, 0.0, 0.7745966692414834, 0},
                            {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526}};
const double kGLWt[5][4] = {{0}, {0},
                            {1.0, 1.0, 0, 0},
                            {0.5555555555555556, 0.8888888888888888, 0.5555555555555556, 0},
                            {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538}};

}  // namespace

void dg_make_tables(int P, DGTab* T, double* phic /* [NM][4] */) {
    std::memset(T, 0, sizeof(DGTab));
    const int NQ = P + 1, NM = NQ * NQ;
    const double* PT = kGLPt[NQ];
    const double* WT = kGLWt[NQ];
    auto phi2 = [&](int m, double xi, double eta) { return legP_h(m / (P + 1), xi) * legP_h(m % (P + 1), eta); };
    for (int qa = 0; qa < NQ; ++qa)
        for (int qb = 0; qb < NQ; ++qb) {
            const int p = qa * NQ + qb;
            const double xi = PT[qa], eta = PT[qb];
            T->vw[p] = WT[qa] * WT[qb];
            for (int m = 0; m < NM; ++m) {
                T->vphi[p][m] = phi2(m, xi, eta);
                T->vdxi[p][m] = legD_h(m / (P + 1), xi) * legP_h(m % (P + 1), eta);
                T->vdet[p][m] = legP_h(m / (P + 1), xi) * legD_h(m % (P + 1), eta);
            }
        }
    for (int q = 0; q < NQ; ++q)
        for (int m = 0; m < NM; ++m) {
            // traces: right side (xi=+1), left (xi=-1), bottom (eta=+1), top (eta=-1)
            T->tr[0][q][m] = phi2(m, +1.0, PT[q]);
            T->tr[1][q][m] = phi2(m, -1.0, PT[q]);
            T->tr[2][q][m] = phi2(m, PT[q], +1.0);
            T->tr[3][q][m] = phi2(m, PT[q], -1.0);
            // face weights bv = phi2(m, face point) * w (src_DG/fluid.cpp:740,756,776,792)
            for (int f = 0; f < 4; ++f) T->bv[f][q][m] = T->tr[f][q][m] * WT[q];
        }
    // Zhang-Shu basis at 4x4 Gauss points, cubic factors dropped
    // (src_DG/fluid.cpp:808-823, :892-895)
    const double* G4 = kGLPt[4];
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            for (int m = 0; m < NM; ++m) {
                const int px = m / (P + 1), py = m % (P + 1);
                const double x = G4[a], y = G4[b];
                const double fa = (px == 0) ? 1.0 : (px == 1) ? x : (px == 2) ? 0.5 * (3.0 * x * x - 1.0) : 0.0;
                const double fb = (py == 0) ? 1.0 : (py == 1) ? y : (py == 2) ? 0.5 * (3.0 * y * y - 1.0) : 0.0;
                T->zs[a * 4 + b][m] = fa * fb;
            }
    const double XI[4] = {-1.0, +1.0, -1.0, +1.0}, ETA[4] = {-1.0, -1.0, +1.0, +1.0};
    for (int m = 0; m < NM; ++m)
        for (int k = 0; k < 4; ++k) phic[m * 4 + k] = phi2(m, XI[k], ETA[k]);
}

void dg_make_sep(int P, DGSep* S) {
    std::memset(S, 0, sizeof(DGSep));
    const int NQ = P + 1;
    for (int n = 0; n < NQ; ++n) {
        for (int q = 0; q < NQ; ++q) {
            S->L[n][q] = legP_h(n, kGLPt[NQ][q]);
            S->D[n][q] = legD_h(n, kGLPt[NQ][q]);
        }
        S->E[n][0] = legP_h(n, +1.0);
        S->E[n][1] = legP_h(n, -1.0);
        for (int a = 0; a < 4; ++a) {
            const double x = kGLPt[4][a];
            S->Z[n][a] = (n == 0) ? 1.0 : (n == 1) ? x : (n == 2) ? 0.5 * (3.0 * x * x - 1.0) : 0.0;
        }
    }
    for (int q = 0; q < NQ; ++q) S->W[q] = kGLWt[NQ][q];
}

int dg_upload_tables(int P, const DGTab& T) {
    // __constant__ memory is per device: upload once per (device, P)
    static std::mutex mu;
    static uint64_t done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ZK_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev] & (1ull << P)) return ZK_OK;
    if (cudaMemcpyToSymbol(c_dgtab, &T, sizeof(DGTab), sizeof(DGTab) * (P - 1)) != cudaSuccess) return ZK_ERR_CUDA;
    done[dev] |= (1ull << P);
    return ZK_OK;
}

namespace {

// eulerFluxX / eulerFluxY, src_DG/fluid.cpp:123-143 (floors 1e-3)
__device__ __forceinline__ void euler_flux(const double U[4], double gam, double F[4], double G[4]) {
    const double eps = 1e-3;
    double rho = ref_max(U[0], eps);
    double u = U[1] / rho, v = U[2] / rho;
    double p = ref_max((gam - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
    F[0] = rho * u; F[1] = rho * u * u + p; F[2] = rho * u * v; F[3] = (U[3] + p) * u;
    G[0] = rho * v; G[1] = rho * u * v; G[2] = rho * v * v + p; G[3] = (U[3] + p) * v;
}

// hllcFlux, DG variant, src_DG/fluid.cpp:450-520
__device__ __forceinline__ void hllc_dg(const double L[4], const double R[4], double gamma, double F[4]) {
    const double eps = 1e-5;
    double rhoL = ref_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3] / rhoL;
    double pL = ref_max((gamma - 1.0) * (L[3] - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(ref_max(gamma * pL / rhoL, eps));
    double rhoR = ref_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3] / rhoR;
    double pR = ref_max((gamma - 1.0) * (R[3] - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(ref_max(gamma * pR / rhoR, eps));
    double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    double den = sqL + sqR;
    if (den < eps) den = eps;
    double u_roe = (sqL * uL + sqR * uR) / den;
    double h_roe = (sqL * (EL + pL / rhoL) + sqR * (ER + pR / rhoR)) / den;
    double c_roe = sqrt(ref_max((gamma - 1.0) * (h_roe - 0.5 * u_roe * u_roe), eps));
    double SL = ref_min(uL - aL, u_roe - c_roe);
    double SR = ref_max(uR + aR, u_roe + c_roe);
    if (SL >= 0.0) {
        F[0] = rhoL * uL; F[1] = rhoL * uL * uL + pL; F[2] = rhoL * uL * vL; F[3] = (L[3] + pL) * uL;
        return;
    }
    if (SR <= 0.0) {
        F[0] = rhoR * uR; F[1] = rhoR * uR * uR + pR; F[2] = rhoR * uR * vR; F[3] = (R[3] + pR) * uR;
        return;
    }
    double num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    double den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabs(den2) < eps) den2 = (den2 >= 0 ? eps : -eps);
    double Ss = num / den2;
    const bool left = (Ss >= 0.0);
    const double rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const double E = left ? EL : ER, p = left ? pL : pR, S = left ? SL : SR;
    const double* Us = left ? L : R;
    double denom = S - Ss;
    if (fabs(denom) < eps) denom = (denom >= 0 ? eps : -eps);
    double c = rho * (S - u) / denom;
    double term = (Ss - u) * (Ss + p / (rho * (S - u)));
    if (isnan(term) || isinf(term)) term = 0.0;
    double s1 = c * Ss, s2 = c * v, s3 = c * (E + term);
    F[0] = (rho * u) + S * (c - Us[0]);
    F[1] = (rho * u * u + p) + S * (s1 - Us[1]);
    F[2] = (rho * u * v) + S * (s2 - Us[2]);
    F[3] = ((Us[3] + p) * u) + S * (s3 - Us[3]);
}

// hlleFlux, src_DG/fluid.cpp:525-580 (the reference defines it, never calls it)
__device__ __forceinline__ void hlle_dg(const double L[4], const double R[4], double gamma, double F[4]) {
    const double eps = 1e-6;
    double rhoL = ref_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3];
    double pL = ref_max((gamma - 1.0) * (EL - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(ref_max(gamma * pL / rhoL, eps));
    double HL = (EL + pL) / rhoL;
    double rhoR = ref_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3];
    double pR = ref_max((gamma - 1.0) * (ER - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(ref_max(gamma * pR / rhoR, eps));
    double HR = (ER + pR) / rhoR;
    double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    double invDen = 1.0 / ref_max(sqL + sqR, eps);
    double u_roe = (sqL * uL + sqR * uR) * invDen;
    double v_roe = (sqL * vL + sqR * vR) * invDen;
    double h_roe = (sqL * HL + sqR * HR) * invDen;
    double c_roe = sqrt(ref_max((gamma - 1.0) * (h_roe - 0.5 * (u_roe * u_roe + v_roe * v_roe)), eps));
    double SL = ref_min(uL - aL, u_roe - c_roe);
    double SR = ref_max(uR + aR, u_roe + c_roe);
    double FL[4] = {rhoL * uL, rhoL * uL * uL + pL, rhoL * uL * vL, (EL + pL) * uL};
    double FR[4] = {rhoR * uR, rhoR * uR * uR + pR, rhoR * uR * vR, (ER + pR) * uR};
    if (SL >= 0.0) {
        for (int c = 0; c < 4; ++c) F[c] = FL[c];
    } else if (SR <= 0.0) {
        for (int c = 0; c < 4; ++c) F[c] = FR[c];
    } else {
        double invDiff = 1.0 / ref_max(SR - SL, eps);
        for (int c = 0; c < 4; ++c) F[c] = (SR * FL[c] - SL * FR[c] + SL * SR * (R[c] - L[c])) * invDiff;
    }
}

// Gathered dof read: the fill source of ghost cells, slip walls negating
// the normal momentum (src_DG/fluid.cpp:600-607, 625-632).
struct CellRef {
    size_t k;  // index to read
    int neg;   // conserved variable to negate (-1 = none)
};
__device__ __forceinline__ CellRef cell_ref(const DGArgs& a, size_t k) {
    const int8_t kd = a.kind[k] & KIND_MASK;
    if (kd < KIND_COPY) return {k, -1};
    return {(size_t)a.gsrc[k], kd == KIND_SLIP_X ? 1 : (kd == KIND_SLIP_Y ? 2 : -1)};
}

// Traces of one cell at the NQ points of one side: U[q][c] = sum_m dof*phi.
template <int P>
__device__ __forceinline__ void cell_traces(const DGArgs& a, CellRef r, const double (&tr)[DG_MAXNQ][DG_MAXNM],
                                            double (&U)[P + 1][4]) {
    constexpr int NQ = P + 1, NM = NQ * NQ;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int c = 0; c < 4; ++c) U[q][c] = 0.0;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        double d[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double x = a.cur[(size_t)(c * NM + m) * a.g.plane + r.k];
            d[c] = (r.neg == c) ? -x : x;
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int c = 0; c < 4; ++c) U[q][c] += d[c] * tr[q][m];
    }
}

// One thread per interface.  DIR 0: x face (i, jf) between cells (i, jf-1)
// and (i, jf); DIR 1: y face (if, j) between (if-1, j) above and (if, j) below.
// Faces (i, jb + threadIdx.x).
template <int P, int DIR>
__device__ __forceinline__ void face_row(const DGArgs& a, int jb, int i) {
    constexpr int NQ = P + 1;
    const DGTab& T = c_dgtab[P - 1];
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const int j = jb + threadIdx.x;
    size_t kl, kr;  // the two cells
    if (DIR == 0) {
        if (j < 1 || j >= nx || i >= ny) return;
        kl = (size_t)i * pitch + (j - 1);
        kr = (size_t)i * pitch + j;
    } else {
        if (j >= nx || i < 1 || i >= ny) return;
        kl = (size_t)(i - 1) * pitch + j;
        kr = (size_t)i * pitch + j;
    }
    if ((a.kind[kl] & KIND_MASK) != KIND_UPDATED && (a.kind[kr] & KIND_MASK) != KIND_UPDATED) return;
    double UL[NQ][4], UR[NQ][4];
    cell_traces<P>(a, cell_ref(a, kl), T.tr[DIR == 0 ? 0 : 2], UL);
    cell_traces<P>(a, cell_ref(a, kr), T.tr[DIR == 0 ? 1 : 3], UR);
    const size_t qstride = (DIR == 0) ? (size_t)ny * a.xpitch : (size_t)(ny + 1) * pitch;
    const size_t o = (DIR == 0) ? (size_t)i * a.xpitch + j : (size_t)i * pitch + j;
    double* F = (DIR == 0) ? a.fx : a.fy;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double f[4];
        if (DIR == 0) {
            if (a.hll) hlle_dg(UL[q], UR[q], a.gamma, f);
            else hllc_dg(UL[q], UR[q], a.gamma, f);
        } else {
            // normal (y) momentum into slot 1, and back (src_DG/fluid.cpp:772-774)
            double l[4] = {UL[q][0], UL[q][2], UL[q][1], UL[q][3]};
            double r[4] = {UR[q][0], UR[q][2], UR[q][1], UR[q][3]};
            double g[4];
            if (a.hll) hlle_dg(l, r, a.gamma, g);
            else hllc_dg(l, r, a.gamma, g);
            f[0] = g[0]; f[1] = g[2]; f[2] = g[1]; f[3] = g[3];
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) F[(size_t)(q * 4 + c) * qstride + o] = f[c];
    }
}

template <int P, int DIR>
__global__ void __launch_bounds__(128) dg_face_kernel(DGArgs a) {
    face_row<P, DIR>(a, blockIdx.x * blockDim.x, blockIdx.y);
}

// applyLimiter for one cell held in registers (src_DG/fluid.cpp:824-992):
// Persson modal filter (bctype-0 cells only) then Zhang-Shu positivity.
template <int P>
__device__ __forceinline__ void limit_cell(double (&o)[4][(P + 1) * (P + 1)], bool persson, const DGTab& T,
                                           double gamma, double s0) {
    constexpr int NM = (P + 1) * (P + 1);
    const double kappa = 1.0, RHO_MIN = 1e-5, P_MIN = 1e-5, EPS = 1e-5;
    if (persson) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double Etot = 0.0, Ep = 0.0;
#pragma unroll
            for (int m = 0; m < NM; ++m) {
                const double x = o[c][m];
                Etot += x * x;
                if (m / (P + 1) == P || m % (P + 1) == P) Ep += x * x;
            }
            const double s = log10(Ep / (Etot + EPS));
            if (s > s0) {
                double eps;
                if (s > s0 + kappa) eps = 1.0;
                else {
                    const double r = (s - s0) / kappa;
                    eps = 0.5 * (1.0 + sin(M_PI * (r - 0.5)));
                }
#pragma unroll
                for (int m = 0; m < NM; ++m)
                    if (m / (P + 1) == P || m % (P + 1) == P) o[c][m] *= (1.0 - eps);
            }
        }
    }
    o[0][0] = ref_max(o[0][0], RHO_MIN);
    const double rho0 = o[0][0], mx0 = o[1][0], my0 = o[2][0];
    double E0 = o[3][0];
    const double p0 = (gamma - 1.0) * (E0 - 0.5 * (mx0 * mx0 + my0 * my0) / rho0);
    if (p0 < P_MIN) {
        E0 = P_MIN / (gamma - 1.0) + 0.5 * (mx0 * mx0 + my0 * my0) / rho0;
        o[3][0] = E0;
    }
    double theta_rho = 1.0;
#pragma unroll 1
    for (int pt = 0; pt < 16; ++pt) {
        double rho = 0.0;
#pragma unroll
        for (int m = 0; m < NM; ++m) rho += o[0][m] * T.zs[pt][m];
        if (rho < RHO_MIN) {
            const double t = (rho0 - RHO_MIN) / (rho0 - rho + EPS);
            theta_rho = ref_min(theta_rho, t);
        }
    }
    if (theta_rho < 1.0) {
#pragma unroll
        for (int m = 1; m < NM; ++m)
#pragma unroll
            for (int c = 0; c < 4; ++c) o[c][m] *= theta_rho;
    }
    double theta_p = 1.0;
#pragma unroll 1
    for (int pt = 0; pt < 16; ++pt) {
        double rho = 0.0, mx = 0.0, my = 0.0, E = 0.0;
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const double phi = T.zs[pt][m];
            rho += o[0][m] * phi;
            mx += o[1][m] * phi;
            my += o[2][m] * phi;
            E += o[3][m] * phi;
        }
        if (rho <= RHO_MIN) continue;
        const double u = mx / rho, v = my / rho;
        const double p = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        if (p < P_MIN) {
            const double p_avg = (gamma - 1.0) * (o[3][0] - 0.5 * (o[1][0] * o[1][0] + o[2][0] * o[2][0]) / o[0][0]);
            const double t = (p_avg - P_MIN) / (p_avg - p + EPS);
            theta_p = ref_min(theta_p, t);
        }
    }
    if (theta_p < 1.0) {
#pragma unroll
        for (int m = 1; m < NM; ++m)
#pragma unroll
            for (int c = 0; c < 4; ++c) o[c][m] *= theta_p;
    }
}

constexpr int kCellBlock = kDgCellBlock;

// Cells (i, jb + threadIdx.x); sd[v][threadIdx.x] is this thread's (filled)
// stage input, column-private.  Returns the cell's max corner wave speed when
// want_lam and the cell is fluid (computeMaxSpeedDG_omp), else 0.
template <int P>
__device__ __forceinline__ double cell_row(const DGArgs& a, int jb, int i,
                                           double (&sd)[4 * (P + 1) * (P + 1)][kCellBlock]) {
    constexpr int NQ = P + 1, NM = NQ * NQ, NV = NQ * NQ;
    const DGTab& T = c_dgtab[P - 1];
    const int t = threadIdx.x;
    const int j = jb + t;
    if (j >= a.g.nx) return 0.0;  // no block-wide synchronisation follows
    const int ny = a.g.ny, nx = a.g.nx;
    const size_t plane = a.g.plane, k = (size_t)i * a.g.pitch + j;
    const int8_t kd = a.kind[k] & KIND_MASK;
    const CellRef r = cell_ref(a, k);
#pragma unroll
    for (int v = 0; v < 4 * NM; ++v) {
        const double x = a.cur[(size_t)v * plane + r.k];
        sd[v][t] = (r.neg == v / NM) ? -x : x;
    }
    double o[4][NM];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int m = 0; m < NM; ++m) o[c][m] = 0.0;

    if (kd == KIND_UPDATED) {
        // volume integral (src_DG/fluid.cpp:698-718)
#pragma unroll 1
        for (int p = 0; p < NV; ++p) {
            double U[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int m = 0; m < NM; ++m) {
                const double b = T.vphi[p][m];
#pragma unroll
                for (int c = 0; c < 4; ++c) U[c] += sd[c * NM + m][t] * b;
            }
            double F[4], G[4];
            euler_flux(U, a.gamma, F, G);
            const double coeff = T.vw[p];
#pragma unroll
            for (int m = 0; m < NM; ++m) {
                const double dxi = T.vdxi[p][m], det = T.vdet[p][m];
#pragma unroll
                for (int c = 0; c < 4; ++c) o[c][m] += coeff * (F[c] * dxi + G[c] * det);
            }
        }
        // face integrals: right (-), left (+), bottom (-), top (+) (src_DG/fluid.cpp:731-796)
        const size_t xq = (size_t)ny * a.xpitch, yq = (size_t)(ny + 1) * a.g.pitch;
        const size_t xr = (size_t)i * a.xpitch + j + 1, xl = (size_t)i * a.xpitch + j;
        const size_t yd = (size_t)(i + 1) * a.g.pitch + j, yu = (size_t)i * a.g.pitch + j;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const double* Fb = (f < 2) ? a.fx : a.fy;
            const size_t qs = (f < 2) ? xq : yq;
            const size_t o_ = (f == 0) ? xr : (f == 1) ? xl : (f == 2) ? yd : yu;
            const bool minus = (f == 0 || f == 2);
#pragma unroll 1
            for (int q = 0; q < NQ; ++q) {
                double Fs[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) Fs[c] = Fb[(size_t)(q * 4 + c) * qs + o_];
#pragma unroll
                for (int m = 0; m < NM; ++m) {
                    const double bv = T.bv[f][q][m];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (minus) o[c][m] -= bv * Fs[c];
                        else o[c][m] += bv * Fs[c];
                    }
                }
            }
        }
        // inverse mass: (2px+1)(2py+1) * 0.5 / h (src_DG/fluid.cpp:800-804)
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const double scale = (double)((2 * (m / NQ) + 1) * (2 * (m % NQ) + 1)) * a.inv2h;
#pragma unroll
            for (int c = 0; c < 4; ++c) o[c][m] = o[c][m] * scale;
        }
    }

    if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 4 * NM; ++v) a.out[(size_t)v * plane + k] = o[v / NM][v % NM];
        return 0.0;
    }
    // Shu-Osher combine with dt applied (src_DG/fluid.cpp:1024-1026, 1036-1038, 1046-1048)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const size_t v = (size_t)(c * NM + m);
            const double dn = a.un[v * plane + k];
            const double dd = a.dt * o[c][m];
            if (a.stage == 1) o[c][m] = dn + dd;
            else if (a.stage == 2) o[c][m] = 0.75 * dn + 0.25 * (sd[v][t] + dd);
            else o[c][m] = (1.0 / 3.0) * dn + (2.0 / 3.0) * (sd[v][t] + dd);
        }
    if (a.limiter == ZK_LIMITER_REFERENCE && i >= 3 && i < ny - 3 && j >= 3 && j < nx - 3)
        limit_cell<P>(o, kd == KIND_UPDATED, T, a.gamma, a.s0);
    if (kd == KIND_UPDATED) {
        uint32_t flags = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (isnan(o[c][0])) flags |= STATUS_NAN;
        if (!(o[0][0] > 0.0)) flags |= STATUS_RHO;
        if (flags) atomicOr(a.status, flags);
    }
#pragma unroll
    for (int v = 0; v < 4 * NM; ++v) a.out[(size_t)v * plane + k] = o[v / NM][v % NM];
    if (!a.want_lam || !(a.kind[k] & KIND_FLUID)) return 0.0;
    double cs[4][4] = {};
#pragma unroll
    for (int m = 0; m < NM; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double b = a.phic[m * 4 + q];
#pragma unroll
            for (int c = 0; c < 4; ++c) cs[q][c] += o[c][m] * b;
        }
    return dg_cell_speed(cs, a.gamma, 0.0);
}

template <int P>
// at least 6 CTAs per SM (at most 168 registers): +4% on the P=3 stage over
// the 255-register build with 4 CTAs
__global__ void __launch_bounds__(kCellBlock, 6) dg_cell_kernel(DGArgs a) {
    __shared__ double sd[4 * (P + 1) * (P + 1)][kCellBlock];
    cell_row<P>(a, blockIdx.x * kCellBlock, blockIdx.y, sd);
}

// Stage-s arguments of batch item `it` (stage s reads U[s-1], writes U[s % 3]).
__device__ __forceinline__ DGArgs batch_args(const DgItem& it, int stage) {
    const BatchCtl* ctl = it.ctl;
    DGArgs a;
    a.cur = it.U[stage - 1];
    a.un = it.U[0];
    a.out = it.U[stage % 3];
    a.kind = it.kind;
    a.gsrc = it.gsrc;
    a.fx = it.fx;
    a.fy = it.fy;
    a.g = it.g;
    a.xpitch = it.xpitch;
    a.dt = ctl->dt;
    a.inv2h = it.inv2h;
    a.gamma = it.gamma;
    a.stage = stage;
    a.limiter = it.limiter;
    a.hll = it.hll;
    a.s0 = it.s0;
    a.status = &it.ctl->status;
    a.phic = it.phic;
    a.want_lam = stage == 3;
    return a;
}

// Persistent face pass of a batch group: a problem's tiles are its x-face
// rows (ny x ceil(nx/128) segments) followed by its y-face rows.
template <int P>
__global__ void __launch_bounds__(128) dg_faces_fp64_batch_kernel(const DgItem* __restrict__ items,
                                                                   const int* __restrict__ dir, int cap, int stage) {
    __shared__ DGArgs sa;
    __shared__ int s_job[4];  // stepping, direction, row, segment start
    const int total = __ldg(dir + 1);
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        if (threadIdx.x == 0) {
            const DirHit h = dir_lookup(dir, cap, t);
            const DgItem& it = items[h.item];
            s_job[0] = it.ctl->stepping;
            if (s_job[0]) {
                const int segs = (it.g.nx + 127) / 128, per = it.g.ny * segs;
                const int d = h.local >= per, r = h.local - d * per;
                s_job[1] = d;
                s_job[2] = r / segs;
                s_job[3] = (r - (r / segs) * segs) * 128;
                sa = batch_args(it, stage);
            }
        }
        __syncthreads();
        if (s_job[0]) {
            if (s_job[1] == 0) face_row<P, 0>(sa, s_job[3], s_job[2]);
            else face_row<P, 1>(sa, s_job[3], s_job[2]);
        }
        __syncthreads();
    }
}

// Persistent cell pass of a batch group: tiles are row segments of kCellBlock cells.
template <int P>
__global__ void __launch_bounds__(kCellBlock, 6) dg_cell_fp64_batch_kernel(const DgItem* __restrict__ items,
                                                                         const int* __restrict__ dir, int cap,
                                                                         int stage) {
    __shared__ double sd[4 * (P + 1) * (P + 1)][kCellBlock];
    __shared__ DGArgs sa;
    __shared__ int s_job[3];  // stepping, row, segment start
    __shared__ unsigned long long* s_lam;
    const int total = __ldg(dir + 1);
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        if (threadIdx.x == 0) {
            const DirHit h = dir_lookup(dir, cap, t);
            const DgItem& it = items[h.item];
            s_job[0] = it.ctl->stepping;
            if (s_job[0]) {
                const int segs = (it.g.nx + kCellBlock - 1) / kCellBlock;
                s_job[1] = h.local / segs;
                s_job[2] = (h.local - s_job[1] * segs) * kCellBlock;
                sa = batch_args(it, stage);
                s_lam = &it.ctl->lam;
            }
        }
        __syncthreads();
        if (s_job[0]) {
            const double m = cell_row<P>(sa, s_job[2], s_job[1], sd);
            if (stage == 3) block_max_commit_to(m, s_lam);  // the next step's wave speed
        }
        __syncthreads();
    }
}

// applyLimiter alone, in place on the state (src_DG/fluid.cpp:824-992).
template <int P>
__global__ void __launch_bounds__(kCellBlock) dg_limit_kernel(DGArgs a) {
    constexpr int NM = (P + 1) * (P + 1);
    const int j = blockIdx.x * kCellBlock + threadIdx.x, i = blockIdx.y;
    const int ny = a.g.ny, nx = a.g.nx;
    if (!(i >= 3 && i < ny - 3 && j >= 3 && j < nx - 3)) return;
    const size_t plane = a.g.plane, k = (size_t)i * a.g.pitch + j;
    double o[4][NM];
#pragma unroll
    for (int v = 0; v < 4 * NM; ++v) o[v / NM][v % NM] = a.out[(size_t)v * plane + k];
    limit_cell<P>(o, (a.kind[k] & KIND_MASK) == KIND_UPDATED, c_dgtab[P - 1], a.gamma, a.s0);
#pragma unroll
    for (int v = 0; v < 4 * NM; ++v) a.out[(size_t)v * plane + k] = o[v / NM][v % NM];
}

template <int P>
cudaError_t launch_stage(const DGArgs& a, cudaStream_t s) {
    const dim3 fb(128);
    dg_face_kernel<P, 0><<<dim3((a.g.nx + 127) / 128, a.g.ny), fb, 0, s>>>(a);
    dg_face_kernel<P, 1><<<dim3((a.g.nx + 127) / 128, a.g.ny), fb, 0, s>>>(a);
    dg_cell_kernel<P><<<dim3((a.g.nx + kCellBlock - 1) / kCellBlock, a.g.ny), kCellBlock, 0, s>>>(a);
    return cudaGetLastError();
}

template <int P>
cudaError_t launch_limit(const DGArgs& a, cudaStream_t s) {
    dg_limit_kernel<P><<<dim3((a.g.nx + kCellBlock - 1) / kCellBlock, a.g.ny), kCellBlock, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dg_stage_fp64(int P, const DGArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return launch_stage<1>(a, s);
        case 2: return launch_stage<2>(a, s);
        case 3: return launch_stage<3>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

// Batch tiles per problem: face pass 2 ny ceil(nx/128), cell pass ny ceil(nx/64).
int dg_fp64_batch_tiles(int pass, int ny, int nx) {
    return pass == 0 ? 2 * ny * ((nx + 127) / 128) : ny * ((nx + kCellBlock - 1) / kCellBlock);
}

template <int P>
cudaError_t launch_batch_p(const DgItem* items, const int* dir_face, const int* dir_cell, int cap, int stage,
                           int grid_face, int grid_cell, cudaStream_t s) {
    dg_faces_fp64_batch_kernel<P><<<grid_face, 128, 0, s>>>(items, dir_face, cap, stage);
    dg_cell_fp64_batch_kernel<P><<<grid_cell, kCellBlock, 0, s>>>(items, dir_cell, cap, stage);
    return cudaGetLastError();
}

// One FP64 DG stage of a batch group (face pass, then cell pass).
cudaError_t launch_dg_stage_fp64_batch(int P, const DgItem* items, const int* dir_face, const int* dir_cell, int cap,
                                       int stage, int grid_face, int grid_cell, cudaStream_t s) {
    switch (P) {
        case 1: return launch_batch_p<1>(items, dir_face, dir_cell, cap, stage, grid_face, grid_cell, s);
        case 2: return launch_batch_p<2>(items, dir_face, dir_cell, cap, stage, grid_face, grid_cell, s);
        case 3: return launch_batch_p<3>(items, dir_face, dir_cell, cap, stage, grid_face, grid_cell, s);
        default: return cudaErrorInvalidValue;
    }
}

// Resident CTAs per SM of the batch face (pass 0) and cell (pass 1) kernels.
int dg_fp64_batch_occupancy(int P, int pass) {
    int n = 0;
    switch (P * 2 + pass) {
        case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_faces_fp64_batch_kernel<1>, 128, 0); break;
        case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_cell_fp64_batch_kernel<1>, kCellBlock, 0); break;
        case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_faces_fp64_batch_kernel<2>, 128, 0); break;
        case 5: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_cell_fp64_batch_kernel<2>, kCellBlock, 0); break;
        case 6: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_faces_fp64_batch_kernel<3>, 128, 0); break;
        case 7: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dg_cell_fp64_batch_kernel<3>, kCellBlock, 0); break;
        default: break;
    }
    return n;
}

cudaError_t launch_dg_limit_fp64(int P, const DGArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return launch_limit<1>(a, s);
        case 2: return launch_limit<2>(a, s);
        case 3: return launch_limit<3>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ZK_FP64_NS
