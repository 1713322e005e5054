/* CPU oracle, discontinuous-Galerkin P=1..3 path: a C restatement of
 * src_DG/fluid.cpp and the dt rules of src_DG/solver.cpp.
 * TEST INFRASTRUCTURE ONLY (the checker, never shipped).
 *
 * Expressions follow the reference in the same evaluation order and are
 * compiled with -ffp-contract=off: bit-identical to the reference built with
 * -ffp-contract=off wherever no libm transcendental is involved (the limiter's
 * log10/sin are the only ones).
 *
 * Layout: dof[4][NM][ny][nx] row-major, NM=(P+1)^2, mode m = px*(P+1)+py. */
#include <stdlib.h>
#include <string.h>
#include "oracle_common.h"

#define OD_MAXNM 16

/* legP / legD, src_DG/fluid.cpp:34-55 */
static double legP(int n, double x) {
    switch (n) {
        case 0: return 1.0;
        case 1: return x;
        case 2: return 0.5 * (3.0 * x * x - 1.0);
        case 3: return 0.5 * (5.0 * x * x * x - 3.0 * x);
        case 4: return 0.125 * (35.0 * x * x * x * x - 30.0 * x * x + 3.0);
        default: return 0.0;
    }
}
static double legD(int n, double x) {
    switch (n) {
        case 0: return 0.0;
        case 1: return 1.0;
        case 2: return 3.0 * x;
        case 3: return 0.5 * (15.0 * x * x - 3.0);
        case 4: return 0.5 * (35.0 * x * x * x - 15.0 * x);
        default: return 0.0;
    }
}

/* Gauss-Legendre nodes/weights for NQ = 2..4, the decimal literals of
 * src_DG/fluid.cpp:94-111 (kept identical: the doubles they round to enter
 * every quadrature sum). */
static const double GL_PT[5][4] = {
    {0}, {0},
    {-0.5773502691896257, 0.5773502691896257, 0, 0},
    {-0.7745966692414834, 0.0, 0.7745966692414834, 0},
    {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526}};
static const double GL_WT[5][4] = {
    {0}, {0},
    {1.0, 1.0, 0, 0},
    {0.5555555555555556, 0.8888888888888888, 0.5555555555555556, 0},
    {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538}};

double od_phi2(int P, int m, double xi, double eta) {
    return legP(m / (P + 1), xi) * legP(m % (P + 1), eta);
}

/* eulerFluxX / eulerFluxY, src_DG/fluid.cpp:123-143 (floors 1e-3) */
static void flux_x(const double U[4], double F[4], double g) {
    const double eps = 1e-3;
    double rho = zk_max(U[0], eps);
    double u = U[1] / rho, v = U[2] / rho;
    double p = zk_max((g - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
    F[0] = rho * u; F[1] = rho * u * u + p; F[2] = rho * u * v; F[3] = (U[3] + p) * u;
}
static void flux_y(const double U[4], double G[4], double g) {
    const double eps = 1e-3;
    double rho = zk_max(U[0], eps);
    double u = U[1] / rho, v = U[2] / rho;
    double p = zk_max((g - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
    G[0] = rho * v; G[1] = rho * u * v; G[2] = rho * v * v + p; G[3] = (U[3] + p) * v;
}

/* hllcFlux (DG variant), src_DG/fluid.cpp:450-520: floors 1e-5, guarded
 * denominators, NaN/inf guard on the star-state energy term. */
void od_hllc(const double* L, const double* R, double gamma, double* F) {
    const double eps = 1e-5;
    double rhoL = zk_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3] / rhoL;
    double pL = zk_max((gamma - 1.0) * (L[3] - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(zk_max(gamma * pL / rhoL, eps));
    double rhoR = zk_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3] / rhoR;
    double pR = zk_max((gamma - 1.0) * (R[3] - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(zk_max(gamma * pR / rhoR, eps));
    double FL0 = rhoL * uL, FL1 = rhoL * uL * uL + pL, FL2 = rhoL * uL * vL, FL3 = (L[3] + pL) * uL;
    double FR0 = rhoR * uR, FR1 = rhoR * uR * uR + pR, FR2 = rhoR * uR * vR, FR3 = (R[3] + pR) * uR;
    double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    double den = sqL + sqR;
    if (den < eps) den = eps;
    double u_roe = (sqL * uL + sqR * uR) / den;
    double h_roe = (sqL * (EL + pL / rhoL) + sqR * (ER + pR / rhoR)) / den;
    double c_roe = sqrt(zk_max((gamma - 1.0) * (h_roe - 0.5 * u_roe * u_roe), eps));
    double SL = zk_min(uL - aL, u_roe - c_roe);
    double SR = zk_max(uR + aR, u_roe + c_roe);
    if (SL >= 0.0) { F[0] = FL0; F[1] = FL1; F[2] = FL2; F[3] = FL3; return; }
    if (SR <= 0.0) { F[0] = FR0; F[1] = FR1; F[2] = FR2; F[3] = FR3; return; }
    double num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    double den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabs(den2) < eps) den2 = (den2 >= 0 ? eps : -eps);
    double Ss = num / den2;
    const int left = (Ss >= 0.0);
    const double rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const double E = left ? EL : ER, p = left ? pL : pR, S = left ? SL : SR;
    double denom = S - Ss;
    if (fabs(denom) < eps) denom = (denom >= 0 ? eps : -eps);
    double c = rho * (S - u) / denom;
    double term = (Ss - u) * (Ss + p / (rho * (S - u)));
    if (isnan(term) || isinf(term)) term = 0.0;
    double s0 = c, s1 = c * Ss, s2 = c * v, s3 = c * (E + term);
    if (left) {
        F[0] = FL0 + SL * (s0 - L[0]); F[1] = FL1 + SL * (s1 - L[1]);
        F[2] = FL2 + SL * (s2 - L[2]); F[3] = FL3 + SL * (s3 - L[3]);
    } else {
        F[0] = FR0 + SR * (s0 - R[0]); F[1] = FR1 + SR * (s1 - R[1]);
        F[2] = FR2 + SR * (s2 - R[2]); F[3] = FR3 + SR * (s3 - R[3]);
    }
}

/* hlleFlux, src_DG/fluid.cpp:525-580 (defined, never called by the reference). */
void od_hlle(const double* L, const double* R, double gamma, double* F) {
    const double eps = 1e-6;
    double rhoL = zk_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3];
    double pL = zk_max((gamma - 1.0) * (EL - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(zk_max(gamma * pL / rhoL, eps));
    double HL = (EL + pL) / rhoL;
    double rhoR = zk_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3];
    double pR = zk_max((gamma - 1.0) * (ER - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(zk_max(gamma * pR / rhoR, eps));
    double HR = (ER + pR) / rhoR;
    double sqL = sqrt(rhoL), sqR = sqrt(rhoR);
    double invDen = 1.0 / zk_max(sqL + sqR, eps);
    double u_roe = (sqL * uL + sqR * uR) * invDen;
    double v_roe = (sqL * vL + sqR * vR) * invDen;
    double h_roe = (sqL * HL + sqR * HR) * invDen;
    double c_roe = sqrt(zk_max((gamma - 1.0) * (h_roe - 0.5 * (u_roe * u_roe + v_roe * v_roe)), eps));
    double SL = zk_min(uL - aL, u_roe - c_roe);
    double SR = zk_max(uR + aR, u_roe + c_roe);
    double FL0 = rhoL * uL, FL1 = rhoL * uL * uL + pL, FL2 = rhoL * uL * vL, FL3 = (EL + pL) * uL;
    double FR0 = rhoR * uR, FR1 = rhoR * uR * uR + pR, FR2 = rhoR * uR * vR, FR3 = (ER + pR) * uR;
    if (SL >= 0.0) { F[0] = FL0; F[1] = FL1; F[2] = FL2; F[3] = FL3; }
    else if (SR <= 0.0) { F[0] = FR0; F[1] = FR1; F[2] = FR2; F[3] = FR3; }
    else {
        double invDiff = 1.0 / zk_max(SR - SL, eps);
        F[0] = (SR * FL0 - SL * FR0 + SL * SR * (R[0] - L[0])) * invDiff;
        F[1] = (SR * FL1 - SL * FR1 + SL * SR * (R[1] - L[1])) * invDiff;
        F[2] = (SR * FL2 - SL * FR2 + SL * SR * (R[2] - L[2])) * invDiff;
        F[3] = (SR * FL3 - SL * FR3 + SL * SR * (R[3] - L[3])) * invDiff;
    }
}

typedef void (*riemann_fn)(const double*, const double*, double, double*);

typedef struct {
    int P, NM, NQ, ny, nx;
    size_t plane;
    signed char* kind;
    int* src;
} od_ctx;

static od_ctx ctx_new(int P, int ny, int nx, const int* bct, int periodic) {
    od_ctx c;
    c.P = P; c.NM = (P + 1) * (P + 1); c.NQ = P + 1; c.ny = ny; c.nx = nx;
    c.plane = (size_t)ny * nx;
    c.kind = (signed char*)malloc(c.plane);
    c.src = (int*)malloc(sizeof(int) * c.plane);
    zk_ghost_map(ny, nx, bct, 1, periodic, c.kind, c.src);
    return c;
}
static void ctx_free(od_ctx* c) { free(c->kind); free(c->src); }

#define DOF(d, c, m, k) (d)[((size_t)(c) * NM + (m)) * plane + (k)]

/* fillDGGhostCells, src_DG/fluid.cpp:581-635, as a gather over the source map. */
static void fill_ghosts(const od_ctx* x, double* d) {
    const int NM = x->NM;
    const size_t plane = x->plane;
    for (size_t k = 0; k < plane; ++k) {
        const int s = x->src[k];
        if (s < 0) continue;
        for (int c = 0; c < 4; ++c) {
            const int neg = (x->kind[k] == ZK_CELL_SLIP_X && c == 1) || (x->kind[k] == ZK_CELL_SLIP_Y && c == 2);
            for (int m = 0; m < NM; ++m) {
                const double v = DOF(d, c, m, (size_t)s);
                DOF(d, c, m, k) = neg ? -v : v;
            }
        }
    }
}

/* evalU, src_DG/fluid.cpp:672-681 */
static void eval_u(const od_ctx* x, const double* d, size_t k, double xi, double eta, double U[4]) {
    const int NM = x->NM;
    const size_t plane = x->plane;
    U[0] = U[1] = U[2] = U[3] = 0.0;
    for (int m = 0; m < NM; ++m) {
        double b = od_phi2(x->P, m, xi, eta);
        U[0] += DOF(d, 0, m, k) * b;
        U[1] += DOF(d, 1, m, k) * b;
        U[2] += DOF(d, 2, m, k) * b;
        U[3] += DOF(d, 3, m, k) * b;
    }
}

/* computeRHS, src_DG/fluid.cpp:656-807, for one fluid cell k. */
static void cell_rhs(const od_ctx* x, const double* d, size_t k, double h, double gam,
                     riemann_fn flux, double out[4][OD_MAXNM]) {
    const int P = x->P, NM = x->NM, NQ = x->NQ, nx = x->nx;
    const double* PT = GL_PT[NQ];
    const double* WT = GL_WT[NQ];
    double rhs[4][OD_MAXNM];
    memset(rhs, 0, sizeof(rhs));
    /* volume integral (:698-718) */
    for (int qa = 0; qa < NQ; ++qa) {
        double xi = PT[qa], wa = WT[qa];
        for (int qb = 0; qb < NQ; ++qb) {
            double eta = PT[qb], wb = WT[qb], ww = wa * wb;
            double U[4], F[4], G[4];
            eval_u(x, d, k, xi, eta, U);
            flux_x(U, F, gam);
            flux_y(U, G, gam);
            for (int m = 0; m < NM; ++m) {
                double dxi = legD(m / (P + 1), xi) * legP(m % (P + 1), eta);
                double det = legP(m / (P + 1), xi) * legD(m % (P + 1), eta);
                double coeff = ww;
                for (int c = 0; c < 4; ++c) rhs[c][m] += coeff * (F[c] * dxi + G[c] * det);
            }
        }
    }
    /* right face xi=+1, neighbour (i, j+1) (:731-744) */
    for (int q = 0; q < NQ; ++q) {
        double eta = PT[q], w = WT[q], UL[4], UR[4], Fs[4];
        eval_u(x, d, k, +1.0, eta, UL);
        eval_u(x, d, k + 1, -1.0, eta, UR);
        flux(UL, UR, gam, Fs);
        for (int m = 0; m < NM; ++m) {
            double bv = od_phi2(P, m, +1.0, eta) * w;
            for (int c = 0; c < 4; ++c) rhs[c][m] -= bv * Fs[c];
        }
    }
    /* left face xi=-1, neighbour (i, j-1) (:747-760) */
    for (int q = 0; q < NQ; ++q) {
        double eta = PT[q], w = WT[q], UL[4], UR[4], Fs[4];
        eval_u(x, d, k - 1, +1.0, eta, UL);
        eval_u(x, d, k, -1.0, eta, UR);
        flux(UL, UR, gam, Fs);
        for (int m = 0; m < NM; ++m) {
            double bv = od_phi2(P, m, -1.0, eta) * w;
            for (int c = 0; c < 4; ++c) rhs[c][m] += bv * Fs[c];
        }
    }
    /* bottom face eta=+1, neighbour (i+1, j); momentum swapped (:765-780) */
    for (int q = 0; q < NQ; ++q) {
        double xi = PT[q], w = WT[q], UL[4], UR[4], Gs[4];
        eval_u(x, d, k, xi, +1.0, UL);
        eval_u(x, d, k + (size_t)nx, xi, -1.0, UR);
        double a[4] = {UL[0], UL[2], UL[1], UL[3]}, b[4] = {UR[0], UR[2], UR[1], UR[3]};
        flux(a, b, gam, Gs);
        double G[4] = {Gs[0], Gs[2], Gs[1], Gs[3]};
        for (int m = 0; m < NM; ++m) {
            double bv = od_phi2(P, m, xi, +1.0) * w;
            for (int c = 0; c < 4; ++c) rhs[c][m] -= bv * G[c];
        }
    }
    /* top face eta=-1, neighbour (i-1, j) (:783-796) */
    for (int q = 0; q < NQ; ++q) {
        double xi = PT[q], w = WT[q], UL[4], UR[4], Gs[4];
        eval_u(x, d, k - (size_t)nx, xi, +1.0, UL);
        eval_u(x, d, k, xi, -1.0, UR);
        double a[4] = {UL[0], UL[2], UL[1], UL[3]}, b[4] = {UR[0], UR[2], UR[1], UR[3]};
        flux(a, b, gam, Gs);
        double G[4] = {Gs[0], Gs[2], Gs[1], Gs[3]};
        for (int m = 0; m < NM; ++m) {
            double bv = od_phi2(P, m, xi, -1.0) * w;
            for (int c = 0; c < 4; ++c) rhs[c][m] += bv * G[c];
        }
    }
    /* diagonal inverse mass (:800-804) */
    const double inv2h = 0.5 / h;
    for (int m = 0; m < NM; ++m) {
        double scale = (double)((2 * (m / (P + 1)) + 1) * (2 * (m % (P + 1)) + 1)) * inv2h;
        for (int c = 0; c < 4; ++c) out[c][m] = rhs[c][m] * scale;
    }
}

static void rhs_all(const od_ctx* x, double h, double gam, double* d, int hll, double* dU) {
    const int NM = x->NM;
    const size_t plane = x->plane;
    fill_ghosts(x, d);
    memset(dU, 0, sizeof(double) * 4 * NM * plane);
    for (size_t k = 0; k < plane; ++k) {
        if (x->kind[k] != ZK_CELL_UPDATED) continue;
        double o[4][OD_MAXNM];
        cell_rhs(x, d, k, h, gam, hll ? od_hlle : od_hllc, o);
        for (int c = 0; c < 4; ++c)
            for (int m = 0; m < NM; ++m) DOF(dU, c, m, k) = o[c][m];
    }
}

/* applyLimiter, src_DG/fluid.cpp:824-992: Persson modal filter on bctype-0
 * cells, then the Zhang-Shu positivity limiter on every cell of [3,n-3)^2
 * (bctype ignored) at 4x4 Gauss points, with the basis that drops cubic
 * factors (src_DG/fluid.cpp:808-823). */
static double zs_basis(int P, int m, double xi, double eta) {
    int px = m / (P + 1), py = m % (P + 1);
    double a = (px == 0) ? 1.0 : (px == 1) ? xi : (px == 2) ? 0.5 * (3.0 * xi * xi - 1.0) : 0.0;
    double b = (py == 0) ? 1.0 : (py == 1) ? eta : (py == 2) ? 0.5 * (3.0 * eta * eta - 1.0) : 0.0;
    return a * b;
}

static void limit_all(const od_ctx* x, const int* bct, double gamma, double* d) {
    const int P = x->P, NM = x->NM, ny = x->ny, nx = x->nx;
    const size_t plane = x->plane;
    const double kappa = 1.0;
    double s0 = (P >= 3) ? -3.0 * log10((double)P) : -4.0 * log10((double)P);
    const double RHO_MIN = 1e-5, P_MIN = 1e-5, EPS = 1e-5;
    for (int i = 3; i < ny - 3; ++i)
        for (int j = 3; j < nx - 3; ++j) {
            const size_t k = (size_t)i * nx + j;
            if (bct[k] != 0) continue;
            for (int c = 0; c < 4; ++c) {
                double Etot = 0.0, Ep = 0.0;
                for (int px = 0; px <= P; ++px)
                    for (int py = 0; py <= P; ++py) {
                        double a = DOF(d, c, px * (P + 1) + py, k);
                        Etot += a * a;
                        if (px == P || py == P) Ep += a * a;
                    }
                double s = log10(Ep / (Etot + EPS));
                if (s > s0) {
                    double eps;
                    if (s > s0 + kappa) eps = 1.0;
                    else {
                        double r = (s - s0) / kappa;
                        eps = 0.5 * (1.0 + sin(M_PI * (r - 0.5)));
                    }
                    for (int px = 0; px <= P; ++px)
                        for (int py = 0; py <= P; ++py)
                            if (px == P || py == P) DOF(d, c, px * (P + 1) + py, k) *= (1.0 - eps);
                }
            }
        }
    static const double gp[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563,
                                 0.8611363115940526};
    for (int i = 3; i < ny - 3; ++i)
        for (int j = 3; j < nx - 3; ++j) {
            const size_t k = (size_t)i * nx + j;
            DOF(d, 0, 0, k) = zk_max(DOF(d, 0, 0, k), RHO_MIN);
            double rho0 = DOF(d, 0, 0, k), mx0 = DOF(d, 1, 0, k), my0 = DOF(d, 2, 0, k);
            double E0 = DOF(d, 3, 0, k);
            double p0 = (gamma - 1.0) * (E0 - 0.5 * (mx0 * mx0 + my0 * my0) / rho0);
            if (p0 < P_MIN) {
                E0 = P_MIN / (gamma - 1.0) + 0.5 * (mx0 * mx0 + my0 * my0) / rho0;
                DOF(d, 3, 0, k) = E0;
            }
            double theta_rho = 1.0;
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) {
                    double rho = 0.0;
                    for (int m = 0; m < NM; ++m) rho += DOF(d, 0, m, k) * zs_basis(P, m, gp[a], gp[b]);
                    if (rho < RHO_MIN) {
                        double t = (rho0 - RHO_MIN) / (rho0 - rho + EPS);
                        theta_rho = zk_min(theta_rho, t);
                    }
                }
            if (theta_rho < 1.0)
                for (int m = 1; m < NM; ++m)
                    for (int c = 0; c < 4; ++c) DOF(d, c, m, k) *= theta_rho;
            double theta_p = 1.0;
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) {
                    double rho = 0.0, mx = 0.0, my = 0.0, E = 0.0;
                    for (int m = 0; m < NM; ++m) {
                        double phi = zs_basis(P, m, gp[a], gp[b]);
                        rho += DOF(d, 0, m, k) * phi;
                        mx += DOF(d, 1, m, k) * phi;
                        my += DOF(d, 2, m, k) * phi;
                        E += DOF(d, 3, m, k) * phi;
                    }
                    if (rho <= RHO_MIN) continue;
                    double u = mx / rho, v = my / rho;
                    double p = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
                    if (p < P_MIN) {
                        double p_avg = (gamma - 1.0) * (DOF(d, 3, 0, k) -
                                                        0.5 * (DOF(d, 1, 0, k) * DOF(d, 1, 0, k) +
                                                               DOF(d, 2, 0, k) * DOF(d, 2, 0, k)) /
                                                            DOF(d, 0, 0, k));
                        double t = (p_avg - P_MIN) / (p_avg - p + EPS);
                        theta_p = zk_min(theta_p, t);
                    }
                }
            if (theta_p < 1.0)
                for (int m = 1; m < NM; ++m)
                    for (int c = 0; c < 4; ++c) DOF(d, c, m, k) *= theta_p;
        }
}

/* ---- exported entry points ------------------------------------------------ */

int od_rhs(int P, int ny, int nx, double da, double gamma, double* dof, const int* bct,
           int periodic, int hll, double* dU) {
    if (P < 1 || P > 3) return 1;
    od_ctx x = ctx_new(P, ny, nx, bct, periodic);
    rhs_all(&x, da, gamma, dof, hll, dU);
    ctx_free(&x);
    return 0;
}

int od_limit(int P, int ny, int nx, double gamma, double* dof, const int* bct) {
    if (P < 1 || P > 3) return 1;
    od_ctx x = ctx_new(P, ny, nx, bct, 0);
    limit_all(&x, bct, gamma, dof);
    ctx_free(&x);
    return 0;
}

/* updateMesh, src_DG/fluid.cpp:1005-1054: per stage RHS (with ghost fill),
 * combine with dt applied, then the limiter. */
int od_step(int P, int ny, int nx, double da, double gamma, double* dof, const int* bct, double dt,
            int nsteps, int periodic, int hll) {
    if (P < 1 || P > 3) return 1;
    od_ctx x = ctx_new(P, ny, nx, bct, periodic);
    const size_t n = (size_t)4 * x.NM * x.plane;
    double* dn = (double*)malloc(sizeof(double) * n);
    double* dU = (double*)malloc(sizeof(double) * n);
    for (int s = 0; s < nsteps; ++s) {
        memcpy(dn, dof, sizeof(double) * n);
        rhs_all(&x, da, gamma, dof, hll, dU);
        for (size_t k = 0; k < n; ++k) dof[k] = dn[k] + dt * dU[k];
        limit_all(&x, bct, gamma, dof);
        rhs_all(&x, da, gamma, dof, hll, dU);
        for (size_t k = 0; k < n; ++k) dof[k] = 0.75 * dn[k] + 0.25 * (dof[k] + dt * dU[k]);
        limit_all(&x, bct, gamma, dof);
        rhs_all(&x, da, gamma, dof, hll, dU);
        for (size_t k = 0; k < n; ++k) dof[k] = (1.0 / 3.0) * dn[k] + (2.0 / 3.0) * (dof[k] + dt * dU[k]);
        limit_all(&x, bct, gamma, dof);
    }
    free(dn); free(dU);
    ctx_free(&x);
    return 0;
}

/* computeMaxSpeedDG_omp, src_DG/solver.cpp:26-64: bctype-0 cells (whole grid),
 * state at the 4 cell corners, floors 1e-12. */
double od_max_speed(int P, int ny, int nx, double gamma, const double* dof, const int* bct) {
    const int NM = (P + 1) * (P + 1);
    const size_t plane = (size_t)ny * nx;
    const double XI[4] = {-1.0, +1.0, -1.0, +1.0}, ETA[4] = {-1.0, -1.0, +1.0, +1.0};
    double PHI[OD_MAXNM][4];
    for (int m = 0; m < NM; ++m)
        for (int q = 0; q < 4; ++q) PHI[m][q] = od_phi2(P, m, XI[q], ETA[q]);
    const double eps = 1e-12;
    double umax = 0.0;
    for (size_t k = 0; k < plane; ++k) {
        if (bct[k] != 0) continue;
        for (int q = 0; q < 4; ++q) {
            double U[4] = {0.0, 0.0, 0.0, 0.0};
            for (int m = 0; m < NM; ++m) {
                double b = PHI[m][q];
                U[0] += DOF(dof, 0, m, k) * b;
                U[1] += DOF(dof, 1, m, k) * b;
                U[2] += DOF(dof, 2, m, k) * b;
                U[3] += DOF(dof, 3, m, k) * b;
            }
            double rho = zk_max(U[0], eps), u = U[1] / rho, v = U[2] / rho;
            double p = zk_max((gamma - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
            double a = sqrt(gamma * p / rho);
            umax = zk_max(umax, sqrt(u * u + v * v) + a);
        }
    }
    return umax;
}

/* dgSafeDt, src_DG/solver.cpp:15-23 */
double od_safe_dt(int P, double lambda_max, double h) {
    return 0.9 / (2.0 * (2 * P + 1)) * h / zk_max(lambda_max, 1e-7);
}

/* initDGModes, src_DG/fluid.cpp:173-182: mode 0 = the cell value, others 0. */
void od_init_modes(int P, int ny, int nx, const double* U, double* dof) {
    const int NM = (P + 1) * (P + 1);
    const size_t plane = (size_t)ny * nx;
    memset(dof, 0, sizeof(double) * 4 * NM * plane);
    for (int c = 0; c < 4; ++c) memcpy(&DOF(dof, c, 0, 0), U + c * plane, sizeof(double) * plane);
}

/* ---- TVB limiter (no reference implementation) ------------------------------
 * Cockburn & Shu (2001, J. Sci. Comput. 16; cited in the reference README) TVB
 * minmod limiting of the linear modes with characteristic decomposition, in
 * the form the reference's own header documents for its DG limiter
 * (src_DG/fluid.h:140-147: minmod on u_{1,0}, u_{0,1}; if limited, the modes
 * with px+py > 1 are set to zero).  Per bctype-0 cell in the update range:
 *   slopes  a_x = mode (1,0), a_y = mode (0,1); mean differences to the
 *           neighbours (filled through the ghost map) D+ and D-;
 *   in characteristic variables of the mean state (x or y eigenvectors),
 *   w~ = m~(w, w+, w-) with m~(a,b,c) = a if |a| <= M h^2 else minmod(a,b,c);
 *   a cell is troubled when any w~ differs from w; a troubled cell gets the
 *   limited linear modes (R w~) and zero higher modes.
 * Cell means are never modified, so the pass reads neighbour means from the
 * same array it writes (a Jacobi sweep). */

/* Left (L) and right (R) eigenvectors of the Euler flux Jacobian in direction
 * dir (0 = x, 1 = y) at conserved state u; returns 0 for a non-physical state. */
int od_euler_eigen(const double u[4], double gamma, int dir, double L[4][4], double R[4][4]) {
    const double rho = u[0];
    if (!(rho > 0.0)) return 0;
    const double vx = u[1] / rho, vy = u[2] / rho;
    const double q2 = vx * vx + vy * vy;
    const double p = (gamma - 1.0) * (u[3] - 0.5 * rho * q2);
    if (!(p > 0.0)) return 0;
    const double c = sqrt(gamma * p / rho);
    const double H = (u[3] + p) / rho;
    const double b1 = (gamma - 1.0) / (c * c), b2 = 0.5 * q2 * b1;
    const double un = dir == 0 ? vx : vy;   /* normal velocity */
    const double ut = dir == 0 ? vy : vx;   /* tangential velocity */
    const int in = dir == 0 ? 1 : 2, it = dir == 0 ? 2 : 1;  /* momentum slots */
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) L[r][k] = R[r][k] = 0.0;
    /* right eigenvectors as columns: (un-c), (un) entropy, (un) shear, (un+c) */
    R[0][0] = 1.0; R[in][0] = un - c; R[it][0] = ut; R[3][0] = H - un * c;
    R[0][1] = 1.0; R[in][1] = un;     R[it][1] = ut; R[3][1] = 0.5 * q2;
    R[0][2] = 0.0; R[in][2] = 0.0;    R[it][2] = 1.0; R[3][2] = ut;
    R[0][3] = 1.0; R[in][3] = un + c; R[it][3] = ut; R[3][3] = H + un * c;
    /* left eigenvectors as rows (L = R^-1) */
    L[0][0] = 0.5 * (b2 + un / c); L[0][in] = -0.5 * (b1 * un + 1.0 / c); L[0][it] = -0.5 * b1 * ut; L[0][3] = 0.5 * b1;
    L[1][0] = 1.0 - b2;            L[1][in] = b1 * un;                    L[1][it] = b1 * ut;         L[1][3] = -b1;
    L[2][0] = -ut;                 L[2][in] = 0.0;                        L[2][it] = 1.0;             L[2][3] = 0.0;
    L[3][0] = 0.5 * (b2 - un / c); L[3][in] = -0.5 * (b1 * un - 1.0 / c); L[3][it] = -0.5 * b1 * ut; L[3][3] = 0.5 * b1;
    return 1;
}

static double tvb_minmod(double a, double b, double c, double mh2) {
    if (fabs(a) <= mh2) return a;
    if (a > 0.0 && b > 0.0 && c > 0.0) return zk_min(a, zk_min(b, c));
    if (a < 0.0 && b < 0.0 && c < 0.0) return zk_max(a, zk_max(b, c));
    return 0.0;
}

/* Limit one direction: slope a[4] against D+ dp[4] and D- dm[4] at mean ub.
 * Returns 1 (troubled) and writes the limited slope, else 0. */
static int tvb_dir(const double ub[4], double gamma, int dir, double mh2, const double a[4],
                   const double dp[4], const double dm[4], double out[4]) {
    double L[4][4], R[4][4];
    const int phys = od_euler_eigen(ub, gamma, dir, L, R);
    double w[4], wp[4], wm[4], wl[4];
    for (int r = 0; r < 4; ++r) {
        if (phys) {
            w[r] = L[r][0] * a[0] + L[r][1] * a[1] + L[r][2] * a[2] + L[r][3] * a[3];
            wp[r] = L[r][0] * dp[0] + L[r][1] * dp[1] + L[r][2] * dp[2] + L[r][3] * dp[3];
            wm[r] = L[r][0] * dm[0] + L[r][1] * dm[1] + L[r][2] * dm[2] + L[r][3] * dm[3];
        } else {
            w[r] = a[r]; wp[r] = dp[r]; wm[r] = dm[r];   /* component-wise fallback */
        }
    }
    int changed = 0;
    for (int r = 0; r < 4; ++r) {
        wl[r] = tvb_minmod(w[r], wp[r], wm[r], mh2);
        if (wl[r] != w[r]) changed = 1;
    }
    if (!changed) return 0;
    for (int r = 0; r < 4; ++r)
        out[r] = phys ? R[r][0] * wl[0] + R[r][1] * wl[1] + R[r][2] * wl[2] + R[r][3] * wl[3] : wl[r];
    return 1;
}

/* Mean (mode 0) of cell k's neighbour, gathered through the fill map. */
static void nb_mean(const od_ctx* x, const double* d, size_t k, double out[4]) {
    const int NM = x->NM;
    const size_t plane = x->plane;
    size_t s = k;
    int neg = -1;
    if (x->src[k] >= 0) {
        s = (size_t)x->src[k];
        neg = x->kind[k] == ZK_CELL_SLIP_X ? 1 : (x->kind[k] == ZK_CELL_SLIP_Y ? 2 : -1);
    }
    for (int c = 0; c < 4; ++c) {
        const double v = DOF(d, c, 0, s);
        out[c] = (neg == c) ? -v : v;
    }
}

static void limit_tvb_all(const od_ctx* x, double da, double gamma, double M, double* d, unsigned char* flags) {
    const int P = x->P, NM = x->NM, nx = x->nx;
    const size_t plane = x->plane;
    const double mh2 = M * da * da;
    const int mx = P + 1, my = 1;  /* modes (px,py) = (1,0) and (0,1) */
    for (size_t k = 0; k < plane; ++k) {
        if (flags) flags[k] = 0;
        if (x->kind[k] != ZK_CELL_UPDATED) continue;
        double ub[4], uL[4], uR[4], uU[4], uD[4];
        for (int c = 0; c < 4; ++c) ub[c] = DOF(d, c, 0, k);
        nb_mean(x, d, k - 1, uL);
        nb_mean(x, d, k + 1, uR);
        nb_mean(x, d, k - (size_t)nx, uU);
        nb_mean(x, d, k + (size_t)nx, uD);
        double ax[4], ay[4], dxp[4], dxm[4], dyp[4], dym[4], lx[4], ly[4];
        for (int c = 0; c < 4; ++c) {
            ax[c] = DOF(d, c, mx, k);
            ay[c] = DOF(d, c, my, k);
            dxp[c] = uR[c] - ub[c];
            dxm[c] = ub[c] - uL[c];
            dyp[c] = uD[c] - ub[c];  /* eta grows with the row index */
            dym[c] = ub[c] - uU[c];
        }
        const int tx = tvb_dir(ub, gamma, 0, mh2, ax, dxp, dxm, lx);
        const int ty = tvb_dir(ub, gamma, 1, mh2, ay, dyp, dym, ly);
        if (!(tx || ty)) continue;
        if (flags) flags[k] = 1;
        for (int c = 0; c < 4; ++c) {
            if (tx) DOF(d, c, mx, k) = lx[c];
            if (ty) DOF(d, c, my, k) = ly[c];
            for (int m = 0; m < NM; ++m)
                if (m / (P + 1) + m % (P + 1) > 1) DOF(d, c, m, k) = 0.0;
        }
    }
}

/* One TVB pass on the state (ghost map built from bct; periodic ring -3). */
int od_limit_tvb(int P, int ny, int nx, double da, double gamma, double* dof, const int* bct, double M,
                 int periodic, unsigned char* flags) {
    if (P < 1 || P > 3) return 1;
    od_ctx x = ctx_new(P, ny, nx, bct, periodic);
    limit_tvb_all(&x, da, gamma, M, dof, flags);
    ctx_free(&x);
    return 0;
}

/* updateMesh with a selectable limiter after each stage:
 * 0 = reference (Persson + Zhang-Shu), 1 = none, 2 = TVB(M). */
int od_step_lim(int P, int ny, int nx, double da, double gamma, double* dof, const int* bct, double dt,
                int nsteps, int periodic, int hll, int limiter, double M) {
    if (P < 1 || P > 3) return 1;
    od_ctx x = ctx_new(P, ny, nx, bct, periodic);
    const size_t n = (size_t)4 * x.NM * x.plane;
    double* dn = (double*)malloc(sizeof(double) * n);
    double* dU = (double*)malloc(sizeof(double) * n);
    for (int s = 0; s < nsteps; ++s) {
        memcpy(dn, dof, sizeof(double) * n);
        for (int stage = 1; stage <= 3; ++stage) {
            rhs_all(&x, da, gamma, dof, hll, dU);
            for (size_t k = 0; k < n; ++k) {
                if (stage == 1) dof[k] = dn[k] + dt * dU[k];
                else if (stage == 2) dof[k] = 0.75 * dn[k] + 0.25 * (dof[k] + dt * dU[k]);
                else dof[k] = (1.0 / 3.0) * dn[k] + (2.0 / 3.0) * (dof[k] + dt * dU[k]);
            }
            if (limiter == 0) limit_all(&x, bct, gamma, dof);
            else if (limiter == 2) limit_tvb_all(&x, da, gamma, M, dof, NULL);
        }
    }
    free(dn); free(dU);
    ctx_free(&x);
    return 0;
}
