/* CPU oracle, WENO5 + HLLC + SSP-RK3 finite-volume path: a C restatement of
 * src_WENO/fluid.cpp.  TEST INFRASTRUCTURE ONLY (the checker, never shipped).
 *
 * Arithmetic follows the reference expression by expression, in the same
 * evaluation order, and is compiled with -ffp-contract=off, so it is
 * bit-identical to the reference built with -ffp-contract=off
 * (oracle/_ref/libref_weno_strict.so) and to the GPU FP64 path built with
 * --fmad=false.  The parity tests pin it against the reference build.
 *
 * Layout: U[4][ny][nx] row-major (row = y, row 0 on top), bct int32[ny][nx]. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_common.h"

/* weno5_reconstruct, src_WENO/fluid.cpp:230-263.  Stencil a..f = cells
 * i-2..i+3; returns the left-biased (ul) and right-biased (ur) states at i+1/2. */
void ow_weno5(double UL2, double UL1, double UP, double UR1, double UR2, double UR3, double* ul,
              double* ur) {
    const double eps = 1e-6, C1 = 13.0 / 12.0, C2 = 0.25;
    double qL0 = (1.0 / 3.0) * UL2 - (7.0 / 6.0) * UL1 + (11.0 / 6.0) * UP;
    double qL1 = -(1.0 / 6.0) * UL1 + (5.0 / 6.0) * UP + (1.0 / 3.0) * UR1;
    double qL2 = (1.0 / 3.0) * UP + (5.0 / 6.0) * UR1 - (1.0 / 6.0) * UR2;
    double d0 = UL2 - 2 * UL1 + UP, d1 = UL2 - 4 * UL1 + 3 * UP;
    double d2 = UL1 - 2 * UP + UR1, d3 = UL1 - UR1;
    double d4 = UP - 2 * UR1 + UR2, d5 = 3 * UP - 4 * UR1 + UR2;
    double b0 = C1 * d0 * d0 + C2 * d1 * d1, b1 = C1 * d2 * d2 + C2 * d3 * d3,
           b2 = C1 * d4 * d4 + C2 * d5 * d5;
    double t0 = eps + b0, t1 = eps + b1, t2 = eps + b2;
    double a0 = 0.1 / (t0 * t0), a1 = 0.6 / (t1 * t1), a2 = 0.3 / (t2 * t2);
    double inv = 1.0 / (a0 + a1 + a2);
    *ul = (a0 * qL0 + a1 * qL1 + a2 * qL2) * inv;

    double qR0 = (11.0 / 6.0) * UR1 - (7.0 / 6.0) * UR2 + (1.0 / 3.0) * UR3;
    double qR1 = (1.0 / 3.0) * UP + (5.0 / 6.0) * UR1 - (1.0 / 6.0) * UR2;
    double qR2 = -(1.0 / 6.0) * UL1 + (5.0 / 6.0) * UP + (1.0 / 3.0) * UR1;
    double r0 = UR1 - 2 * UR2 + UR3, r1 = 3 * UR1 - 4 * UR2 + UR3;
    double r2 = UP - 2 * UR1 + UR2, r3 = UP - UR2;
    double r4 = UL1 - 2 * UP + UR1, r5 = UL1 - 4 * UP + 3 * UR1;
    double c0 = C1 * r0 * r0 + C2 * r1 * r1, c1 = C1 * r2 * r2 + C2 * r3 * r3,
           c2 = C1 * r4 * r4 + C2 * r5 * r5;
    double s0 = eps + c0, s1 = eps + c1, s2 = eps + c2;
    double e0 = 0.1 / (s0 * s0), e1 = 0.6 / (s1 * s1), e2 = 0.3 / (s2 * s2);
    double inv2 = 1.0 / (e0 + e1 + e2);
    *ur = (e0 * qR0 + e1 * qR1 + e2 * qR2) * inv2;
}

/* muscl_reconstruct, src_WENO/fluid.cpp:203-225 (dead code in the reference,
 * kept there as an option): cells UL2, UL1 | UR1, UR2 around the face; slopes
 * from the one-sided differences through minmod (limiter 0), van Leer (1) or
 * superbee (2); returns the left and right face states. */
static double ow_minmod2(double a, double b) { return a * b <= 0.0 ? 0.0 : (fabs(a) < fabs(b) ? a : b); }
static double ow_vanleer(double a, double b) {
    double ab = a * b;
    return ab <= 0.0 ? 0.0 : 2.0 * ab / (a + b);
}
static double ow_superbee(double a, double b) {
    double s1 = ow_minmod2(a, 2.0 * b), s2 = ow_minmod2(2.0 * a, b);
    return s1 * s2 <= 0.0 ? 0.0 : (fabs(s1) > fabs(s2) ? s1 : s2);
}
void ow_muscl(double UL2, double UL1, double UR1, double UR2, int limiter, double* ul, double* ur) {
    double dL = UL1 - UL2, dC = UR1 - UL1, dR = UR2 - UR1;
    double sL = 0.0, sR = 0.0;
    switch (limiter) {
        case 0: sL = ow_minmod2(dL, dC); sR = ow_minmod2(dC, dR); break;
        case 1: sL = ow_vanleer(dL, dC); sR = ow_vanleer(dC, dR); break;
        case 2: sL = ow_superbee(dL, dC); sR = ow_superbee(dC, dR); break;
        default: break;
    }
    *ul = UL1 + 0.5 * sL;
    *ur = UR1 - 0.5 * sR;
}

/* Face states of the face between cells a1 and b1 of the stencil
 * a3 a2 a1 | b1 b2 b3: WENO5 (recon 0) or MUSCL with limiter recon - 1. */
static void ow_face(int recon, double a3, double a2, double a1, double b1, double b2, double b3, double* ul,
                    double* ur) {
    if (recon == 0) ow_weno5(a3, a2, a1, b1, b2, b3, ul, ur);
    else ow_muscl(a2, a1, b1, b2, recon - 1, ul, ur);
}

/* hllcFlux (WENO variant), src_WENO/fluid.cpp:268-317: x-direction HLLC with
 * Roe/Einfeldt wave speeds and floors of 1e-12. */
void ow_hllc(const double* L, const double* R, double gamma, double* F) {
    const double eps = 1e-12;
    double rhoL = zk_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3] / rhoL;
    double pL = zk_max((gamma - 1.0) * (L[3] - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(gamma * pL / rhoL);
    double rhoR = zk_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3] / rhoR;
    double pR = zk_max((gamma - 1.0) * (R[3] - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(gamma * pR / rhoR);

    double FL0 = rhoL * uL, FL1 = rhoL * uL * uL + pL, FL2 = rhoL * uL * vL, FL3 = (L[3] + pL) * uL;
    double FR0 = rhoR * uR, FR1 = rhoR * uR * uR + pR, FR2 = rhoR * uR * vR, FR3 = (R[3] + pR) * uR;

    double sqL = sqrt(rhoL), sqR = sqrt(rhoR), den = sqL + sqR;
    double u_roe = (sqL * uL + sqR * uR) / den;
    double h_roe = (sqL * (EL + pL / rhoL) + sqR * (ER + pR / rhoR)) / den;
    double c_roe = sqrt(zk_max((gamma - 1.0) * (h_roe - 0.5 * u_roe * u_roe), eps));
    double SL = zk_min(uL - aL, u_roe - c_roe);
    double SR = zk_max(uR + aR, u_roe + c_roe);

    if (SL >= 0.0) { F[0] = FL0; F[1] = FL1; F[2] = FL2; F[3] = FL3; return; }
    if (SR <= 0.0) { F[0] = FR0; F[1] = FR1; F[2] = FR2; F[3] = FR3; return; }

    double num = pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR);
    double den2 = rhoL * (SL - uL) - rhoR * (SR - uR);
    if (fabs(den2) < 1e-12) den2 = (den2 >= 0 ? 1e-12 : -1e-12);
    double Ss = num / den2;
    if (Ss >= 0.0) {
        double c = rhoL * (SL - uL) / (SL - Ss);
        double s0 = c, s1 = c * Ss, s2 = c * vL, s3 = c * (EL + (Ss - uL) * (Ss + pL / (rhoL * (SL - uL))));
        F[0] = FL0 + SL * (s0 - L[0]); F[1] = FL1 + SL * (s1 - L[1]);
        F[2] = FL2 + SL * (s2 - L[2]); F[3] = FL3 + SL * (s3 - L[3]);
    } else {
        double c = rhoR * (SR - uR) / (SR - Ss);
        double s0 = c, s1 = c * Ss, s2 = c * vR, s3 = c * (ER + (Ss - uR) * (Ss + pR / (rhoR * (SR - uR))));
        F[0] = FR0 + SR * (s0 - R[0]); F[1] = FR1 + SR * (s1 - R[1]);
        F[2] = FR2 + SR * (s2 - R[2]); F[3] = FR3 + SR * (s3 - R[3]);
    }
}

/* Apply the ghost source map in place (see zk_ghost_map). */
static void apply_fill(int nfield, size_t plane, const signed char* kind, const int* src, double* U) {
    for (size_t k = 0; k < plane; ++k) {
        if (src[k] < 0) continue;
        for (int c = 0; c < nfield; ++c) U[c * plane + k] = U[c * plane + (size_t)src[k]];
        (void)kind;
    }
}

/* Flux difference of one fluid cell, src_WENO/fluid.cpp:402-460 (dU includes dt). */
static void cell_rhs(int nx, size_t plane, const double* U, size_t k, double gamma, double dtdx,
                     double dtdy, int recon, double out[4]) {
    double s[13][4];
    /* stencil order: P, r1 r2 r3, l1 l2 l3, u1 u2 u3 (row-1..), d1 d2 d3 (row+1..) */
    const long off[13] = {0, 1, 2, 3, -1, -2, -3, -(long)nx, -2L * nx, -3L * nx, nx, 2L * nx, 3L * nx};
    for (int n = 0; n < 13; ++n)
        for (int c = 0; c < 4; ++c) s[n][c] = U[c * plane + (size_t)((long)k + off[n])];
    double QLr[4], QRr[4], QLl[4], QRl[4], QLd[4], QRd[4], QLu[4], QRu[4];
    for (int c = 0; c < 4; ++c) {
        ow_face(recon, s[5][c], s[4][c], s[0][c], s[1][c], s[2][c], s[3][c], &QLr[c], &QRr[c]);
        ow_face(recon, s[6][c], s[5][c], s[4][c], s[0][c], s[1][c], s[2][c], &QLl[c], &QRl[c]);
        ow_face(recon, s[8][c], s[7][c], s[0][c], s[10][c], s[11][c], s[12][c], &QLd[c], &QRd[c]);
        ow_face(recon, s[9][c], s[8][c], s[7][c], s[0][c], s[10][c], s[11][c], &QLu[c], &QRu[c]);
    }
    double Fr[4], Fl[4], Fd[4], Fu[4];
    ow_hllc(QLr, QRr, gamma, Fr);
    ow_hllc(QLl, QRl, gamma, Fl);
    /* y faces: normal momentum swapped into slot 1 (src_WENO/fluid.cpp:444-451) */
    double a[4] = {QLd[0], QLd[2], QLd[1], QLd[3]}, b[4] = {QRd[0], QRd[2], QRd[1], QRd[3]};
    ow_hllc(a, b, gamma, Fd);
    double e[4] = {QLu[0], QLu[2], QLu[1], QLu[3]}, f[4] = {QRu[0], QRu[2], QRu[1], QRu[3]};
    ow_hllc(e, f, gamma, Fu);
    out[0] = -(dtdx * (Fr[0] - Fl[0]) + dtdy * (Fd[0] - Fu[0]));
    out[1] = -(dtdx * (Fr[1] - Fl[1]) + dtdy * (Fd[2] - Fu[2]));
    out[2] = -(dtdx * (Fr[2] - Fl[2]) + dtdy * (Fd[1] - Fu[1]));
    out[3] = -(dtdx * (Fr[3] - Fl[3]) + dtdy * (Fd[3] - Fu[3]));
}

typedef struct {
    int ny, nx;
    signed char* kind;
    int* src;
} ow_map;

static ow_map map_new(int ny, int nx, const int* bct, int periodic) {
    ow_map m;
    m.ny = ny; m.nx = nx;
    m.kind = (signed char*)malloc((size_t)ny * nx);
    m.src = (int*)malloc(sizeof(int) * (size_t)ny * nx);
    zk_ghost_map(ny, nx, bct, 0, periodic, m.kind, m.src);
    return m;
}
static void map_free(ow_map* m) { free(m->kind); free(m->src); }

static void rhs_with_map(const ow_map* m, double da, double gamma, double* U, double dt, int recon, double* dU) {
    const int ny = m->ny, nx = m->nx;
    const size_t plane = (size_t)ny * nx;
    apply_fill(4, plane, m->kind, m->src, U);
    memset(dU, 0, sizeof(double) * 4 * plane);
    const double dtdx = dt / da, dtdy = dt / da;
    for (size_t k = 0; k < plane; ++k) {
        if (m->kind[k] != ZK_CELL_UPDATED) continue;
        double o[4];
        cell_rhs(nx, plane, U, k, gamma, dtdx, dtdy, recon, o);
        for (int c = 0; c < 4; ++c) dU[c * plane + k] = o[c];
    }
}

/* computeRHS, src_WENO/fluid.cpp:328-463: fill ghosts in U (in place), dU with dt. */
void ow_rhs(int ny, int nx, double da, double gamma, double* U, const int* bct, double dt,
            int periodic, double* dU) {
    ow_map m = map_new(ny, nx, bct, periodic);
    rhs_with_map(&m, da, gamma, U, dt, 0, dU);
    map_free(&m);
}

/* updateMesh, src_WENO/fluid.cpp:468-493: Shu-Osher SSP-RK3 on whole arrays. */
/* updateMesh with the face reconstruction `recon` (0: WENO5, 1..3: MUSCL with
 * minmod, van Leer, superbee). */
void ow_step_recon(int ny, int nx, double da, double gamma, double* U, const int* bct, double dt,
                   int nsteps, int periodic, int recon);
void ow_step(int ny, int nx, double da, double gamma, double* U, const int* bct, double dt,
             int nsteps, int periodic) {
    ow_step_recon(ny, nx, da, gamma, U, bct, dt, nsteps, periodic, 0);
}
void ow_step_recon(int ny, int nx, double da, double gamma, double* U, const int* bct, double dt,
                   int nsteps, int periodic, int recon) {
    const size_t n = (size_t)4 * ny * nx;
    ow_map m = map_new(ny, nx, bct, periodic);
    double* Un = (double*)malloc(sizeof(double) * n);
    double* dU = (double*)malloc(sizeof(double) * n);
    for (int s = 0; s < nsteps; ++s) {
        memcpy(Un, U, sizeof(double) * n);
        rhs_with_map(&m, da, gamma, U, dt, recon, dU);
        for (size_t k = 0; k < n; ++k) U[k] = Un[k] + dU[k];
        rhs_with_map(&m, da, gamma, U, dt, recon, dU);
        for (size_t k = 0; k < n; ++k) U[k] = 0.75 * Un[k] + 0.25 * (U[k] + dU[k]);
        rhs_with_map(&m, da, gamma, U, dt, recon, dU);
        for (size_t k = 0; k < n; ++k) U[k] = (1.0 / 3.0) * Un[k] + (2.0 / 3.0) * (U[k] + dU[k]);
    }
    free(Un); free(dU);
    map_free(&m);
}

/* computeMaxSpeed, src_WENO/fluid.cpp:539-553: max over ALL cells of
 * sqrt(u^2+v^2) + sqrt(gamma p / rho), no floors (NaN never wins). */
double ow_max_speed(int ny, int nx, double gamma, const double* U) {
    const size_t plane = (size_t)ny * nx;
    double umax = 0.0;
    for (size_t k = 0; k < plane; ++k) {
        double rho = U[k], u = U[plane + k] / rho, v = U[2 * plane + k] / rho;
        double p = (gamma - 1.0) * (U[3 * plane + k] - 0.5 * rho * (u * u + v * v));
        double a = sqrt(gamma * p / rho);
        double spd = sqrt(u * u + v * v) + a;
        if (spd > umax) umax = spd;
    }
    return umax;
}

/* recoverPrimitives, src_WENO/fluid.cpp:500-515: prim = [rho, u, v, p]. */
void ow_recover(int ny, int nx, double gamma, const double* U, double* prim) {
    const size_t plane = (size_t)ny * nx;
    for (size_t k = 0; k < plane; ++k) {
        double rho = U[k], ux = U[plane + k] / rho, vy = U[2 * plane + k] / rho;
        prim[k] = rho;
        prim[plane + k] = ux;
        prim[2 * plane + k] = vy;
        prim[3 * plane + k] = (gamma - 1.0) * (U[3 * plane + k] - 0.5 * rho * (ux * ux + vy * vy));
    }
}

/* The ghost source map itself, exported so tests can compare it with the GPU
 * library's host-side map builder. */
void ow_ghost_map(int ny, int nx, const int* bct, int with_slip, int periodic, signed char* kind,
                  int* src) {
    zk_ghost_map(ny, nx, bct, with_slip, periodic, kind, src);
}
