// Shared definitions of the DG kernels: basis tables and launch arguments.
#pragma once

#include "zk_common.cuh"

namespace zk {

constexpr int DG_MAXNM = 16, DG_MAXNQ = 4;

// Basis values of one polynomial degree P (NQ = P+1 Gauss points, NM modes).
struct DGTab {
    double vw[DG_MAXNQ * DG_MAXNQ];                // volume weights w_a w_b, point p = qa*NQ+qb
    double vphi[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];   // phi2(m, xi_a, eta_b)
    double vdxi[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];   // d phi2 / d xi
    double vdet[DG_MAXNQ * DG_MAXNQ][DG_MAXNM];   // d phi2 / d eta
    double tr[4][DG_MAXNQ][DG_MAXNM];             // traces: 0 xi=+1, 1 xi=-1, 2 eta=+1, 3 eta=-1
    double bv[4][DG_MAXNQ][DG_MAXNM];             // trace * face weight
    double zs[16][DG_MAXNM];                      // Zhang-Shu basis at the 4x4 Gauss points
};

// One-dimensional factors of P's tensor-product basis phi_m(xi, eta) =
// P_px(xi) P_py(eta), m = px (P+1) + py, at the NQ = P+1 Gauss points (the
// 2D quadrature is their tensor grid): L[n][q] = P_n(x_q), D[n][q] = P_n'(x_q),
// W[q] = w_q, E[n][0|1] = P_n(+1|-1), Z[n][a] = the Zhang-Shu factor of
// degree n at the 4-point Gauss node a (cubic factor dropped, as the
// reference's basis() does, src_DG/fluid.cpp:808-823).
struct DGSep {
    double L[DG_MAXNQ][DG_MAXNQ];
    double D[DG_MAXNQ][DG_MAXNQ];
    double W[DG_MAXNQ];
    double E[DG_MAXNQ][2];
    double Z[DG_MAXNQ][4];
};
void dg_make_sep(int P, DGSep* S);

// Host: tabulate P's basis (and the 4 corner values used by the CFL
// reduction, phic[m*4+k]); upload to the calling TU's constant bank.
void dg_make_tables(int P, DGTab* T, double* phic);
int dg_upload_tables(int P, const DGTab& T);

struct DGArgs {
    const double* cur;   // stage input (ghosts unfilled)
    const double* un;    // state at the start of the step
    double* out;         // stage output (may alias un at stage 3)
    const int8_t* kind;
    const int32_t* gsrc;
    double* fx;          // x-face fluxes [q][c][ny][xpitch]
    double* fy;          // y-face fluxes [q][c][ny+1][pitch]
    Grid g;
    int xpitch;
    double dt, inv2h, gamma;
    int stage;           // 0: write d(dof)/dt only; 1..3 Shu-Osher stages
    int limiter;         // ZK_LIMITER_*
    int hll;             // 1: HLLE instead of HLLC
    double s0;           // Persson threshold -4 log10 P (P<3) or -3 log10 P, from the host's libm
    uint32_t* status;
    const double* phic;  // basis at the 4 cell corners [NM][4] (want_lam only)
    int want_lam;        // 1: report the max corner wave speed of the fluid cells written
};

// The learned indicator fused into a mixed-precision stage: fragment-packed
// weights (MlpFrag, mlp_infer.cuh), the list the flagged cells are appended
// to (pitched indices, capacity cap), its device counter, and an optional
// per-cell debug output (features and logit, 41 floats per pitched cell),
// and the screen of smooth cells.
struct FusedIndicator {
    const void* mlp;
    int32_t* list;
    uint32_t* count;
    uint32_t cap;
    float* dbg;
    float screen;  // cells within this of a constant state's features skip the network (< 0: none)
};

}  // namespace zk
