// WENO5 + HLLC + SSP-RK3 stage, FP64, the reference's arithmetic op for op.
//
// This file is compiled with --fmad=false: every multiply and add rounds on
// its own, as the reference built with -ffp-contract=off does, so the result
// is bit-identical to it.  It is also the plain FP64 GPU path the mixed
// precision kernel is measured against.
//
// One CTA owns a 32 x 8 tile of cells.  It stages the tile plus a 3-cell halo
// of the stage input in shared memory (ghost cells already replaced by their
// fill source), computes every x and y interface flux of the tile ONCE
// (the reference computes each interface twice, from both neighbours; both
// evaluations see the same six inputs in the same order and give the same
// bits), then forms dU and the Shu-Osher combine for every cell of the tile,
// ghosts included, exactly as the reference's whole-array Eigen expressions do.
#include "batch.cuh"
#include "zk_common.cuh"
#include "zk_kernels.h"

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
namespace {

// A tile is 32 x TY cells; NW warps (TY + 1 by default) take the 2 TY + 2
// face-row tasks (TY + 1 x-face rows, TY + 1 y-face rows) in turn.
constexpr int TX = 32, HX = TX + 6;
template <int TY, int NW = TY + 1>
struct Tile {
    static constexpr int HY = TY + 6, NWARP = NW, NTHREAD = NW * 32;
};

// weno5_reconstruct, src_WENO/fluid.cpp:230-263
__device__ __forceinline__ void weno5(double UL2, double UL1, double UP, double UR1, double UR2,
                                      double UR3, double& UL, double& UR) {
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
    UL = (a0 * qL0 + a1 * qL1 + a2 * qL2) * inv;

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
    UR = (e0 * qR0 + e1 * qR1 + e2 * qR2) * inv2;
}

// muscl_reconstruct, src_WENO/fluid.cpp:203-225 (not called by the reference's
// solvers; the ZK_RECON_MUSCL_* options): cells UL2, UL1 | UR1, UR2 around the
// face, slopes through minmod (LIM 0), van Leer (1) or superbee (2).
__device__ __forceinline__ double minmod2(double a, double b) {
    return a * b <= 0.0 ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}
template <int LIM>
__device__ __forceinline__ double muscl_slope(double a, double b) {
    if constexpr (LIM == 0) {
        return minmod2(a, b);
    } else if constexpr (LIM == 1) {
        const double ab = a * b;
        return ab <= 0.0 ? 0.0 : 2.0 * ab / (a + b);
    } else {
        const double s1 = minmod2(a, 2.0 * b), s2 = minmod2(2.0 * a, b);
        return s1 * s2 <= 0.0 ? 0.0 : (fabs(s1) > fabs(s2) ? s1 : s2);
    }
}
template <int LIM>
__device__ __forceinline__ void muscl(double UL2, double UL1, double UR1, double UR2, double& UL, double& UR) {
    const double dL = UL1 - UL2, dC = UR1 - UL1, dR = UR2 - UR1;
    UL = UL1 + 0.5 * muscl_slope<LIM>(dL, dC);
    UR = UR1 - 0.5 * muscl_slope<LIM>(dC, dR);
}

// Face states from the six cells a3 a2 a1 | b1 b2 b3 around a face: WENO5
// (RECON 0, the reference's scheme) or MUSCL with limiter RECON - 1.
template <int RECON>
__device__ __forceinline__ void face_states(double a3, double a2, double a1, double b1, double b2, double b3,
                                            double& UL, double& UR) {
    if constexpr (RECON == 0) weno5(a3, a2, a1, b1, b2, b3, UL, UR);
    else muscl<RECON - 1>(a2, a1, b1, b2, UL, UR);
}

// hllcFlux (WENO variant), src_WENO/fluid.cpp:268-317
__device__ __forceinline__ void hllc(const double L[4], const double R[4], double gamma, double F[4]) {
    const double eps = 1e-12;
    double rhoL = ref_max(L[0], eps), uL = L[1] / rhoL, vL = L[2] / rhoL, EL = L[3] / rhoL;
    double pL = ref_max((gamma - 1.0) * (L[3] - 0.5 * rhoL * (uL * uL + vL * vL)), eps);
    double aL = sqrt(gamma * pL / rhoL);
    double rhoR = ref_max(R[0], eps), uR = R[1] / rhoR, vR = R[2] / rhoR, ER = R[3] / rhoR;
    double pR = ref_max((gamma - 1.0) * (R[3] - 0.5 * rhoR * (uR * uR + vR * vR)), eps);
    double aR = sqrt(gamma * pR / rhoR);

    double sqL = sqrt(rhoL), sqR = sqrt(rhoR), den = sqL + sqR;
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
    if (fabs(den2) < 1e-12) den2 = (den2 >= 0 ? 1e-12 : -1e-12);
    double Ss = num / den2;
    // star state of the upwind side (the reference's star_state lambda)
    const bool left = (Ss >= 0.0);
    const double rho = left ? rhoL : rhoR, u = left ? uL : uR, v = left ? vL : vR;
    const double E = left ? EL : ER, p = left ? pL : pR, S = left ? SL : SR;
    const double* Us = left ? L : R;
    double c = rho * (S - u) / (S - Ss);
    double s0 = c, s1 = c * Ss, s2 = c * v, s3 = c * (E + (Ss - u) * (Ss + p / (rho * (S - u))));
    double F0 = rho * u, F1 = rho * u * u + p, F2 = rho * u * v, F3 = (Us[3] + p) * u;
    F[0] = F0 + S * (s0 - Us[0]);
    F[1] = F1 + S * (s1 - Us[1]);
    F[2] = F2 + S * (s2 - Us[2]);
    F[3] = F3 + S * (s3 - Us[3]);
}

struct StageArgs {
    const double* Ucur;  // stage input (ghosts unfilled)
    const double* Un;    // state at the start of the step
    double* Uout;        // stage output (may alias Un at stage 3: read-before-write per cell)
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double dtdx, dtdy, gamma;
    int stage;  // 0: write dU only, 1..3: Shu-Osher stage
    uint32_t* status;
    int want_lam;  // 1: return the max wave speed of the cells written
};

template <int TY>
struct Smem {
    double sU[4][TY + 6][HX];
    double sFx[4][TY][TX + 1];
    double sFy[4][TY + 1][TX];
    int8_t sK[TY + 6][HX];
};

// One tile whose top-left cell is (i0, j0).  Ends with every thread past its
// last shared-memory read, so a persistent caller may reuse S after a barrier.
// Returns the thread's max wave speed of the cells it wrote (want_lam), else 0.
template <int TY, int NW = TY + 1, int RECON = 0>
__device__ __forceinline__ double stage_tile(const StageArgs& a, int j0, int i0, Smem<TY>& S) {
    constexpr int HY = Tile<TY, NW>::HY, NWARP = Tile<TY, NW>::NWARP, NTHREAD = Tile<TY, NW>::NTHREAD;
    auto& sU = S.sU;
    auto& sFx = S.sFx;
    auto& sFy = S.sFy;
    auto& sK = S.sK;
    const int ny = a.g.ny, nx = a.g.nx, pitch = a.g.pitch;
    const size_t plane = a.g.plane;

    // 1. tile + halo of the stage input, ghosts replaced by their source
    for (int t = threadIdx.x; t < HY * HX; t += NTHREAD) {
        const int r = t / HX, c = t - r * HX;
        const int gi = i0 - 3 + r, gj = j0 - 3 + c;
        int8_t kd = KIND_PASSIVE;
        double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
        if (gi >= 0 && gi < ny && gj >= 0 && gj < nx) {
            const size_t k = (size_t)gi * pitch + gj;
            kd = a.kind[k] & KIND_MASK;
            const size_t ks = (kd >= KIND_COPY) ? (size_t)a.gsrc[k] : k;
            v0 = a.Ucur[ks];
            v1 = a.Ucur[plane + ks];
            v2 = a.Ucur[2 * plane + ks];
            v3 = a.Ucur[3 * plane + ks];
        }
        sU[0][r][c] = v0; sU[1][r][c] = v1; sU[2][r][c] = v2; sU[3][r][c] = v3;
        sK[r][c] = kd;
    }
    __syncthreads();

    // 2. interface fluxes, each computed once
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int task = warp; task < 2 * TY + 2; task += NWARP) {
        if (task <= TY) {
            // x face on the left of tile cell (r, c): cells (r, c-3 .. c+2)
            int r, c;
            if (task < TY) { r = task; c = lane; }
            else { if (lane >= TY) continue; r = lane; c = TX; }
            const bool need = sK[r + 3][c + 2] == KIND_UPDATED || sK[r + 3][c + 3] == KIND_UPDATED;
            if (!need) continue;
            double QL[4], QR[4], F[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                face_states<RECON>(sU[q][r + 3][c], sU[q][r + 3][c + 1], sU[q][r + 3][c + 2], sU[q][r + 3][c + 3],
                                   sU[q][r + 3][c + 4], sU[q][r + 3][c + 5], QL[q], QR[q]);
            hllc(QL, QR, a.gamma, F);
#pragma unroll
            for (int q = 0; q < 4; ++q) sFx[q][r][c] = F[q];
        } else {
            // y face above tile cell (r, c): cells (r-3 .. r+2, c); normal momentum swapped in
            const int r = task - TY - 1, c = lane;
            const bool need = sK[r + 2][c + 3] == KIND_UPDATED || sK[r + 3][c + 3] == KIND_UPDATED;
            if (!need) continue;
            double QL[4], QR[4], F[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                face_states<RECON>(sU[q][r][c + 3], sU[q][r + 1][c + 3], sU[q][r + 2][c + 3], sU[q][r + 3][c + 3],
                                   sU[q][r + 4][c + 3], sU[q][r + 5][c + 3], QL[q], QR[q]);
            double L[4] = {QL[0], QL[2], QL[1], QL[3]}, R[4] = {QR[0], QR[2], QR[1], QR[3]};
            hllc(L, R, a.gamma, F);
#pragma unroll
            for (int q = 0; q < 4; ++q) sFy[q][r][c] = F[q];
        }
    }
    __syncthreads();

    // 3. dU and the stage combine for every cell of the tile
    uint32_t flags = 0;
    double umax = 0.0;
    for (int t = threadIdx.x; t < TY * TX; t += NTHREAD) {
        const int r = t / TX, c = t - r * TX;
        const int gi = i0 + r, gj = j0 + c;
        if (gi >= ny || gj >= nx) continue;
        const size_t k = (size_t)gi * pitch + gj;
        const int8_t kd = sK[r + 3][c + 3];
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        if (kd == KIND_UPDATED) {
            // src_WENO/fluid.cpp:454-460; y-face fluxes carry the momentum swap
            d[0] = -(a.dtdx * (sFx[0][r][c + 1] - sFx[0][r][c]) + a.dtdy * (sFy[0][r + 1][c] - sFy[0][r][c]));
            d[1] = -(a.dtdx * (sFx[1][r][c + 1] - sFx[1][r][c]) + a.dtdy * (sFy[2][r + 1][c] - sFy[2][r][c]));
            d[2] = -(a.dtdx * (sFx[2][r][c + 1] - sFx[2][r][c]) + a.dtdy * (sFy[1][r + 1][c] - sFy[1][r][c]));
            d[3] = -(a.dtdx * (sFx[3][r][c + 1] - sFx[3][r][c]) + a.dtdy * (sFy[3][r + 1][c] - sFy[3][r][c]));
        }
        double o[4];
        if (a.stage == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) o[q] = d[q];
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double un = a.Un[q * plane + k];
                const double v = sU[q][r + 3][c + 3];
                if (a.stage == 1) o[q] = un + d[q];
                else if (a.stage == 2) o[q] = 0.75 * un + 0.25 * (v + d[q]);
                else o[q] = (1.0 / 3.0) * un + (2.0 / 3.0) * (v + d[q]);
            }
            if (kd == KIND_UPDATED) {
                if (isnan(o[0]) || isnan(o[1]) || isnan(o[2]) || isnan(o[3])) flags |= STATUS_NAN;
                if (!(o[0] > 0.0)) flags |= STATUS_RHO;
            }
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
    return umax;
}

// 3 CTAs per SM (72 registers, no spills): +19% over 2 CTAs at 84 registers.
template <int RECON>
__global__ void __launch_bounds__(Tile<8>::NTHREAD, 3) weno_stage_fp64_kernel(StageArgs a) {
    __shared__ Smem<8> S;
    stage_tile<8, 9, RECON>(a, blockIdx.x * TX, blockIdx.y * 8, S);
}

// Persistent stage over every listed problem of a batch group: CTA b takes
// global tiles b, b + gridDim.x, ...; stage s reads U[s-1] (U^n at stage 1)
// and writes U[s % 3].  Stage 3 also leaves the max wave speed of the new
// state (computeMaxSpeed over all cells) in the problem's control block.
// Tile variant V (batch.cuh); the register share is that of 864 threads per
// SM (72 registers).
template <int V, int TY = weno_variant_rows(V), int NW = weno_variant_warps(V)>
__global__ void __launch_bounds__(NW * 32, batch_min_blocks(NW * 32, 864, sizeof(Smem<TY>)))
    weno_stage_fp64_batch_kernel(const WenoItem* __restrict__ items, const int* __restrict__ dir, int cap,
                                 int stage) {
    __shared__ Smem<TY> S;
    __shared__ StageArgs sa;  // the current tile's problem, kept out of registers
    __shared__ int s_org[3];  // tile origin x, y; 0 when the problem is not stepping
    __shared__ unsigned long long* s_lam;
    const int total = __ldg(dir + 1);
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
                sa = StageArgs{it.U[stage - 1], it.U[0], it.U[stage % 3], it.kind, it.gsrc, it.g,
                               ctl->dtdx, ctl->dtdy, it.gamma, stage, &ctl->status, stage == 3};
                s_lam = &ctl->lam;
            }
        }
        __syncthreads();
        if (s_org[2]) {
            const double m = stage_tile<TY, NW>(sa, s_org[0], s_org[1], S);
            if (stage == 3) block_max_commit_to(m, s_lam);  // the next step's wave speed
        }
        __syncthreads();
    }
}

}  // namespace

namespace {
template <int V>
cudaError_t launch_batch_v(const WenoItem* items, const int* dir, int cap, int stage, int grid, cudaStream_t s) {
    weno_stage_fp64_batch_kernel<V><<<grid, weno_variant_warps(V) * 32, 0, s>>>(items, dir, cap, stage);
    return cudaGetLastError();
}
template <int V>
int occupancy_v() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, weno_stage_fp64_batch_kernel<V>, weno_variant_warps(V) * 32, 0);
    return n;
}
}  // namespace

cudaError_t launch_weno_stage_fp64_batch(int variant, const WenoItem* items, const int* dir, int cap, int stage,
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

int weno_fp64_batch_occupancy(int variant) {
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

cudaError_t launch_weno_stage_fp64(const double* Ucur, const double* Un, double* Uout,
                                   const int8_t* kind, const int32_t* gsrc, const Grid& g,
                                   double dtdx, double dtdy, double gamma, int stage,
                                   uint32_t* status, cudaStream_t s, int recon) {
    StageArgs a{Ucur, Un, Uout, kind, gsrc, g, dtdx, dtdy, gamma, stage, status};
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + 7) / 8);
    switch (recon) {
        case 0: weno_stage_fp64_kernel<0><<<grid, Tile<8>::NTHREAD, 0, s>>>(a); break;
        case 1: weno_stage_fp64_kernel<1><<<grid, Tile<8>::NTHREAD, 0, s>>>(a); break;
        case 2: weno_stage_fp64_kernel<2><<<grid, Tile<8>::NTHREAD, 0, s>>>(a); break;
        case 3: weno_stage_fp64_kernel<3><<<grid, Tile<8>::NTHREAD, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ZK_FP64_NS
