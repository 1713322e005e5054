// Whole-grid FP64 kernels that are not stencils: the ghost fill applied in
// place, the CFL max-wavespeed reductions (WENO and DG semantics) and the
// primitive recovery.  Compiled with --fmad=false (reference arithmetic).
#include "zk_common.cuh"
#include "zk_kernels.h"

namespace zk {
namespace {

// Ghost fill in place: U[g] = U[src(g)] for every filled cell, all nvar
// planes, with the slip-wall sign flips of src_DG/fluid.cpp:600-607,625-632.
// Sources are never filled cells, so the gather has no write/read hazard.
__global__ void fill_ghosts_kernel(double* U, const int8_t* kind, const int32_t* gsrc, Grid g,
                                   int nvar, int nm) {
    const size_t total = (size_t)g.ny * g.pitch;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const int8_t kd = kind[k] & KIND_MASK;
        if (kd < KIND_COPY) continue;
        const size_t s = (size_t)gsrc[k];
        for (int v = 0; v < nvar; ++v) {
            const int c = v / nm;  // conserved variable of plane v ([variable][mode] order)
            const bool neg = (kd == KIND_SLIP_X && c == 1) || (kd == KIND_SLIP_Y && c == 2);
            const double x = U[v * g.plane + s];
            U[v * g.plane + k] = neg ? -x : x;
        }
    }
}

__device__ __forceinline__ double warp_max(double m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, m, o);
        m = (x > m) ? x : m;
    }
    return m;
}

// Block max -> one atomicMax on the bit pattern.  Values are >= +0 and never
// NaN here, and the IEEE order of non-negative doubles is the integer order
// of their bits, so the integer max is the double max.
__device__ __forceinline__ void block_max_commit(double m, unsigned long long* out) {
    __shared__ double part[32];
    m = warp_max(m);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = m;
    __syncthreads();
    if (warp == 0) {
        m = (lane < (int)(blockDim.x >> 5)) ? part[lane] : 0.0;
        m = warp_max(m);
        if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// computeMaxSpeed, src_WENO/fluid.cpp:539-553: all cells, no floors; a NaN
// speed never wins (spd > umax is false), umax starts at 0.
__global__ void max_speed_weno_kernel(const double* U, Grid g, double gamma, unsigned long long* out) {
    double umax = 0.0;
    const size_t n = (size_t)g.ny * g.nx;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / g.nx, j = t - i * g.nx, k = i * g.pitch + j;
        double rho = U[k];
        double u = U[g.plane + k] / rho, v = U[2 * g.plane + k] / rho;
        double p = (gamma - 1.0) * (U[3 * g.plane + k] - 0.5 * rho * (u * u + v * v));
        double a = sqrt(gamma * p / rho);
        double spd = sqrt(u * u + v * v) + a;
        if (spd > umax) umax = spd;
    }
    block_max_commit(umax, out);
}

// computeMaxSpeedDG_omp, src_DG/solver.cpp:26-64: bctype-0 cells of the whole
// grid, state at the 4 corners (xi,eta) = (-1,-1),(+1,-1),(-1,+1),(+1,+1)
// through phi2 (corner values of the basis in phic[m][4]), floors 1e-12.
__global__ void max_speed_dg_kernel(const double* dof, const int8_t* kind, Grid g, int nm,
                                    double gamma, const double* phic, unsigned long long* out) {
    double umax = 0.0;
    const size_t n = (size_t)g.ny * g.nx;
    const double eps = 1e-12;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / g.nx, j = t - i * g.nx, k = i * g.pitch + j;
        if (!(kind[k] & KIND_FLUID)) continue;
        for (int q = 0; q < 4; ++q) {
            double U[4] = {0.0, 0.0, 0.0, 0.0};
            for (int m = 0; m < nm; ++m) {
                const double b = phic[m * 4 + q];
#pragma unroll
                for (int c = 0; c < 4; ++c) U[c] += dof[(size_t)(c * nm + m) * g.plane + k] * b;
            }
            double rho = ref_max(U[0], eps), u = U[1] / rho, v = U[2] / rho;
            double p = ref_max((gamma - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
            double a = sqrt(gamma * p / rho);
            umax = ref_max(umax, sqrt(u * u + v * v) + a);
        }
    }
    block_max_commit(umax, out);
}

// recoverPrimitives, src_WENO/fluid.cpp:500-515 (mode-0 planes for DG).
// U points at variable 0 (mode 0 for DG); vs = plane stride between variables.
__global__ void recover_kernel(const double* U, Grid g, size_t vs, double gamma, double* prim) {
    const size_t n = (size_t)g.ny * g.nx;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / g.nx, j = t - i * g.nx, k = i * g.pitch + j;
        double rho = U[k], ux = U[vs + k] / rho, vy = U[2 * vs + k] / rho;
        prim[k] = rho;
        prim[g.plane + k] = ux;
        prim[2 * g.plane + k] = vy;
        prim[3 * g.plane + k] = (gamma - 1.0) * (U[3 * vs + k] - 0.5 * rho * (ux * ux + vy * vy));
    }
}

int grid_for(size_t n, int threads, int sms) {
    size_t b = (n + threads - 1) / threads;
    size_t cap = (size_t)sms * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

cudaError_t launch_fill_ghosts(double* U, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                               int nvar, int nm, int sms, cudaStream_t s) {
    fill_ghosts_kernel<<<grid_for((size_t)g.ny * g.pitch, 256, sms), 256, 0, s>>>(U, kind, gsrc, g, nvar, nm);
    return cudaGetLastError();
}

cudaError_t launch_max_speed_weno(const double* U, const Grid& g, double gamma,
                                  unsigned long long* out, int sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    max_speed_weno_kernel<<<grid_for((size_t)g.ny * g.nx, 256, sms), 256, 0, s>>>(U, g, gamma, out);
    return cudaGetLastError();
}

cudaError_t launch_max_speed_dg(const double* dof, const int8_t* kind, const Grid& g, int nm,
                                double gamma, const double* phic, unsigned long long* out, int sms,
                                cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    max_speed_dg_kernel<<<grid_for((size_t)g.ny * g.nx, 256, sms), 256, 0, s>>>(dof, kind, g, nm, gamma, phic, out);
    return cudaGetLastError();
}

cudaError_t launch_recover(const double* U, const Grid& g, int nm, double gamma, double* prim,
                           int sms, cudaStream_t s) {
    recover_kernel<<<grid_for((size_t)g.ny * g.nx, 256, sms), 256, 0, s>>>(U, g, (size_t)nm * g.plane, gamma, prim);
    return cudaGetLastError();
}

}  // namespace zk
