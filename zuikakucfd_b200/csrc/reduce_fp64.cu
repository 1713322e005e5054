// Whole-grid FP64 kernels that are not stencils: the ghost fill applied in
// place, the CFL max-wavespeed reductions (WENO and DG semantics) and the
// primitive recovery.  Compiled with --fmad=false (reference arithmetic).
#include "batch.cuh"
#include "zk_common.cuh"
#include "zk_kernels.h"
#include "zuikaku.h"

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

// Mach number and speed of the cell averages, the plot notebook's
// compute_mach (plot.ipynb cell 0): |u| / sqrt(gamma p / rho), p recovered as
// recoverPrimitives does.  U points at variable 0 (mode 0 for DG); vs = plane
// stride between variables.
__global__ void mach_kernel(const double* U, Grid g, size_t vs, double gamma, double* mach, double* speed) {
    const size_t n = (size_t)g.ny * g.nx;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / g.nx, j = t - i * g.nx, k = i * g.pitch + j;
        const double rho = U[k], ux = U[vs + k] / rho, vy = U[2 * vs + k] / rho;
        const double p = (gamma - 1.0) * (U[3 * vs + k] - 0.5 * rho * (ux * ux + vy * vy));
        const double vel = sqrt(ux * ux + vy * vy);
        speed[k] = vel;
        mach[k] = vel / sqrt(gamma * p / rho);
    }
}

// ---- batched runner: per-problem CFL reductions and step control ---------------

constexpr int kRedChunk = 2048;  // cells per reduction tile of the batched runner

// Max wave speed of every listed problem of a batch group that is not finished
// and whose speed the previous step's stage 3 did not already leave (first
// step after admission), committed to its control block (same per-cell semantics as the kernels
// above; the max is exact, so the tiling does not change the result).
__global__ void __launch_bounds__(256) max_speed_batch_kernel(const void* __restrict__ items, int method,
                                                              const int* __restrict__ dir, int cap) {
    const int total = __ldg(dir + 1);
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const DirHit h = dir_lookup(dir, cap, t);
        double umax = 0.0;
        BatchCtl* ctl;
        if (method == ZK_METHOD_DG) {
            const DgItem& it = static_cast<const DgItem*>(items)[h.item];
            ctl = it.ctl;
            if (ctl->state >= BATCH_DONE || ctl->lam_ready) continue;
            const Grid g = it.g;
            const size_t n = (size_t)g.ny * g.nx, c1 = min(n, (size_t)(h.local + 1) * kRedChunk);
            const double eps = 1e-12, gamma = it.gamma;
            for (size_t c = (size_t)h.local * kRedChunk + threadIdx.x; c < c1; c += blockDim.x) {
                const size_t i = c / g.nx, j = c - i * g.nx, k = i * g.pitch + j;
                if (!(it.kind[k] & KIND_FLUID)) continue;
                for (int q = 0; q < 4; ++q) {
                    double U[4] = {0.0, 0.0, 0.0, 0.0};
                    for (int m = 0; m < it.nm; ++m) {
                        const double b = it.phic[m * 4 + q];
#pragma unroll
                        for (int v = 0; v < 4; ++v) U[v] += it.U[0][(size_t)(v * it.nm + m) * g.plane + k] * b;
                    }
                    double rho = ref_max(U[0], eps), u = U[1] / rho, v = U[2] / rho;
                    double p = ref_max((gamma - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v)), eps);
                    double a = sqrt(gamma * p / rho);
                    umax = ref_max(umax, sqrt(u * u + v * v) + a);
                }
            }
        } else {
            const WenoItem& it = static_cast<const WenoItem*>(items)[h.item];
            ctl = it.ctl;
            if (ctl->state >= BATCH_DONE || ctl->lam_ready) continue;
            const Grid g = it.g;
            const double* U = it.U[0];
            const double gamma = it.gamma;
            const size_t n = (size_t)g.ny * g.nx, c1 = min(n, (size_t)(h.local + 1) * kRedChunk);
            for (size_t c = (size_t)h.local * kRedChunk + threadIdx.x; c < c1; c += blockDim.x) {
                const size_t i = c / g.nx, j = c - i * g.nx, k = i * g.pitch + j;
                double rho = U[k];
                double u = U[g.plane + k] / rho, v = U[2 * g.plane + k] / rho;
                double p = (gamma - 1.0) * (U[3 * g.plane + k] - 0.5 * rho * (u * u + v * v));
                double a = sqrt(gamma * p / rho);
                double spd = sqrt(u * u + v * v) + a;
                if (spd > umax) umax = spd;
            }
        }
        block_max_commit(umax, &ctl->lam);
        __syncthreads();
    }
}

// Start of a step: admitted problems that are not finished take a time step
// from their CFL rule -- WENO dt = cfl da / lambda (the per-step form of
// src_WENO/solver.cpp:159-171), DG dt = cfl * dgSafeDt (src_DG/solver.cpp:19-23)
// -- and reset the speed accumulator.  A non-finite or non-positive dt fails
// the problem.
__global__ void batch_ctl_pre_kernel(BatchCtl* ctl, const int* __restrict__ members, int n,
                                     const int* __restrict__ admitted) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        BatchCtl& c = ctl[members[s]];
        c.stepping = 0;
        if (!admitted[members[s]] || c.state >= BATCH_DONE) continue;
        c.state = BATCH_RUNNING;
        const double lam = __longlong_as_double((long long)c.lam);
        c.lam = 0ull;
        c.lam_ready = 0;
        double dt;
        if (c.method == ZK_METHOD_DG) dt = c.cfl * (0.9 / (2.0 * (2 * c.order + 1)) * c.da / ref_max(lam, 1e-7));
        else dt = c.cfl * c.da / lam;
        if (!(dt > 0.0) || isinf(dt)) {
            c.state = BATCH_FAILED;
            c.status |= STATUS_NAN;
            c.t_done = global_ns();
            continue;
        }
        c.dt = dt;
        c.dtdx = dt / c.da;
        c.dtdy = dt / c.da;
        c.stepping = 1;
    }
}

// End of a step: count it, log its dt, finish or fail the problem.
__global__ void batch_ctl_post_kernel(BatchCtl* ctl, const int* __restrict__ members, int n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        BatchCtl& c = ctl[members[s]];
        if (!c.stepping) continue;
        c.stepping = 0;
        c.dtlog[c.steps_done] = c.dt;
        c.steps_done += 1;
        c.t += c.dt;
        if (c.status & (STATUS_NAN | STATUS_TIMEOUT)) {
            c.state = BATCH_FAILED;
            c.t_done = global_ns();
        } else if (c.steps_done >= c.steps_target) {
            c.state = BATCH_DONE;
            c.t_done = global_ns();
        } else {
            c.lam_ready = 1;  // stage 3 left the new state's wave speed in lam
        }
    }
}

__global__ void batch_clock_kernel(unsigned long long* t) { *t = global_ns(); }

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

cudaError_t launch_mach(const double* U, const Grid& g, int nm, double gamma, double* mach, double* speed, int sms,
                        cudaStream_t s) {
    mach_kernel<<<grid_for((size_t)g.ny * g.nx, 256, sms), 256, 0, s>>>(U, g, (size_t)nm * g.plane, gamma, mach, speed);
    return cudaGetLastError();
}

int batch_red_tiles(int ny, int nx) { return (int)(((size_t)ny * nx + kRedChunk - 1) / kRedChunk); }

cudaError_t launch_batch_max_speed(int method, const void* items, const int* dir, int cap, int grid, cudaStream_t s) {
    max_speed_batch_kernel<<<grid, 256, 0, s>>>(items, method, dir, cap);
    return cudaGetLastError();
}

cudaError_t launch_batch_ctl(int post, BatchCtl* ctl, const int* members, int n, const int* admitted,
                             cudaStream_t s) {
    const int grid = (n + 127) / 128;
    if (post) batch_ctl_post_kernel<<<grid, 128, 0, s>>>(ctl, members, n);
    else batch_ctl_pre_kernel<<<grid, 128, 0, s>>>(ctl, members, n, admitted);
    return cudaGetLastError();
}

cudaError_t launch_batch_clock(unsigned long long* t, cudaStream_t s) {
    batch_clock_kernel<<<1, 1, 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace zk
