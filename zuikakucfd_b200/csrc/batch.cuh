// Device-side structures of the batched runner: many independent problems of
// uneven grid sizes advanced together by persistent kernels.
//
// Every problem owns a control block (BatchCtl) that the per-step control
// kernels update on the device: the time step from the problem's own CFL
// rule, the step counter, the done/failed state and the completion time.
// A problem group (problems sharing method, precision and order) owns one
// item array (per-problem pointers and sizes) and, per tiling, a directory:
//
//   dir[0] = n (problems listed), dir[1] = total tiles,
//   dir[2 .. 2+cap)        = item index of each listed problem,
//   dir[2+cap .. 2+2cap)   = exclusive end of each problem's tile range.
//
// The host rewrites directories between graph launches (admission), so the
// captured kernels stay valid while the set of running problems changes.
#pragma once

#include <cuda.h>
#include <cstdint>
#include "zk_common.cuh"

namespace zk {

enum : int { BATCH_WAITING = 0, BATCH_RUNNING = 1, BATCH_DONE = 2, BATCH_FAILED = 3 };

struct BatchCtl {
    double dt, dtdx, dtdy;      // time step of the current step, and dt/da
    double t;                   // simulated time reached
    double cfl;                 // CFL number of the problem's dt rule
    double da;
    unsigned long long lam;     // max wave speed of the step's input (double bits, atomicMax)
    unsigned long long t_done;  // %globaltimer (ns) when the problem finished or failed
    double* dtlog;              // dt of every step taken, [steps_target]
    int steps_done, steps_target;
    int state;                  // BATCH_*
    int stepping;               // 1 while the current step advances this problem
    int method, order;
    uint32_t status;            // STATUS_* bits of this problem's kernels
    int lam_ready;              // lam already holds the current state's speed (stage-3 epilogue)
};

// Tile variants of the WENO stage kernels the autotuner chooses between:
// v = 3 * h + k is a 32 x kWenoTileRows[h] tile worked by weno_tile_warps
// warps.  A tile has 2 rows + 2 face-row tasks (rows + 1 of x faces, rows + 1
// of y faces); k = 0, 1, 2 give each warp about four, two or one of them, so
// threads per cell is about 0.6, 1.2 or 2.4: fewer threads leave each more
// registers, more threads hide more latency per resident tile.
constexpr int kWenoTileRows[2] = {4, 8};
constexpr int kWenoVariants = 6;
constexpr int weno_tile_warps(int rows, int k) { return k == 0 ? rows / 2 + 1 : k == 1 ? rows + 1 : 2 * rows + 2; }
constexpr int weno_variant_rows(int v) { return kWenoTileRows[v / 3]; }
constexpr int weno_variant_warps(int v) { return weno_tile_warps(kWenoTileRows[v / 3], v % 3); }
constexpr int kWenoDefaultVariant = 4;  // 32 x 8, 9 warps
// Tile variants of the mixed-precision DG stage kernel: v = 2 * t + h is a
// 32 x kDgTileRows[h] tile worked by t + 1 threads per cell (two threads
// split a cell's four conserved variables into pairs).
constexpr int kDgTileRows[2] = {2, 4};
constexpr int kDgVariants = 4;
constexpr int dg_variant_rows(int v) { return kDgTileRows[v & 1]; }
constexpr int dg_variant_tpc(int v) { return 1 + (v >> 1); }
constexpr int kDgDefaultVariant = 1;  // 32 x 4, one thread per cell
// Row segment of the FP64 DG cell pass (one thread per cell).
constexpr int kDgCellBlock = 64;

// CTAs per SM to promise in __launch_bounds__ for a persistent stage kernel:
// as many as keep every thread within the register share of `thread_budget`
// threads per SM and as many as the SM's 228 KB of shared memory holds (with
// the 1 KB each resident CTA reserves).
constexpr int batch_min_blocks(int nthread, int thread_budget, unsigned long smem) {
    const int by_regs = thread_budget / nthread;
    const int by_smem = (int)(233472ul / (smem + 1024ul + 512ul));
    const int b = by_regs < by_smem ? by_regs : by_smem;
    return b < 1 ? 1 : b;
}

// One WENO problem of a group.  tmap[h][b]: TMA map over buffer b (U^n,
// stage 1, stage 2) with the box of tile height kWenoTileRows[h] (mixed
// precision only).
struct alignas(64) WenoItem {
    CUtensorMap tmap[2][3];
    double* U[3];
    const int8_t* kind;
    const int32_t* gsrc;
    BatchCtl* ctl;
    Grid g;
    double gamma;
};

// One DG problem of a group.
struct DgItem {
    double* U[3];       // U^n and the two FP64 stage states (FP64 path)
    float* F[2];        // FP32 stage states (mixed path)
    double* fx;         // face fluxes (FP64 path)
    double* fy;
    const int8_t* kind;
    const int32_t* gsrc;
    const double* phic;  // basis at the 4 cell corners [NM][4] (CFL reduction)
    BatchCtl* ctl;
    Grid g;
    int xpitch, nm;
    double inv2h, gamma, s0;
    int limiter, hll;
};

// Index of the listed problem whose tile range holds global tile t.
__device__ __forceinline__ int dir_find(const int* __restrict__ end, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(end + mid) > t) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// The problem (item index) and problem-local tile of global tile t.
struct DirHit {
    int item, local;
};
__device__ __forceinline__ DirHit dir_lookup(const int* __restrict__ dir, int cap, int t) {
    const int n = __ldg(dir);
    const int* end = dir + 2 + cap;
    const int s = dir_find(end, n, t);
    return {__ldg(dir + 2 + s), t - (s ? __ldg(end + s - 1) : 0)};
}

// Wave speed |u| + a of one WENO cell, FP64, with the operations and order of
// computeMaxSpeed (src_WENO/fluid.cpp:539-553).  The round-to-nearest
// intrinsics keep it free of FMA contraction in any translation unit, so every
// kernel that evaluates it gets the bits of the standalone reduction.
__device__ __forceinline__ double weno_cell_speed(double r, double mx, double my, double E, double gamma) {
    const double u = __ddiv_rn(mx, r), v = __ddiv_rn(my, r);
    const double q = __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v));
    const double p = __dmul_rn(__dsub_rn(gamma, 1.0), __dsub_rn(E, __dmul_rn(__dmul_rn(0.5, r), q)));
    const double a = __dsqrt_rn(__ddiv_rn(__dmul_rn(gamma, p), r));
    return __dadd_rn(__dsqrt_rn(q), a);
}

// Largest corner wave speed of one DG cell (computeMaxSpeedDG_omp,
// src_DG/solver.cpp:26-64): U at the corners accumulated over the modes in
// increasing order, floors 1e-12.  cs[k][c] = variable c at corner k.
__device__ __forceinline__ double dg_cell_speed(const double (&cs)[4][4], double gamma, double umax) {
    const double eps = 1e-12;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double rho = ref_max(cs[k][0], eps);
        const double u = __ddiv_rn(cs[k][1], rho), v = __ddiv_rn(cs[k][2], rho);
        const double q = __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v));
        const double p =
            ref_max(__dmul_rn(__dsub_rn(gamma, 1.0), __dsub_rn(cs[k][3], __dmul_rn(__dmul_rn(0.5, rho), q))), eps);
        const double a = __dsqrt_rn(__ddiv_rn(__dmul_rn(gamma, p), rho));
        umax = ref_max(umax, __dadd_rn(__dsqrt_rn(q), a));
    }
    return umax;
}

// CTA-wide max of per-thread speeds (>= 0, never NaN) committed with one
// atomicMax on the bits (the IEEE order of non-negative doubles is the
// integer order of their bits).  Every thread of the CTA must call it.
__device__ __forceinline__ void block_max_commit_to(double m, unsigned long long* out) {
    __shared__ double part[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, m, o);
        m = (x > m) ? x : m;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = m;
    __syncthreads();
    if (warp == 0) {
        m = (lane < (int)(blockDim.x >> 5)) ? part[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_xor_sync(0xffffffffu, m, o);
            m = (x > m) ? x : m;
        }
        if (lane == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace zk
