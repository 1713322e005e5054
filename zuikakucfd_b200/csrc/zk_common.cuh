// Shared device/host definitions of the ZuikakuCFD B200 kernels.
//
// Device layout of every field: planes of ny rows x pitch doubles (pitch =
// nx rounded up to 32 elements, 256-byte rows), plane stride ny*pitch.  WENO
// keeps 4 planes (rho, rho*u, rho*v, E); DG keeps 4*NM planes ordered
// [variable][mode] like the reference's dof[c][m] (src_DG/fluid.h:84).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace zk {

// Per-cell kind byte (low 3 bits) plus the "bctype == 0" flag (bit 3).
// Meaning identical to the oracle's ZK_CELL_* codes.
enum : int8_t {
    KIND_UPDATED = 0,  // bctype 0 inside [3,ny-3)x[3,nx-3): receives the RHS
    KIND_PASSIVE = 1,  // not updated, not filled (dU = 0)
    KIND_COPY = 2,     // ghost: refilled from gsrc before every RHS evaluation
    KIND_SLIP_X = 3,   // DG slip wall, x normal (rho*u negated)
    KIND_SLIP_Y = 4,   // DG slip wall, y normal (rho*v negated)
    KIND_MASK = 0x7,
    KIND_FLUID = 0x8   // bctype == 0 (the DG CFL reduction visits these)
};

// Status word bits (atomicOr'd by kernels, read by zk_status_word).
enum : uint32_t { STATUS_NAN = 1u, STATUS_RHO = 2u, STATUS_P = 4u, STATUS_TIMEOUT = 8u };

// std::max(a,b) / std::min(a,b) exactly as the reference's std:: calls
// evaluate them: a NaN first argument is returned unchanged.
__host__ __device__ __forceinline__ double ref_max(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double ref_min(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float ref_maxf(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float ref_minf(float a, float b) { return (b < a) ? b : a; }

struct Grid {
    int ny, nx, pitch;
    size_t plane;  // ny * pitch
};

inline int round_pitch(int nx) { return (nx + 31) / 32 * 32; }

}  // namespace zk
