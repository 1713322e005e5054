// Packed FP32 pairs (sm_100 add/mul/fma .f32x2): one instruction issues the
// same operation on two values, e.g. two conserved variables that share every
// coefficient.  Each lane rounds exactly as the scalar instruction does.
#pragma once

#include <cuda_runtime.h>

namespace zk {

__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

}  // namespace zk
