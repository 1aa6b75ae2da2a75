// f2.cuh -- a pair of FP32 values computed with the packed two-lane FP32 instructions
// of sm_100 (FFMA2 / FADD2 / FMUL2 through __ffma2_rn, __fadd2_rn, __fmul2_rn).
//
// The element kernels are written once over an arithmetic type T; instantiated with
// f2 they evaluate two elements at once, one per lane, with one instruction per pair
// of operations.  Every lane rounds like the scalar FP32 operation (round to
// nearest); a - b is formed as fma(b, -1, a), which is exact up to the one rounding
// of the subtraction.
#pragma once

#include <cuda_runtime.h>

namespace vfgpu {

// keep the scalar overloads visible next to fma(f2, f2, f2) for unqualified calls
using ::fma;

struct f2 {
  float2 v;
  f2() = default;
  __device__ __forceinline__ constexpr f2(float2 a) : v(a) {}
  __device__ __forceinline__ constexpr f2(float a, float b) : v{a, b} {}
  // broadcast (constants, material parameters shared by both lanes)
  __device__ __forceinline__ constexpr explicit f2(double a) : v{(float)a, (float)a} {}
  __device__ __forceinline__ constexpr explicit f2(float a) : v{a, a} {}
  __device__ __forceinline__ constexpr explicit f2(int a) : v{(float)a, (float)a} {}
};

__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return f2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return f2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) {
  return f2(__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v));
}
__device__ __forceinline__ f2 operator-(f2 a) { return f2(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ f2& operator+=(f2& a, f2 b) { return a = a + b; }
__device__ __forceinline__ f2& operator-=(f2& a, f2 b) { return a = a - b; }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return f2(__ffma2_rn(a.v, b.v, c.v)); }
// a product kept apart from later adds: formed by a fused multiply-add with zero, which
// nothing can fuse further (a zero product may come out +0 where the multiply gives -0)
__device__ __forceinline__ f2 mul_rn(f2 a, f2 b) {
  return f2(__ffma2_rn(a.v, b.v, make_float2(0.f, 0.f)));
}

}  // namespace vfgpu
