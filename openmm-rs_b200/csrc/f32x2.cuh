// Blackwell packed single precision: one instruction performs the same IEEE round-to-nearest
// add, multiply or fused multiply-add on two float lanes (PTX add/sub/mul/fma .f32x2,
// sm_100 and later).  The pair kernels evaluate two pairs per thread in the two lanes, so
// the floating-point work of a pair takes half the issue slots; the results are bit-for-bit
// those of the scalar instructions.  SFU functions have no packed form and run per lane.
#pragma once

#include <cuda_runtime.h>

namespace ommb200 {
namespace x2 {

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 select(bool u, bool v, float2 a, float b) {
  return make_float2(u ? a.x : b, v ? a.y : b);
}

// SFU approximations per lane (rsqrt / rcp / exp2, flush-to-zero forms).
__device__ __forceinline__ float2 rsqrt_approx(float2 a) {
  float2 y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(a.x));
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(a.y));
  return y;
}
__device__ __forceinline__ float2 rcp_approx(float2 a) {
  float2 y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(a.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(a.y));
  return y;
}
__device__ __forceinline__ float2 exp2_approx(float2 a) {
  float2 y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(a.x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(a.y));
  return y;
}
__device__ __forceinline__ float2 log2_approx(float2 a) {
  float2 y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(a.x));
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(a.y));
  return y;
}

}  // namespace x2
}  // namespace ommb200
