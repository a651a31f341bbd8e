// OBC / HCT arithmetic shared by the exact GBSAOBCForce passes (gbsa.cu) and the learned-radii
// passes (learned_gb.cu): forces/gbsa_obc.rs:8-9 constants and the descreening integral with
// its radial derivative (gbsa_obc.rs:278-309).
#pragma once

#include <cuda_runtime.h>

namespace ommb200 {
namespace gb {

constexpr double kDielectricOffset = 0.009;  // gbsa_obc.rs:8
constexpr double kProbeRadius = 0.14;        // gbsa_obc.rs:9
constexpr double kBornScale = 1099511627776.0;  // 2^40
constexpr double kBornScaleInv = 1.0 / 1099511627776.0;

__device__ __forceinline__ float log_r(float x) { return logf(x); }
__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float exp_gb(float x) { return expf(x); }
__device__ __forceinline__ double exp_gb(double x) { return exp(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }

// gbsa_obc.rs:278-295; `radius` = rho_i - 0.009, `scaled` = s_j (rho_j - 0.009)
template <class Real>
__device__ __forceinline__ Real descreening(Real radius, Real scaled, Real r) {
  if (radius >= r + scaled) return Real(0);
  const Real lower = Real(1) / fmax(radius, fabs(r - scaled));
  const Real upper = Real(1) / (r + scaled);
  const Real inverse = Real(1) / r;
  Real value = lower - upper + Real(0.25) * r * (upper * upper - lower * lower) +
               Real(0.5) * inverse * log_r(upper / lower) +
               Real(0.25) * scaled * scaled * inverse * (lower * lower - upper * upper);
  if (radius < scaled - r) value += Real(2) * (Real(1) / radius - lower);
  return value;
}

// gbsa_obc.rs:297-309
template <class Real>
__device__ __forceinline__ Real descreening_gradient(Real radius, Real scaled, Real r) {
  if (radius >= r + scaled) return Real(0);
  const Real lower = Real(1) / fmax(radius, fabs(r - scaled));
  const Real upper = Real(1) / (r + scaled);
  const Real inverse = Real(1) / r;
  return (Real(0.125) * (Real(1) + scaled * scaled * inverse * inverse) *
              (lower * lower - upper * upper) +
          Real(0.25) * log_r(upper / lower) * inverse * inverse) *
         inverse;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP32 form of the integral and its gradient together, with SFU reciprocals and logarithm;
// inv_r = 1 / r.
__device__ __forceinline__ void descreening_fast(float radius, float scaled, float r, float inv_r,
                                                 float* h, float* grad) {
  if (radius >= r + scaled) {
    *h = 0.f;
    *grad = 0.f;
    return;
  }
  const float lo_den = fmaxf(radius, fabsf(r - scaled));
  const float lower = rcp_approx(lo_den), upper = rcp_approx(r + scaled);
  const float l2u2 = lower * lower - upper * upper;
  const float lg = __logf(lo_den * upper);  // log(upper / lower)
  float v = lower - upper - 0.25f * r * l2u2 + 0.5f * inv_r * lg +
            0.25f * scaled * scaled * inv_r * l2u2;
  if (radius < scaled - r) v += 2.f * (rcp_approx(radius) - lower);
  *h = v;
  *grad = (0.125f * (1.f + scaled * scaled * inv_r * inv_r) * l2u2 + 0.25f * lg * inv_r * inv_r) *
          inv_r;
}

// The pair passes' forms: SFU arithmetic in FP32, the exact expressions in FP64.
__device__ __forceinline__ float descreening_pair(float radius, float scaled, float r, float inv_r) {
  float h, g;
  descreening_fast(radius, scaled, r, inv_r, &h, &g);
  return h;
}
__device__ __forceinline__ double descreening_pair(double radius, double scaled, double r, double) {
  return descreening<double>(radius, scaled, r);
}
__device__ __forceinline__ float descreening_gradient_pair(float radius, float scaled, float r,
                                                           float inv_r) {
  float h, g;
  descreening_fast(radius, scaled, r, inv_r, &h, &g);
  return g;
}
__device__ __forceinline__ double descreening_gradient_pair(double radius, double scaled, double r,
                                                            double) {
  return descreening_gradient<double>(radius, scaled, r);
}

}  // namespace gb
}  // namespace ommb200
