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

}  // namespace gb
}  // namespace ommb200
