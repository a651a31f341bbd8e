// Pair-interaction math shared by the nonbonded pair kernels (pair.cu, noalloc.cu):
// LJ 12-6 with optional switching plus Ewald-screened, reaction-field or bare Coulomb
// electrostatics (forces/nonbonded.rs:842-924 and 1186-1288).
#pragma once

#include "f32x2.cuh"
#include "kernels.h"

namespace ommb200 {
namespace {

template <class Real>
struct V4;
template <>
struct V4<float> {
  using T4 = float4;
  using T2 = float2;
};
template <>
struct V4<double> {
  using T4 = double4;
  using T2 = double2;
};

// Approximate SFU forms for the FP32 kernel; exact library forms for the FP64 kernel.
__device__ __forceinline__ float rsqrt_r(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float rcp_r(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rcp_r(double x) { return 1.0 / x; }
__device__ __forceinline__ float exp2_r(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double exp2_r(double x) { return exp2(x); }

// erfc(x) = exp(-x^2) P(1 / (1 + 0.46 x)), own least-squares fit (csrc/fit_erfc.py).
__device__ __forceinline__ float erfc_poly(float x) {
  const float t = rcp_r(fmaf(0.46f, x, 1.0f));
  float p = 0.10014041224442242f;
  p = fmaf(p, t, -0.504550213499043f);
  p = fmaf(p, t, 0.8277608617691994f);
  p = fmaf(p, t, -0.35775472734883446f);
  p = fmaf(p, t, 0.4707476000236329f);
  p = fmaf(p, t, 0.1949991373822864f);
  p = fmaf(p, t, 0.2692933367874065f);
  p = fmaf(p, t, -0.0006363939510855f);
  return p;
}

// The reference's cutoff decision for particles a, b (original indices).
__device__ __forceinline__ bool exact_inside(const double* pos, int a, int b, int periodic,
                                             const Box<double>& box, double rc2) {
  const int i = a < b ? a : b, j = a < b ? b : a;
  double dx = __dsub_rn(pos[3 * j], pos[3 * i]);
  double dy = __dsub_rn(pos[3 * j + 1], pos[3 * i + 1]);
  double dz = __dsub_rn(pos[3 * j + 2], pos[3 * i + 2]);
  if (periodic) min_image_exact(dx, dy, dz, box);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return r2 < rc2;
}

// dE/dr / r and E of one pair at squared distance r2 with inv_r = 1 / sqrt(r2);
// `eps4` = 4 sqrt(eps_i eps_j), `sig` = (sigma_i + sigma_j) / 2.
template <class Real, int kElec, bool kEnergy, bool kSwitch>
__device__ __forceinline__ void pair_terms_r(const PairArgs<Real>& a, Real r2, Real inv_r, Real qq,
                                             Real sig, Real eps4, Real& f_over_r, Real& energy) {
  const Real inv_r2 = inv_r * inv_r;
  // LJ 12-6 (nonbonded.rs:1203-1214)
  const Real s2 = sig * sig * inv_r2;
  const Real s6 = s2 * s2 * s2;
  Real f_lj = eps4 * s6 * fma(Real(-12), s6, Real(6)) * inv_r2;
  Real e_lj = kEnergy ? eps4 * s6 * (s6 - Real(1)) : Real(0);
  if (eps4 == Real(0)) {
    f_lj = Real(0);
    e_lj = Real(0);
  }
  // switching (nonbonded.rs:888-900)
  if (kSwitch) {
    const Real r = r2 * inv_r;
    if (r > a.switch_r) {
      const Real e_full = eps4 * s6 * (s6 - Real(1));
      const Real t = (r - a.switch_r) * a.switch_inv_width;
      const Real sw = Real(1) + t * t * t * (Real(-10) + t * (Real(15) - Real(6) * t));
      const Real dsw = Real(-30) * t * t * (Real(1) - t) * (Real(1) - t) * a.switch_inv_width;
      f_lj = sw * f_lj + (eps4 == Real(0) ? Real(0) : e_full) * dsw * inv_r;
      e_lj = kEnergy ? e_lj * sw : Real(0);
    }
  }
  Real f_el, e_el = Real(0);
  if (kElec == kElecEwald) {
    // screened_coulomb (nonbonded.rs:1263-1273)
    const Real r = r2 * inv_r;
    Real ex, ec;
    if constexpr (sizeof(Real) == 4) {
      ex = exp2_r(a.exp_scale * r2);
      ec = ex * erfc_poly(a.alpha * r);
    } else {
      ex = exp(a.exp_scale * r2);
      ec = erfc(a.alpha * r);
    }
    f_el = -qq * fma(ec, inv_r, a.two_alpha_sqrtpi * ex) * inv_r2;
    if (kEnergy) e_el = qq * ec * inv_r;
  } else if (kElec == kElecReactionField) {
    // reaction_field (nonbonded.rs:1222-1243)
    f_el = qq * (Real(2) * a.krf - inv_r * inv_r2);
    if (kEnergy) e_el = qq * (inv_r + a.krf * r2 - a.crf);
  } else {
    // coulomb_pair (nonbonded.rs:1186-1192)
    f_el = -qq * inv_r * inv_r2;
    if (kEnergy) e_el = qq * inv_r;
  }
  f_over_r = f_lj + f_el;
  energy = e_lj + e_el;
}

template <class Real, int kElec, bool kEnergy, bool kSwitch>
__device__ __forceinline__ void pair_terms(const PairArgs<Real>& a, Real r2, Real qq, Real sig,
                                           Real eps4, Real& f_over_r, Real& energy) {
  pair_terms_r<Real, kElec, kEnergy, kSwitch>(a, r2, rsqrt_r(r2), qq, sig, eps4, f_over_r, energy);
}

// pair_terms for two pairs at once in the lanes of packed FP32 values (same operations and
// rounding as the scalar FP32 form, erfc by the same fit).
template <int kElec, bool kEnergy, bool kSwitch>
__device__ __forceinline__ void pair_terms_x2(const PairArgs<float>& a, float2 r2, float2 qq,
                                              float2 sig, float2 eps4, float2& f_over_r,
                                              float2& energy) {
  const float2 inv_r = x2::rsqrt_approx(r2);
  const float2 inv_r2 = x2::mul(inv_r, inv_r);
  // LJ 12-6 (nonbonded.rs:1203-1214)
  const float2 s2 = x2::mul(x2::mul(sig, sig), inv_r2);
  const float2 s6 = x2::mul(x2::mul(s2, s2), s2);
  const float2 e6 = x2::mul(eps4, s6);
  float2 f_lj = x2::mul(x2::mul(e6, x2::fma(x2::bc(-12.f), s6, x2::bc(6.f))), inv_r2);
  float2 e_lj = kEnergy ? x2::mul(e6, x2::add(s6, x2::bc(-1.f))) : x2::bc(0.f);
  if (eps4.x == 0.f) f_lj.x = e_lj.x = 0.f;
  if (eps4.y == 0.f) f_lj.y = e_lj.y = 0.f;
  if (kSwitch) {  // nonbonded.rs:888-900, per lane (switching is the uncommon path)
    const float2 r = x2::mul(r2, inv_r);
    auto sw = [&](float rr, float e4, float s6v, float ir, float& f, float& e) {
      if (rr > a.switch_r) {
        const float e_full = e4 * s6v * (s6v - 1.f);
        const float t = (rr - a.switch_r) * a.switch_inv_width;
        const float s = 1.f + t * t * t * (-10.f + t * (15.f - 6.f * t));
        const float ds = -30.f * t * t * (1.f - t) * (1.f - t) * a.switch_inv_width;
        f = s * f + (e4 == 0.f ? 0.f : e_full) * ds * ir;
        e = kEnergy ? e * s : 0.f;
      }
    };
    sw(r.x, eps4.x, s6.x, inv_r.x, f_lj.x, e_lj.x);
    sw(r.y, eps4.y, s6.y, inv_r.y, f_lj.y, e_lj.y);
  }
  // The energy adds the electrostatic term to the LJ one with one rounding (a fused multiply-add):
  // rounding the product first would drop every LJ tail smaller than half its unit in the last
  // place, a bias that grows with the number of distant pairs.
  if (kElec == kElecEwald) {
    // screened_coulomb (nonbonded.rs:1263-1273): exp(-a^2 r^2) by exp2, erfc by the fit
    const float2 r = x2::mul(r2, inv_r);
    const float2 ex = x2::exp2_approx(x2::mul(x2::bc(a.exp_scale), r2));
    const float2 t = x2::rcp_approx(x2::fma(x2::bc(0.46f), x2::mul(x2::bc(a.alpha), r), x2::bc(1.f)));
    float2 p = x2::bc(0.10014041224442242f);
    p = x2::fma(p, t, x2::bc(-0.504550213499043f));
    p = x2::fma(p, t, x2::bc(0.8277608617691994f));
    p = x2::fma(p, t, x2::bc(-0.35775472734883446f));
    p = x2::fma(p, t, x2::bc(0.4707476000236329f));
    p = x2::fma(p, t, x2::bc(0.1949991373822864f));
    p = x2::fma(p, t, x2::bc(0.2692933367874065f));
    p = x2::fma(p, t, x2::bc(-0.0006363939510855f));
    const float2 ec = x2::mul(ex, p);
    const float2 v = x2::fma(ec, inv_r, x2::mul(x2::bc(a.two_alpha_sqrtpi), ex));
    f_over_r = x2::sub(f_lj, x2::mul(x2::mul(qq, v), inv_r2));
    if (kEnergy) energy = x2::fma(x2::mul(qq, ec), inv_r, e_lj);
  } else if (kElec == kElecReactionField) {
    // reaction_field (nonbonded.rs:1222-1243)
    f_over_r = x2::add(f_lj, x2::mul(qq, x2::sub(x2::bc(2.f * a.krf), x2::mul(inv_r, inv_r2))));
    if (kEnergy)
      energy = x2::fma(qq, x2::sub(x2::fma(x2::bc(a.krf), r2, inv_r), x2::bc(a.crf)), e_lj);
  } else {
    // coulomb_pair (nonbonded.rs:1186-1192)
    f_over_r = x2::sub(f_lj, x2::mul(x2::mul(qq, inv_r), inv_r2));
    if (kEnergy) energy = x2::fma(qq, inv_r, e_lj);
  }
  if (!kEnergy) energy = x2::bc(0.f);
}


}  // namespace
}  // namespace ommb200
