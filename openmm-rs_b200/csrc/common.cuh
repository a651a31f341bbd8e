// Shared device helpers of the B200 force/integration engine: fixed-point accumulation,
// minimum image, the single-precision erfc, the Philox Gaussian stream and error words.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace ommb200 {

// 1/(4 pi eps0) in kJ/mol nm / e^2 (crates/openmm-core/src/forces/nonbonded.rs:16).
constexpr double kOne4PiEps0 = 138.93545764438198;
constexpr double kPiD = 3.14159265358979323846;
// Boltzmann constant in kJ/mol/K (crates/openmm-core/src/integrators/langevin.rs:13).
constexpr double kBoltzmann = 1.380649e-23 * 6.02214076e23 / 1000.0;

// Forces accumulate as signed 64-bit integers in units of 2^-32 kJ/mol/nm; integer addition
// is associative, so the sum is independent of launch order and bit-identical run to run.
constexpr double kForceScale = 4294967296.0;        // 2^32
constexpr double kForceScaleInv = 1.0 / 4294967296.0;
// Energies and virials accumulate in units of 2^-32 kJ/mol (range +-2.1e9 kJ/mol).
constexpr double kEnergyScale = 4294967296.0;        // 2^32
constexpr double kEnergyScaleInv = 1.0 / 4294967296.0;
// PME charge grid: units of 2^-40 e (a grid point can hold up to 8.4e6 e).
constexpr double kGridScale = 1099511627776.0;  // 2^40
constexpr double kGridScaleInv = 1.0 / 1099511627776.0;

// Device status word bits (first error wins; the host maps them to OMMB200_ERR_*).
enum DeviceStatus : int {
  kStatusOk = 0,
  kStatusConstraint = 1,
  kStatusNonfinite = 2,
  kStatusTileOverflow = 3,
  kStatusTimeout = 4,
};

__device__ __forceinline__ void report_status(int* status, int code) {
  atomicCAS(status, 0, code);
}

__device__ __forceinline__ long long to_fixed(float v, float scale) {
  return __float2ll_rn(v * scale);
}
__device__ __forceinline__ long long to_fixed(double v, double scale) {
  return __double2ll_rn(v * scale);
}
__device__ __forceinline__ void add_fixed(long long* dst, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(dst), static_cast<unsigned long long>(v));
}

template <class Real>
struct Vec3 {
  Real x, y, z;
};

// Reduced-triclinic box: rows a=(ax,0,0), b=(bx,by,0), c=(cx,cy,cz) plus reciprocal rows.
template <class Real>
struct Box {
  Real ax, bx, by, cx, cy, cz;
  Real inv_ax, inv_by, inv_cz;
};

// Position x of a particle relative to the centre c of its block, in the frame of the lattice
// image n it was given at the last neighbour-list rebuild, with explicitly rounded operations
// (the pack kernel and the integrator both write these and must agree bit for bit).
__device__ __forceinline__ void block_local(const double x[3], double n0, double n1, double n2,
                                            const double* c, const Box<double>& b, double o[3]) {
  o[0] = __dsub_rn(__dsub_rn(x[0], __dadd_rn(__dadd_rn(__dmul_rn(n0, b.ax), __dmul_rn(n1, b.bx)),
                                             __dmul_rn(n2, b.cx))),
                   c[0]);
  o[1] = __dsub_rn(__dsub_rn(x[1], __dadd_rn(__dmul_rn(n1, b.by), __dmul_rn(n2, b.cy))), c[1]);
  o[2] = __dsub_rn(__dsub_rn(x[2], __dmul_rn(n2, b.cz)), c[2]);
}

// Minimum image in the reference's exact sequence (harmonic_bond.rs:152-159), computed
// with explicitly rounded operations so that no fused multiply-add changes the result.
__device__ __forceinline__ void min_image_exact(double& dx, double& dy, double& dz,
                                                const Box<double>& b) {
  double s = floor(__dadd_rn(__ddiv_rn(dz, b.cz), 0.5));
  dx = __dsub_rn(dx, __dmul_rn(s, b.cx));
  dy = __dsub_rn(dy, __dmul_rn(s, b.cy));
  dz = __dsub_rn(dz, __dmul_rn(s, b.cz));
  s = floor(__dadd_rn(__ddiv_rn(dy, b.by), 0.5));
  dx = __dsub_rn(dx, __dmul_rn(s, b.bx));
  dy = __dsub_rn(dy, __dmul_rn(s, b.by));
  s = floor(__dadd_rn(__ddiv_rn(dx, b.ax), 0.5));
  dx = __dsub_rn(dx, __dmul_rn(s, b.ax));
}

// Fast minimum image for the arithmetic path (same sequence, any rounding).
template <class Real>
__device__ __forceinline__ void min_image_fast(Real& dx, Real& dy, Real& dz, const Box<Real>& b) {
  Real s = floor(dz * b.inv_cz + Real(0.5));
  dx -= s * b.cx;
  dy -= s * b.cy;
  dz -= s * b.cz;
  s = floor(dy * b.inv_by + Real(0.5));
  dx -= s * b.bx;
  dy -= s * b.by;
  s = floor(dx * b.inv_ax + Real(0.5));
  dx -= s * b.ax;
}

// erfc(x) for 0 <= x <= 4.2 as exp(-x^2) * P(t), t = 1/(1 + 0.46 x): an own least-squares
// fit of erfcx (csrc/fit_erfc.py), ~4e-7 relative in float.  `expmx2` = exp(-x^2).
__device__ __forceinline__ float erfc_fit(float x, float expmx2) {
  const float t = __frcp_rn(fmaf(0.46f, x, 1.0f));
  float p = 0.10014041224442242f;
  p = fmaf(p, t, -0.504550213499043f);
  p = fmaf(p, t, 0.8277608617691994f);
  p = fmaf(p, t, -0.35775472734883446f);
  p = fmaf(p, t, 0.4707476000236329f);
  p = fmaf(p, t, 0.1949991373822864f);
  p = fmaf(p, t, 0.2692933367874065f);
  p = fmaf(p, t, -0.0006363939510855f);
  return expmx2 * p;
}

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11) and Box-Muller normals.  The counter is
// (atom, step lo, step hi, stream) and the key the 64-bit seed, so every atom's noise at every
// step is an independent, reproducible draw (the CPU oracle implements the same stream).
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)M0 * c[0];
    const uint64_t p1 = (uint64_t)M1 * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0;
    const uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

__device__ __forceinline__ void gaussian3(uint64_t seed, uint64_t stream, uint64_t step,
                                          uint32_t atom, double out[3]) {
  uint32_t c[4] = {atom, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)stream};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double s = 2.3283064365386962890625e-10;  // 2^-32
  const double u0 = ((double)c[0] + 0.5) * s, u1 = ((double)c[1] + 0.5) * s;
  const double u2 = ((double)c[2] + 0.5) * s, u3 = ((double)c[3] + 0.5) * s;
  const double m0 = sqrt(-2.0 * log(u0));
  const double m1 = sqrt(-2.0 * log(u2));
  double s1, c1, s3, c3;
  sincos(2.0 * kPiD * u1, &s1, &c1);
  sincos(2.0 * kPiD * u3, &s3, &c3);
  out[0] = m0 * c1;
  out[1] = m0 * s1;
  out[2] = m1 * c3;
}

__host__ __device__ __forceinline__ int ceil_div(long long a, long long b) {
  return (int)((a + b - 1) / b);
}

}  // namespace ommb200
