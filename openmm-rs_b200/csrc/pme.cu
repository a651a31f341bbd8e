// PME reciprocal space (forces/pme.rs:141-425): order-5 cardinal B-spline spreading of the
// charges, 3-D FFT (cuFFT, real-to-complex), multiplication by the influence function, inverse
// FFT and force gather.
//
// The reference transforms the full complex grid; here the charge grid is real, so the
// forward transform is R2C and only the kz <= nz/2 half is stored.  The influence table holds
// 0.5 * (G(m) + G(m')) for each stored element m and its conjugate partner m' (the reference's
// mode numbering makes them differ only on Nyquist planes of triclinic boxes), which is exactly
// what the reference's "real part of the inverse transform" keeps.  The energy is
// 0.5 * sum_full G |S|^2 = sum_half w * 0.5 * G_sym |S|^2 with w = 1 on the kz = 0 and
// kz = nz/2 planes and 2 elsewhere.
//
// Charges are spread into a 64-bit fixed-point grid (units of 2^-40 e) so the grid, and every
// force derived from it, is independent of the order of the atomic additions.
#include "kernels.h"

namespace ommb200 {
namespace {

// pme.rs:151-174
template <class Real>
__device__ __forceinline__ void spline5(Real f, Real w[5], Real dw[5]) {
  w[0] = Real(1) - f;
  w[1] = f;
  w[2] = w[3] = w[4] = Real(0);
#pragma unroll
  for (int order = 3; order <= 5; ++order) {
    if (order == 5) {
      dw[0] = -w[0];
#pragma unroll
      for (int i = 1; i < 5; ++i) dw[i] = w[i - 1] - w[i];
    }
    const Real inv = Real(1) / Real(order - 1);
    w[order - 1] = f * w[order - 2] * inv;
#pragma unroll
    for (int i = order - 2; i >= 1; --i)
      w[i] = ((f + Real(order - 1 - i)) * w[i - 1] + (Real(i + 1) - f) * w[i]) * inv;
    w[0] *= (Real(1) - f) * inv;
  }
}

// pme.rs:201-218: base grid index and fraction along each axis, in f64.  Returns false for a
// nonfinite position, which then touches no grid point (the integrator reports it).
template <class Real>
__device__ __forceinline__ bool stencil(const PmeArgs<Real>& a, int atom, int base[3],
                                        Real frac[3]) {
  const double x = a.pos[3 * atom], y = a.pos[3 * atom + 1], z = a.pos[3 * atom + 2];
  const int dims[3] = {a.nx, a.ny, a.nz};
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double f = x * a.recip[d][0] + y * a.recip[d][1] + z * a.recip[d][2];
    const double coord = (f - floor(f)) * (double)dims[d];
    ok = ok && coord >= 0.0 && coord <= (double)dims[d];
    const double fl = ok ? floor(coord) : 0.0;
    int b = (int)fl;
    b %= dims[d];
    base[d] = b;
    frac[d] = (Real)(ok ? coord - fl : 0.0);
  }
  return ok;
}

template <class Real>
__global__ void spread_kernel(const PmeArgs<Real> a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_order) return;
  const int atom = a.order ? a.order[s] : s;
  if (atom < 0) return;
  const double qd = a.charge[atom];
  if (qd == 0.0) return;
  const Real q = (Real)qd;
  int base[3];
  Real frac[3], w[3][5], dw[3][5];
  if (!stencil(a, atom, base, frac)) return;
#pragma unroll
  for (int d = 0; d < 3; ++d) spline5(frac[d], w[d], dw[d]);
  const Real gscale = Real(kGridScale);
  for (int ix = 0; ix < 5; ++ix) {
    int gx = base[0] + ix;
    gx -= gx >= a.nx ? a.nx : 0;
    const Real qx = q * w[0][ix];
    for (int iy = 0; iy < 5; ++iy) {
      int gy = base[1] + iy;
      gy -= gy >= a.ny ? a.ny : 0;
      const Real qxy = qx * w[1][iy];
      long long* row = a.grid_fixed + ((long long)gx * a.ny + gy) * a.nz;
#pragma unroll
      for (int iz = 0; iz < 5; ++iz) {
        int gz = base[2] + iz;
        gz -= gz >= a.nz ? a.nz : 0;
        add_fixed(row + gz, to_fixed(qxy * w[2][iz], gscale));
      }
    }
  }
}

// Staged spreading: a CTA takes 64 consecutive sorted slots (spatially compact: part of one
// x-y column, z-sorted), two threads per atom, and adds the atoms' 125-point stencils into a
// shared-memory copy of the grid box they touch, then adds that box to the global grid, so
// each grid point receives one global atomic per CTA instead of one per stencil.  Shared
// accumulation uses native 32-bit integer atomics (64-bit shared atomics measured 1.5-1.8x
// slower).  FP64 form: a split of each 2^-40 fixed-point value, v = hi 2^20 + lo with
// 0 <= lo < 2^20; at most 64 contributions per cell keep both partial sums inside 32 bits (for
// |q| < 16 e), and hi_sum 2^20 + lo_sum recovers the exact 64-bit total.  FP32 form: one atomic
// per point, each contribution (a float product) rounded to 2^-26 e, which keeps 64 of them
// inside 32 bits for |q| < 2 e (the order-5 B-spline peaks at 115/192 per axis, so a point gets
// at most 0.22 |q| from an atom); the box is added to the 2^-40 global grid scaled by 2^14,
// exactly.  Either way the sums are exact integers, so the grid does not depend on the order
// of the additions.  A CTA whose box exceeds kSpreadCells (it straddles a periodic edge of the
// column order) or that holds a larger charge spreads directly.
constexpr int kSpreadAtoms = 64;
constexpr int kSpreadCells = 4096;
constexpr float kSpreadScale32 = 67108864.f;           // 2^26 (FP32 form, staged)
constexpr long long kSpreadWiden32 = 1ll << 14;        // 2^40 / 2^26

template <class Real>
__global__ void __launch_bounds__(2 * kSpreadAtoms) spread_staged_kernel(const PmeArgs<Real> a) {
  __shared__ int c_hi[kSpreadCells];
  __shared__ unsigned int c_lo[kSpreadCells];
  __shared__ int s_lo[3], s_hi[3], s_big;
  const int tid = threadIdx.x, half = tid / kSpreadAtoms;  // half 0: ix 0..2, half 1: ix 3..4
  const int s = blockIdx.x * kSpreadAtoms + (tid % kSpreadAtoms);
  int atom = -1;
  if (s < a.n_order) atom = a.order ? a.order[s] : s;
  const double qd = atom >= 0 ? a.charge[atom] : 0.0;
  int base[3] = {0, 0, 0};
  Real frac[3] = {Real(0), Real(0), Real(0)};
  const bool ok = atom >= 0 && qd != 0.0 && stencil(a, atom, base, frac);
  if (tid < 3) {
    s_lo[tid] = 0x7fffffff;
    s_hi[tid] = -1;
  }
  if (tid == 0) s_big = 0;
  __syncthreads();
  if (ok && half == 0) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(&s_lo[d], base[d]);
      atomicMax(&s_hi[d], base[d]);
    }
    // the 32-bit partial sums need |q| < 2 e (FP32 form) or |q| < 16 e (FP64 form)
    if (fabs(qd) >= (sizeof(Real) == 4 ? 2.0 : 16.0)) s_big = 1;
  }
  __syncthreads();
  if (s_hi[0] < 0) return;  // no charged atom in this CTA (uniform)
  const int lo0 = s_lo[0], lo1 = s_lo[1], lo2 = s_lo[2];
  const int ex = s_hi[0] - lo0 + 5, ey = s_hi[1] - lo1 + 5, ez = s_hi[2] - lo2 + 5;
  const long long n_cells = s_big ? (long long)kSpreadCells + 1 : (long long)ex * ey * ez;
  Real w[3][5], dw[3][5];
  if (ok) {
#pragma unroll
    for (int d = 0; d < 3; ++d) spline5(frac[d], w[d], dw[d]);
  }
  const Real q = (Real)qd;
  const Real gscale = Real(kGridScale);
  const int ix0 = half == 0 ? 0 : 3, ix1 = half == 0 ? 3 : 5;
  if (n_cells > kSpreadCells) {  // direct spreading (uniform branch)
    if (!ok) return;
    for (int ix = ix0; ix < ix1; ++ix) {
      int gx = base[0] + ix;
      gx -= gx >= a.nx ? a.nx : 0;
      const Real qx = q * w[0][ix];
      for (int iy = 0; iy < 5; ++iy) {
        int gy = base[1] + iy;
        gy -= gy >= a.ny ? a.ny : 0;
        const Real qxy = qx * w[1][iy];
        long long* row = a.grid_fixed + ((long long)gx * a.ny + gy) * a.nz;
#pragma unroll
        for (int iz = 0; iz < 5; ++iz) {
          int gz = base[2] + iz;
          gz -= gz >= a.nz ? a.nz : 0;
          add_fixed(row + gz, to_fixed(qxy * w[2][iz], gscale));
        }
      }
    }
    return;
  }
  const int nc = (int)n_cells;
  for (int c = tid; c < nc; c += 2 * kSpreadAtoms) {
    c_hi[c] = 0;
    if constexpr (sizeof(Real) == 8) c_lo[c] = 0u;
  }
  __syncthreads();
  if (ok) {
    for (int ix = ix0; ix < ix1; ++ix) {
      const Real qx = q * w[0][ix];
      for (int iy = 0; iy < 5; ++iy) {
        const Real qxy = qx * w[1][iy];
        const int row = ((base[0] - lo0 + ix) * ey + (base[1] - lo1 + iy)) * ez + (base[2] - lo2);
#pragma unroll
        for (int iz = 0; iz < 5; ++iz) {
          if constexpr (sizeof(Real) == 4) {
            atomicAdd(&c_hi[row + iz], __float2int_rn(qxy * w[2][iz] * kSpreadScale32));
          } else {
            const long long v = to_fixed(qxy * w[2][iz], gscale);
            atomicAdd(&c_hi[row + iz], (int)(v >> 20));
            atomicAdd(&c_lo[row + iz], (unsigned int)(v & 0xFFFFF));
          }
        }
      }
    }
  }
  __syncthreads();
  for (int c = tid; c < nc; c += 2 * kSpreadAtoms) {
    const long long v = sizeof(Real) == 4 ? (long long)c_hi[c] * kSpreadWiden32
                                          : (long long)c_hi[c] * (1ll << 20) + (long long)c_lo[c];
    if (v == 0) continue;
    const int cz = c % ez, cy = (c / ez) % ey, cx = c / (ez * ey);
    int gx = lo0 + cx, gy = lo1 + cy, gz = lo2 + cz;
    gx -= gx >= a.nx ? a.nx : 0;
    gy -= gy >= a.ny ? a.ny : 0;
    gz -= gz >= a.nz ? a.nz : 0;
    add_fixed(a.grid_fixed + ((long long)gx * a.ny + gy) * a.nz + gz, v);
  }
}

template <class Real>
__global__ void convert_kernel(const PmeArgs<Real> a) {
  const long long total = (long long)a.nx * a.ny * a.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    a.grid_real[i] = (Real)((double)a.grid_fixed[i] * kGridScaleInv);
    a.grid_fixed[i] = 0;
  }
}

template <class Real>
struct Cplx;
template <>
struct Cplx<float> {
  using T = float2;
};
template <>
struct Cplx<double> {
  using T = double2;
};

__device__ __forceinline__ double freq(int k, int n) { return k < (n + 1) / 2 ? (double)k : (double)(k - n); }

template <class Real, bool kEnergy>
__global__ void convolve_kernel(const PmeArgs<Real> a, const double* moduli) {
  using C2 = typename Cplx<Real>::T;
  C2* g = reinterpret_cast<C2*>(a.grid_k);
  const int nzh = a.nz / 2 + 1;
  const long long total = (long long)a.nx * a.ny * nzh;
  double e = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    C2 v = g[i];
    const Real infl = a.influence[i];
    if (kEnergy && i != 0) {
      const int z = (int)(i % nzh);
      const int y = (int)((i / nzh) % a.ny);
      const int x = (int)(i / ((long long)nzh * a.ny));
      const double wz = (z == 0 || (a.nz % 2 == 0 && z == a.nz / 2)) ? 1.0 : 2.0;
      const double s2 = (double)v.x * v.x + (double)v.y * v.y;
      e += wz * 0.5 * (double)infl * s2;
      // virial: average over the element's mode and its conjugate partner's mode
      const int idx[2][3] = {{x, y, z}, {(a.nx - x) % a.nx, (a.ny - y) % a.ny, (a.nz - z) % a.nz}};
      for (int p = 0; p < 2; ++p) {
        const double m[3] = {freq(idx[p][0], a.nx), freq(idx[p][1], a.ny), freq(idx[p][2], a.nz)};
        double k[3];
        for (int c = 0; c < 3; ++c) k[c] = m[0] * a.recip[0][c] + m[1] * a.recip[1][c] + m[2] * a.recip[2][c];
        const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        const double bm = moduli[idx[p][0]] * moduli[a.nx + idx[p][1]] * moduli[a.nx + a.ny + idx[p][2]];
        const double pa = kPiD * kPiD / (a.alpha * a.alpha);
        const double g_m = kOne4PiEps0 * exp(-pa * k2) / (kPiD * a.volume * k2 * bm);
        const double em = wz * 0.5 * 0.5 * g_m * s2;
        const double c = 2.0 * (1.0 + pa * k2) / k2;
        w[0] += em * (1.0 - c * k[0] * k[0]);
        w[1] += em * (1.0 - c * k[1] * k[1]);
        w[2] += em * (1.0 - c * k[2] * k[2]);
        w[3] -= em * c * k[0] * k[1];
        w[4] -= em * c * k[0] * k[2];
        w[5] -= em * c * k[1] * k[2];
      }
    }
    v.x *= infl;
    v.y *= infl;
    g[i] = v;
  }
  if (kEnergy) {
    long long ef = to_fixed(e, kEnergyScale);
    long long wf[6];
    for (int c = 0; c < 6; ++c) wf[c] = to_fixed(w[c], kEnergyScale);
    for (int off = 16; off > 0; off >>= 1) {
      ef += __shfl_xor_sync(0xffffffffu, ef, off);
      for (int c = 0; c < 6; ++c) wf[c] += __shfl_xor_sync(0xffffffffu, wf[c], off);
    }
    if ((threadIdx.x & 31) == 0) {
      add_fixed(a.energy, ef);
      for (int c = 0; c < 6; ++c) add_fixed(a.energy + 1 + c, wf[c]);
    }
  }
}

// pme.rs:377-425.  Eight lanes per atom: lane k < 5 sums the 25 grid points of stencil plane
// ix = k, then the group reduces by a fixed shuffle tree and lane 0 commits the force.
template <class Real>
__global__ void gather_kernel(const PmeArgs<Real> a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t >> 3, k = t & 7;
  int atom = -1;
  if (s < a.n_order) atom = a.order ? a.order[s] : s;
  const double qd = atom >= 0 ? a.charge[atom] : 0.0;
  int base[3] = {0, 0, 0};
  Real frac[3] = {Real(0), Real(0), Real(0)};
  const bool ok = atom >= 0 && qd != 0.0 && stencil(a, atom, base, frac);
  Real g0 = 0, g1 = 0, g2 = 0;
  if (ok && k < 5) {
    Real w[3][5], dw[3][5];
#pragma unroll
    for (int d = 0; d < 3; ++d) spline5(frac[d], w[d], dw[d]);
    int gx = base[0] + k;
    gx -= gx >= a.nx ? a.nx : 0;
    Real wx = w[0][0], dwx = dw[0][0];
#pragma unroll
    for (int i = 1; i < 5; ++i)
      if (k == i) {
        wx = w[0][i];
        dwx = dw[0][i];
      }
    for (int iy = 0; iy < 5; ++iy) {
      int gy = base[1] + iy;
      gy -= gy >= a.ny ? a.ny : 0;
      const Real* row = a.grid_real + ((long long)gx * a.ny + gy) * a.nz;
      const Real wxy = wx * w[1][iy];
      const Real dxy = dwx * w[1][iy];
      const Real xdy = wx * dw[1][iy];
#pragma unroll
      for (int iz = 0; iz < 5; ++iz) {
        int gz = base[2] + iz;
        gz -= gz >= a.nz ? a.nz : 0;
        const Real phi = row[gz];
        g0 += phi * dxy * w[2][iz];
        g1 += phi * xdy * w[2][iz];
        g2 += phi * wxy * dw[2][iz];
      }
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    g0 += __shfl_xor_sync(0xffffffffu, g0, o, 8);
    g1 += __shfl_xor_sync(0xffffffffu, g1, o, 8);
    g2 += __shfl_xor_sync(0xffffffffu, g2, o, 8);
  }
  if (!ok || k != 0) return;
  const double gd[3] = {(double)g0 * a.nx, (double)g1 * a.ny, (double)g2 * a.nz};
  for (int c = 0; c < 3; ++c) {
    const double f = -qd * (gd[0] * a.recip[0][c] + gd[1] * a.recip[1][c] + gd[2] * a.recip[2][c]);
    add_fixed(a.force + (long long)c * a.n_atoms + atom, to_fixed(f, kForceScale));
  }
}

// ---- own 3-D transform of the PME grid -------------------------------------------------
// Replaces the fixed-point conversion, the real-to-complex / complex-to-real cuFFT pair and
// the convolution by three kernels over the half spectrum [x][y][kz <= nz/2]:
//   planes_forward  one CTA per x plane: fixed-point grid -> real (grid zeroed), z transform
//                   of two real rows at once as one complex row, y transform
//   x_convolve      one CTA per (y, run of kz): x transform, influence function (+ energy
//                   and virial), inverse x transform
//   planes_inverse  one CTA per x plane: inverse y transform, inverse z transform of two
//                   Hermitian rows at once, real rows -> potential grid for the gather
// Every 1-D transform is a mixed-radix Stockham FFT in shared memory (radices 2, 3, 4, 5, 7,
// 8; one radix-R butterfly per thread and stage), forward sign exp(-2 pi i jk/n) and
// unnormalised like cuFFT; the inverse is conj(F(conj(x))).  Sizes with other prime factors
// use cuFFT.
template <class C2>
__device__ __forceinline__ C2 cmul(C2 a, C2 w) {
  C2 r;
  r.x = a.x * w.x - a.y * w.y;
  r.y = a.x * w.y + a.y * w.x;
  return r;
}
template <class C2>
__device__ __forceinline__ C2 conjg(C2 a) {
  a.y = -a.y;
  return a;
}
template <class C2>
__device__ __forceinline__ void bfly2(C2& a, C2& b) {
  const C2 t = a;
  a.x = t.x + b.x;
  a.y = t.y + b.y;
  b.x = t.x - b.x;
  b.y = t.y - b.y;
}
// multiplication by -i
template <class C2>
__device__ __forceinline__ C2 mul_mi(C2 a) {
  C2 r;
  r.x = a.y;
  r.y = -a.x;
  return r;
}
template <class C2>
__device__ __forceinline__ void dft4(C2& a0, C2& a1, C2& a2, C2& a3) {
  bfly2(a0, a2);  // a0 = x0 + x2, a2 = x0 - x2
  bfly2(a1, a3);  // a1 = x1 + x3, a3 = x1 - x3
  a3 = mul_mi(a3);
  bfly2(a0, a1);  // y0, y2
  bfly2(a2, a3);  // y1, y3
  const C2 y1 = a2, y2 = a1;
  a1 = y1;
  a2 = y2;
}

// Forward DFT of R values in registers.  Radices 2, 4, 8 use butterflies; the odd primes use
// the direct sum with W_R^q = tw[q n / R] from the length-n twiddle table.
template <int R, class C2>
__device__ __forceinline__ void dft_reg(C2 (&v)[R], const C2* tw, int n) {
  using S = decltype(v[0].x);
  if constexpr (R == 2) {
    bfly2(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft4(v[0], v[2], v[4], v[6]);
    dft4(v[1], v[3], v[5], v[7]);
    const S h = (S)0.70710678118654752440;  // 1/sqrt(2)
    C2 o1, o2, o3;
    o1.x = h * (v[3].x + v[3].y);  // W_8 = (1 - i)/sqrt(2)
    o1.y = h * (v[3].y - v[3].x);
    o2 = mul_mi(v[5]);              // W_8^2 = -i
    o3.x = h * (v[7].y - v[7].x);  // W_8^3 = -(1 + i)/sqrt(2)
    o3.y = -h * (v[7].x + v[7].y);
    C2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], d0 = v[1];
    bfly2(e0, d0);
    bfly2(e1, o1);
    bfly2(e2, o2);
    bfly2(e3, o3);
    v[0] = e0; v[4] = d0;
    v[1] = e1; v[5] = o1;
    v[2] = e2; v[6] = o2;
    v[3] = e3; v[7] = o3;
  } else {
    const int st = n / R;
    C2 out[R];
#pragma unroll
    for (int s = 0; s < R; ++s) {
      C2 acc = v[0];
#pragma unroll
      for (int q = 1; q < R; ++q) {
        const C2 w = tw[((q * s) % R) * st];
        acc.x += v[q].x * w.x - v[q].y * w.y;
        acc.y += v[q].x * w.y + v[q].y * w.x;
      }
      out[s] = acc;
    }
#pragma unroll
    for (int s = 0; s < R; ++s) v[s] = out[s];
  }
}

// One Stockham stage over P pencils of length n (pencil p at in + p n): butterfly j of a
// pencil reads in[j + r n/R], applies the twiddles W_n^(r k n/(ns R)) of its position
// k = j mod ns in the current sub-transforms of length ns, and writes out[(j/ns) ns R + k + r ns].
// Not inlined: every transform of a kernel shares one copy of each radix's code, which keeps
// the instruction footprint of a CTA (one CTA per SM, every stage a new code path) small.
template <int R, class C2>
__device__ __noinline__ void stockham_stage(const C2* in, C2* out, const C2* tw, int n, int ns, int P) {
  const int nr = n / R, items = P * nr, span = n / (ns * R);
  for (int t = threadIdx.x; t < items; t += blockDim.x) {
    const int p = t / nr, j = t - p * nr, q = j / ns, k = j - q * ns;
    const C2* src = in + p * n + j;
    C2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[r * nr];
    if (ns > 1) {
      const int step = k * span;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[r * step]);
    }
    dft_reg<R>(v, tw, n);
    C2* dst = out + p * n + q * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * ns] = v[r];
  }
}

// Forward transform of P pencils held in a (b: scratch of the same size); returns the buffer
// that holds the result.  The callers synchronise before and after.
template <class C2>
__device__ C2* stockham(C2* a, C2* b, const C2* tw, const PmeFft& f, int axis, int n, int P) {
  int ns = 1;
  for (int s = 0; s < f.nrad[axis]; ++s) {
    const int R = f.rad[axis][s];
    switch (R) {
      case 2: stockham_stage<2>(a, b, tw, n, ns, P); break;
      case 3: stockham_stage<3>(a, b, tw, n, ns, P); break;
      case 4: stockham_stage<4>(a, b, tw, n, ns, P); break;
      case 5: stockham_stage<5>(a, b, tw, n, ns, P); break;
      case 7: stockham_stage<7>(a, b, tw, n, ns, P); break;
      default: stockham_stage<8>(a, b, tw, n, ns, P); break;
    }
    __syncthreads();
    C2* t = a;
    a = b;
    b = t;
    ns *= R;
  }
  return a;
}

template <class C2>
__device__ __forceinline__ void load_twiddles(C2* dst, const void* src, int n) {
  const C2* t = reinterpret_cast<const C2*>(src);
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = t[i];
}

// Reciprocal-space energy and virial of half-spectrum element (x, y, z) with |S|^2 = s2 and
// influence value infl (pme.rs:307-372): the element and its conjugate partner each carry
// half of the virial, elements with 0 < z < nz/2 count twice.
template <class Real>
__device__ __forceinline__ void mode_energy(const PmeArgs<Real>& a, int x, int y, int z, double s2,
                                            double infl, double& e, double (&w)[6]) {
  const double wz = (z == 0 || (a.nz % 2 == 0 && z == a.nz / 2)) ? 1.0 : 2.0;
  e += wz * 0.5 * infl * s2;
  const int idx[2][3] = {{x, y, z}, {(a.nx - x) % a.nx, (a.ny - y) % a.ny, (a.nz - z) % a.nz}};
  for (int p = 0; p < 2; ++p) {
    const double m[3] = {freq(idx[p][0], a.nx), freq(idx[p][1], a.ny), freq(idx[p][2], a.nz)};
    double k[3];
    for (int c = 0; c < 3; ++c) k[c] = m[0] * a.recip[0][c] + m[1] * a.recip[1][c] + m[2] * a.recip[2][c];
    const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    const double bm = a.moduli[idx[p][0]] * a.moduli[a.nx + idx[p][1]] * a.moduli[a.nx + a.ny + idx[p][2]];
    const double pa = kPiD * kPiD / (a.alpha * a.alpha);
    const double g_m = kOne4PiEps0 * exp(-pa * k2) / (kPiD * a.volume * k2 * bm);
    const double em = wz * 0.5 * 0.5 * g_m * s2;
    const double c = 2.0 * (1.0 + pa * k2) / k2;
    w[0] += em * (1.0 - c * k[0] * k[0]);
    w[1] += em * (1.0 - c * k[1] * k[1]);
    w[2] += em * (1.0 - c * k[2] * k[2]);
    w[3] -= em * c * k[0] * k[1];
    w[4] -= em * c * k[0] * k[2];
    w[5] -= em * c * k[1] * k[2];
  }
}

// Warp sums of the energy and virial in fixed point, one atomic per warp and term (every
// thread of the block calls it).
template <class Real>
__device__ __forceinline__ void commit_energy(const PmeArgs<Real>& a, double e, const double (&w)[6]) {
  long long ef = to_fixed(e, kEnergyScale);
  long long wf[6];
  for (int c = 0; c < 6; ++c) wf[c] = to_fixed(w[c], kEnergyScale);
  for (int off = 16; off > 0; off >>= 1) {
    ef += __shfl_xor_sync(0xffffffffu, ef, off);
    for (int c = 0; c < 6; ++c) wf[c] += __shfl_xor_sync(0xffffffffu, wf[c], off);
  }
  if ((threadIdx.x & 31) == 0) {
    add_fixed(a.energy, ef);
    for (int c = 0; c < 6; ++c) add_fixed(a.energy + 1 + c, wf[c]);
  }
}

// Shared memory of a plane kernel: z and y twiddles, two buffers of `plane` elements.
__host__ __device__ inline int fft_plane_elems(int ny, int nz) {
  const int a = (ny + 1) / 2 * nz, b = (nz / 2 + 1) * ny;
  return a > b ? a : b;
}

constexpr int kPlaneThreads = 512, kXPassThreads = 256;  // block size caps of the transform
constexpr int kLoadBatch = 4;  // global loads each thread keeps in flight in the copy loops

// for i in [0, total), strided over the block: v = load(i) for kLoadBatch items at a time,
// then use(i, v) for each, so that the loads of a batch overlap.
template <class T, class Load, class Use>
__device__ __forceinline__ void batched(int total, Load load, Use use) {
  for (int i0 = threadIdx.x; i0 < total; i0 += kLoadBatch * blockDim.x) {
    T v[kLoadBatch];
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < total) v[u] = load(i);
    }
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < total) use(i, v[u]);
    }
  }
}

template <class Real>
__global__ void __launch_bounds__(kPlaneThreads) planes_forward(const PmeArgs<Real> a, const PmeFft f) {
  using C2 = typename Cplx<Real>::T;
  extern __shared__ __align__(16) unsigned char fsm[];
  const int ny = a.ny, nz = a.nz, nzh = nz / 2 + 1, nyp = (ny + 1) / 2, x = blockIdx.x;
  const int pe = fft_plane_elems(ny, nz);
  C2* twz = reinterpret_cast<C2*>(fsm);
  C2* twy = twz + nz;
  C2* A = twy + ny;
  C2* B = A + pe;
  load_twiddles(twz, f.tw[2], nz);
  load_twiddles(twy, f.tw[1], ny);
  // rows y = 2 yp (real part) and 2 yp + 1 (imaginary part) as one complex row
  long long* plane = a.grid_fixed + (long long)x * ny * nz;
  batched<longlong2>(
      nyp * nz,
      [&](int i) {
        const int yp = i / nz, z = i - yp * nz;
        const long long* g0 = plane + (long long)(2 * yp) * nz + z;
        longlong2 r;
        r.x = __ldcg(g0);
        r.y = 2 * yp + 1 < ny ? __ldcg(g0 + nz) : 0;
        return r;
      },
      [&](int i, longlong2 r) {
        C2 v;
        v.x = (Real)((double)r.x * kGridScaleInv);
        v.y = (Real)((double)r.y * kGridScaleInv);
        A[i] = v;
      });
  __syncthreads();
  for (int i = threadIdx.x; i < ny * nz; i += blockDim.x) plane[i] = 0;  // ready for the next spread
  C2* r = stockham(A, B, twz, f, 2, nz, nyp);
  C2* o = r == A ? B : A;
  // split the two real rows' spectra: X_even = (Z_k + conj Z_-k)/2, X_odd = -i (Z_k - conj Z_-k)/2,
  // into pencils along y: o[kz][y]
  for (int i = threadIdx.x; i < nzh * ny; i += blockDim.x) {
    const int kz = i / ny, y = i - kz * ny, yp = y >> 1;
    const C2 zk = r[yp * nz + kz], zm = r[yp * nz + (kz == 0 ? 0 : nz - kz)];
    C2 v;
    if ((y & 1) == 0) {
      v.x = (Real)0.5 * (zk.x + zm.x);
      v.y = (Real)0.5 * (zk.y - zm.y);
    } else {
      v.x = (Real)0.5 * (zk.y + zm.y);
      v.y = (Real)0.5 * (zm.x - zk.x);
    }
    o[i] = v;
  }
  __syncthreads();
  C2* s = stockham(o, r, twy, f, 1, ny, nzh);
  C2* out = reinterpret_cast<C2*>(a.grid_k) + (long long)x * ny * nzh;
  for (int i = threadIdx.x; i < ny * nzh; i += blockDim.x) {
    const int y = i / nzh, kz = i - y * nzh;
    out[i] = s[kz * ny + y];
  }
}

template <class Real, bool kEnergy>
__global__ void __launch_bounds__(kXPassThreads) x_convolve(const PmeArgs<Real> a, const PmeFft f) {
  using C2 = typename Cplx<Real>::T;
  extern __shared__ __align__(16) unsigned char fsm[];
  const int nx = a.nx, nzh = a.nz / 2 + 1, P0 = f.pencils_x;
  const int nkb = (nzh + P0 - 1) / P0;
  const int y = blockIdx.x / nkb, kz0 = (blockIdx.x - y * nkb) * P0, P = min(P0, nzh - kz0);
  C2* tw = reinterpret_cast<C2*>(fsm);
  C2* A = tw + nx;
  C2* B = A + P0 * nx;
  load_twiddles(tw, f.tw[0], nx);
  C2* g = reinterpret_cast<C2*>(a.grid_k);
  const long long sx = (long long)a.ny * nzh, base = (long long)y * nzh + kz0;
  batched<C2>(
      nx * P, [&](int i) { const int x = i / P, p = i - x * P; return __ldcg(g + base + x * sx + p); },
      [&](int i, C2 v) { const int x = i / P, p = i - x * P; A[p * nx + x] = v; });
  __syncthreads();
  C2* r = stockham(A, B, tw, f, 0, nx, P);
  C2* o = r == A ? B : A;
  double e = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  batched<Real>(
      P * nx, [&](int i) { const int p = i / nx, x = i - p * nx; return __ldg(a.influence + base + x * sx + p); },
      [&](int i, Real infl) {
        const int p = i / nx, x = i - p * nx;
        C2 v = r[i];
        if (kEnergy && base + x * sx + p != 0)
          mode_energy(a, x, y, kz0 + p, (double)v.x * v.x + (double)v.y * v.y, (double)infl, e, w);
        v.x *= infl;
        v.y *= -infl;  // conjugated for the inverse transform
        r[i] = v;
      });
  if (kEnergy) commit_energy(a, e, w);
  __syncthreads();
  C2* s = stockham(r, o, tw, f, 0, nx, P);
  for (int i = threadIdx.x; i < nx * P; i += blockDim.x) {
    const int x = i / P, p = i - x * P;
    g[base + x * sx + p] = conjg(s[p * nx + x]);
  }
}

template <class Real>
__global__ void __launch_bounds__(kPlaneThreads) planes_inverse(const PmeArgs<Real> a, const PmeFft f) {
  using C2 = typename Cplx<Real>::T;
  extern __shared__ __align__(16) unsigned char fsm[];
  const int ny = a.ny, nz = a.nz, nzh = nz / 2 + 1, nyp = (ny + 1) / 2, x = blockIdx.x;
  const int pe = fft_plane_elems(ny, nz);
  C2* twz = reinterpret_cast<C2*>(fsm);
  C2* twy = twz + nz;
  C2* A = twy + ny;
  C2* B = A + pe;
  load_twiddles(twz, f.tw[2], nz);
  load_twiddles(twy, f.tw[1], ny);
  const C2* in = reinterpret_cast<const C2*>(a.grid_k) + (long long)x * ny * nzh;
  batched<C2>(
      ny * nzh, [&](int i) { return __ldcg(in + i); },
      [&](int i, C2 v) { const int y = i / nzh, kz = i - y * nzh; A[kz * ny + y] = conjg(v); });
  __syncthreads();
  // r = F(conj H): the inverse y transform of H is conj(r)
  C2* r = stockham(A, B, twy, f, 1, ny, nzh);
  C2* o = r == A ? B : A;
  // rows 2 yp and 2 yp + 1 of the inverse, Hermitian-completed along z, as one row
  // Z = Ha + i Hb, stored conjugated: conj Z = conj Ha - i conj Hb
  for (int i = threadIdx.x; i < nyp * nz; i += blockDim.x) {
    const int yp = i / nz, k = i - yp * nz, y0 = 2 * yp;
    const bool lo = k < nzh;
    const int kk = lo ? k : nz - k;
    C2 ca = r[kk * ny + y0];  // conj Ha[k] for k < nzh
    if (!lo) ca = conjg(ca);
    C2 cb;
    cb.x = cb.y = 0;
    if (y0 + 1 < ny) {
      cb = r[kk * ny + y0 + 1];
      if (!lo) cb = conjg(cb);
    }
    C2 v;
    v.x = ca.x + cb.y;
    v.y = ca.y - cb.x;
    o[i] = v;
  }
  __syncthreads();
  // s = F(conj Z); the inverse is conj(s): row 2 yp = Re s, row 2 yp + 1 = -Im s
  C2* s = stockham(o, r, twz, f, 2, nz, nyp);
  Real* out = a.grid_real + (long long)x * ny * nz;
  for (int i = threadIdx.x; i < ny * nz; i += blockDim.x) {
    const int y = i / nz, z = i - y * nz;
    const C2 v = s[(y >> 1) * nz + z];
    out[i] = (y & 1) ? -v.y : v.x;
  }
}

}  // namespace

template <class Real>
size_t pme_transform_smem(const PmeArgs<Real>& a, const PmeFft& f, int kernel) {
  using C2 = typename Cplx<Real>::T;
  if (kernel == 1) return sizeof(C2) * (size_t)a.nx * (1 + 2 * f.pencils_x);
  return sizeof(C2) * ((size_t)a.ny + a.nz + 2 * (size_t)fft_plane_elems(a.ny, a.nz));
}

template <class Real>
void launch_pme_transform(const PmeArgs<Real>& a, const PmeFft& f, bool energy, cudaStream_t s) {
  const size_t sp = pme_transform_smem(a, f, 0), sx = pme_transform_smem(a, f, 1);
  const int nzh = a.nz / 2 + 1, nkb = ceil_div(nzh, f.pencils_x);
  planes_forward<Real><<<a.nx, f.threads[0], sp, s>>>(a, f);
  if (energy)
    x_convolve<Real, true><<<a.ny * nkb, f.threads[1], sx, s>>>(a, f);
  else
    x_convolve<Real, false><<<a.ny * nkb, f.threads[1], sx, s>>>(a, f);
  planes_inverse<Real><<<a.nx, f.threads[2], sp, s>>>(a, f);
}

template <class Real>
void prepare_pme_transform(const PmeArgs<Real>& a, const PmeFft& f) {
  const int sp = (int)pme_transform_smem(a, f, 0), sx = (int)pme_transform_smem(a, f, 1);
  cudaFuncSetAttribute((const void*)planes_forward<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp);
  cudaFuncSetAttribute((const void*)planes_inverse<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp);
  cudaFuncSetAttribute((const void*)x_convolve<Real, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
  cudaFuncSetAttribute((const void*)x_convolve<Real, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sx);
}

template size_t pme_transform_smem<float>(const PmeArgs<float>&, const PmeFft&, int);
template size_t pme_transform_smem<double>(const PmeArgs<double>&, const PmeFft&, int);
template void launch_pme_transform<float>(const PmeArgs<float>&, const PmeFft&, bool, cudaStream_t);
template void launch_pme_transform<double>(const PmeArgs<double>&, const PmeFft&, bool, cudaStream_t);
template void prepare_pme_transform<float>(const PmeArgs<float>&, const PmeFft&);
template void prepare_pme_transform<double>(const PmeArgs<double>&, const PmeFft&);

namespace {
// pme.rs:332-350: the influence function on the half spectrum, averaged over each mode and its
// conjugate partner, zero at k = 0 (one thread per half-grid point, f64).
template <class Real>
__global__ void influence_kernel(Real* out, const double* moduli, int nx, int ny, int nz,
                                 PmeRecip r, double alpha, double volume) {
  const int nzh = nz / 2 + 1;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny * nzh) return;
  const int z = (int)(i % nzh), y = (int)((i / nzh) % ny), x = (int)(i / ((long long)nzh * ny));
  if (i == 0) {
    out[0] = Real(0);
    return;
  }
  const double pa = kPiD * kPiD / (alpha * alpha);
  auto g = [&](int gx, int gy, int gz) {
    const double m[3] = {freq(gx, nx), freq(gy, ny), freq(gz, nz)};
    double k2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      const double kc = m[0] * r.m[0][c] + m[1] * r.m[1][c] + m[2] * r.m[2][c];
      k2 += kc * kc;
    }
    return kOne4PiEps0 * exp(-pa * k2) /
           (kPiD * volume * k2 * moduli[gx] * moduli[nx + gy] * moduli[nx + ny + gz]);
  };
  out[i] = (Real)(0.5 * (g(x, y, z) + g((nx - x) % nx, (ny - y) % ny, (nz - z) % nz)));
}
}  // namespace

template <class Real>
void launch_pme_influence(Real* out, const double* moduli, int nx, int ny, int nz,
                          const PmeRecip& recip, double alpha, double volume, cudaStream_t s) {
  const long long n = (long long)nx * ny * (nz / 2 + 1);
  influence_kernel<Real><<<(int)((n + 255) / 256), 256, 0, s>>>(out, moduli, nx, ny, nz, recip,
                                                                alpha, volume);
}
template void launch_pme_influence<float>(float*, const double*, int, int, int, const PmeRecip&,
                                          double, double, cudaStream_t);
template void launch_pme_influence<double>(double*, const double*, int, int, int, const PmeRecip&,
                                           double, double, cudaStream_t);

template <class Real>
void launch_pme_spread(const PmeArgs<Real>& a, cudaStream_t s) {
  if (a.order) {  // sorted slots: spatially compact CTAs
    spread_staged_kernel<Real><<<ceil_div(a.n_order, kSpreadAtoms), 2 * kSpreadAtoms, 0, s>>>(a);
  } else {
    spread_kernel<Real><<<ceil_div(a.n_order, 128), 128, 0, s>>>(a);
  }
}
template <class Real>
void launch_pme_convert(const PmeArgs<Real>& a, cudaStream_t s) {
  const long long total = (long long)a.nx * a.ny * a.nz;
  convert_kernel<Real><<<(int)std::min<long long>((total + 255) / 256, 148LL * 16), 256, 0, s>>>(a);
}
template <class Real>
void launch_pme_convolve(const PmeArgs<Real>& a, bool energy, cudaStream_t s) {
  const long long total = (long long)a.nx * a.ny * (a.nz / 2 + 1);
  const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  if (energy)
    convolve_kernel<Real, true><<<grid, 256, 0, s>>>(a, a.moduli);
  else
    convolve_kernel<Real, false><<<grid, 256, 0, s>>>(a, a.moduli);
}
template <class Real>
void launch_pme_gather(const PmeArgs<Real>& a, cudaStream_t s) {
  gather_kernel<Real><<<ceil_div((long long)a.n_order * 8, 128), 128, 0, s>>>(a);
}

template void launch_pme_spread<float>(const PmeArgs<float>&, cudaStream_t);
template void launch_pme_spread<double>(const PmeArgs<double>&, cudaStream_t);
template void launch_pme_convert<float>(const PmeArgs<float>&, cudaStream_t);
template void launch_pme_convert<double>(const PmeArgs<double>&, cudaStream_t);
template void launch_pme_convolve<float>(const PmeArgs<float>&, bool, cudaStream_t);
template void launch_pme_convolve<double>(const PmeArgs<double>&, bool, cudaStream_t);
template void launch_pme_gather<float>(const PmeArgs<float>&, cudaStream_t);
template void launch_pme_gather<double>(const PmeArgs<double>&, cudaStream_t);

// ---- brick-owned gathering --------------------------------------------------------------
// For large grids in rectangular boxes.  A first kernel stores every slot's stencil (base point,
// fractions, charge).  Then one CTA per brick of kBrickEdge^3 grid points reads the brick and
// its 4-point halo of the potential grid into shared memory once, collects its candidates from
// the per-rebuild slot ranges of the x-y columns in reach (one 16-byte stencil load each), and
// takes those whose stencil starts inside the brick, so every particle is gathered by one CTA
// from shared memory instead of by eight lanes from L2.  Each atom's stencil planes are summed
// in the order of the eight-lane kernel, so both forms give the same forces.  (A brick-owned
// spread, storing each brick's sums once, measured slower than the atomic spread on the 196^3
// grid: its shared-memory sums cost more than the global atomics they replace.)
namespace {

constexpr int kBrickThreads = 256;
constexpr int kBrickHalo = (kBrickEdge + 4) * (kBrickEdge + 4) * (kBrickEdge + 4);
constexpr int kBrickOwnChunk = 2048;  // candidates tested before their owners are gathered
static_assert(kBrickMaxRanges <= kBrickThreads, "one range per thread when collecting");

// first slot k in [s0, s0 + n) of a z-sorted column with zkey >= z (s0 + n if none)
__device__ int column_lower(const NlistArgs& a, int s0, int n, float z) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a.zkey[a.sorted_atom[s0 + mid]] < z)
      lo = mid + 1;
    else
      hi = mid;
  }
  return s0 + lo;
}

// One thread per (column, z layer of bricks): the slots of the column's atoms whose wrapped
// rebuild z lies within the layer's reach, as one range or two (the reach wraps the box).
__global__ void brick_ranges_kernel(const NlistArgs a, const PmeBricks b) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_cols * b.nb[2]) return;
  const int c = i % a.n_cols, bz = i / a.n_cols;
  const int s0 = a.col_start[c];
  const int n = min(a.col_scatter[c + 1] - a.col_scatter[c], a.col_max);
  const double L = b.len[2];
  const double z0 = bz * kBrickEdge * b.cell[2] - b.below[2];
  const double z1 = min((bz + 1) * kBrickEdge, b.grid[2]) * b.cell[2] + b.above;
  int2 r0 = make_int2(s0, s0), r1 = make_int2(s0, s0);
  if (z1 - z0 >= L) {
    r0.y = s0 + n;
  } else if (z0 < 0.0) {
    r0 = make_int2(column_lower(a, s0, n, (float)(z0 + L)), s0 + n);
    r1 = make_int2(s0, column_lower(a, s0, n, (float)z1));
  } else if (z1 > L) {
    r0 = make_int2(column_lower(a, s0, n, (float)z0), s0 + n);
    r1 = make_int2(s0, column_lower(a, s0, n, (float)(z1 - L)));
  } else {
    r0 = make_int2(column_lower(a, s0, n, (float)z0), column_lower(a, s0, n, (float)z1));
  }
  b.ranges[2 * i] = r0;
  b.ranges[2 * i + 1] = r1;
}

// first grid point and extent of brick `id` along each axis
__device__ __forceinline__ void brick_box(const PmeBricks& b, int id, int b0[3], int e[3],
                                          int bi[3]) {
  bi[0] = id % b.nb[0];
  bi[1] = (id / b.nb[0]) % b.nb[1];
  bi[2] = id / (b.nb[0] * b.nb[1]);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    b0[d] = bi[d] * kBrickEdge;
    e[d] = min(kBrickEdge, b.grid[d] - b0[d]);
  }
}

// columns along axis d (0: x, 1: y) whose rebuild positions can reach brick index bd
__device__ __forceinline__ void column_span(const PmeBricks& b, int d, int bd, int& c0, int& nc) {
  const int ncol = b.n_col[d];
  const double w = b.len[d] / ncol;
  const double lo = bd * kBrickEdge * b.cell[d] - b.below[d];
  const double hi = min((bd + 1) * kBrickEdge, b.grid[d]) * b.cell[d] + b.above;
  c0 = (int)floor(lo / w);
  nc = (int)floor(hi / w) - c0 + 1;
  if (nc >= ncol) {
    c0 = 0;
    nc = ncol;
  }
}

// The brick's candidate slot ranges into s_rng, their exclusive prefix into s_pre; returns the
// number of ranges (the candidate count is s_pre[ranges]).  Block-wide, with barriers.
__device__ int brick_candidates(const PmeBricks& b, const NlistArgs& nl, const int bi[3],
                                int2* s_rng, int* s_pre, int* s_warp) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int cx0, ncx, cy0, ncy;
  column_span(b, 0, bi[0], cx0, ncx);
  column_span(b, 1, bi[1], cy0, ncy);
  const int nr = min(2 * ncx * ncy, kBrickMaxRanges);  // the host keeps 2 ncx ncy within
  int len = 0;
  if (t < nr) {
    const int k = t >> 1, piece = t & 1;
    int cx = (cx0 + k % ncx) % b.n_col[0];
    int cy = (cy0 + k / ncx) % b.n_col[1];
    cx += cx < 0 ? b.n_col[0] : 0;
    cy += cy < 0 ? b.n_col[1] : 0;
    const int col = cy * b.n_col[0] + cx;
    const int2 r = b.ranges[2 * ((size_t)bi[2] * nl.n_cols + col) + piece];
    s_rng[t] = r;
    len = max(r.y - r.x, 0);
  }
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    int v = lane < kBrickThreads / 32 ? s_warp[lane] : 0, x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane < kBrickThreads / 32) s_warp[lane] = x - v;  // exclusive warp offsets
  }
  __syncthreads();
  const int excl = incl - len + s_warp[w];
  if (t < nr) s_pre[t] = excl;
  if (t == nr - 1) s_pre[nr] = excl + len;
  __syncthreads();
  return nr;
}

// slot of candidate i: the last range whose prefix does not exceed i holds it
__device__ __forceinline__ int candidate_slot(const int2* s_rng, const int* s_pre, int nr, int i) {
  int lo = 0, hi = nr - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s_pre[mid] <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return s_rng[lo].x + (i - s_pre[lo]);
}

template <class Real>
struct Real4Of;
template <>
struct Real4Of<float> {
  using T = float4;
};
template <>
struct Real4Of<double> {
  using T = double4;
};

// This step's stencil of every sorted slot (the spread and the gather of the brick form read it
// once per candidate instead of recomputing it from the position): base point per axis and the
// fractions, as `stencil` gives them, and the charge as Real.
template <class Real>
__global__ void brick_stencils_kernel(const PmeArgs<Real> a, const PmeBricks b, const NlistArgs nl) {
  using R4 = typename Real4Of<Real>::T;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.n_slots) return;
  const int atom = nl.sorted_atom[s];
  const double qd = atom >= 0 ? a.charge[atom] : 0.0;
  int base[3] = {0, 0, 0};
  Real frac[3] = {Real(0), Real(0), Real(0)};
  const bool ok = qd != 0.0 && stencil(a, atom, base, frac);
  b.base[s] = make_int4(base[0], base[1], base[2], ok ? 1 : 0);
  R4 f;
  f.x = frac[0];
  f.y = frac[1];
  f.z = frac[2];
  f.w = (Real)qd;
  reinterpret_cast<R4*>(b.frac)[s] = f;
}

template <class Real>
__global__ void __launch_bounds__(kBrickThreads) gather_bricks_kernel(const PmeArgs<Real> a,
                                                                      const PmeBricks b,
                                                                      const NlistArgs nl) {
  using R4 = typename Real4Of<Real>::T;
  extern __shared__ __align__(16) unsigned char brick_smem[];
  Real* phi = reinterpret_cast<Real*>(brick_smem);  // [(e0 + 4)(e1 + 4)(e2 + 4)]
  __shared__ int2 s_rng[kBrickMaxRanges];
  __shared__ int s_pre[kBrickMaxRanges + 1];
  __shared__ int s_warp[kBrickThreads / 32];
  __shared__ int s_own[kBrickOwnChunk];
  __shared__ int s_nown;
  int b0[3], e[3], bi[3];
  brick_box(b, blockIdx.x, b0, e, bi);
  const int h1 = e[1] + 4, h2 = e[2] + 4, nh = (e[0] + 4) * h1 * h2;
  for (int c = threadIdx.x; c < nh; c += kBrickThreads) {
    const int hz = c % h2, hy = (c / h2) % h1, hx = c / (h1 * h2);
    int gx = b0[0] + hx, gy = b0[1] + hy, gz = b0[2] + hz;
    gx -= gx >= a.nx ? a.nx : 0;
    gy -= gy >= a.ny ? a.ny : 0;
    gz -= gz >= a.nz ? a.nz : 0;
    phi[c] = a.grid_real[((long long)gx * a.ny + gy) * a.nz + gz];
  }
  const int nr = brick_candidates(b, nl, bi, s_rng, s_pre, s_warp);  // barriers cover phi
  const int n_cand = s_pre[nr];
  // The candidates are tested in chunks; the owners (stencil starting in this brick, about a
  // third) are listed in shared memory and then gathered one per thread, so that the 125-point
  // sums run on full warps.  The order of the list does not matter: each particle's force is
  // its own sum, added in fixed point.
  for (int i0 = 0; i0 < n_cand; i0 += kBrickOwnChunk) {
    if (threadIdx.x == 0) s_nown = 0;
    __syncthreads();
    const int i1 = min(i0 + kBrickOwnChunk, n_cand);
    for (int i = i0 + threadIdx.x; i < i1; i += kBrickThreads) {
      const int slot = candidate_slot(s_rng, s_pre, nr, i);
      const int4 sb = b.base[slot];
      const bool own = sb.w && (unsigned)(sb.x - b0[0]) < (unsigned)e[0] &&
                       (unsigned)(sb.y - b0[1]) < (unsigned)e[1] &&
                       (unsigned)(sb.z - b0[2]) < (unsigned)e[2];
      const unsigned m = __ballot_sync(__activemask(), own);
      if (own) {
        const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
        int at = 0;
        if (lane == leader) at = atomicAdd(&s_nown, __popc(m));
        at = __shfl_sync(m, at, leader) + __popc(m & ((1u << lane) - 1u));
        s_own[at] = slot;
      }
    }
    __syncthreads();
    const int n_own = s_nown;
    for (int o = threadIdx.x; o < n_own; o += kBrickThreads) {
    const int slot = s_own[o];
    const int4 sb = b.base[slot];
    const int lx = sb.x - b0[0], ly = sb.y - b0[1], lz = sb.z - b0[2];
    const R4 sf = reinterpret_cast<const R4*>(b.frac)[slot];
    const int atom = nl.sorted_atom[slot];
    const double qd = a.charge[atom];
    Real w[3][5], dw[3][5];
    spline5(sf.x, w[0], dw[0]);
    spline5(sf.y, w[1], dw[1]);
    spline5(sf.z, w[2], dw[2]);
    Real p0[5], p1[5], p2[5];  // stencil plane ix: the sums of lane ix of the eight-lane kernel
#pragma unroll
    for (int ix = 0; ix < 5; ++ix) {
      Real g0 = 0, g1 = 0, g2 = 0;
      const Real wx = w[0][ix], dwx = dw[0][ix];
      for (int iy = 0; iy < 5; ++iy) {
        const Real* row = phi + ((lx + ix) * h1 + (ly + iy)) * h2 + lz;
        const Real wxy = wx * w[1][iy];
        const Real dxy = dwx * w[1][iy];
        const Real xdy = wx * dw[1][iy];
#pragma unroll
        for (int iz = 0; iz < 5; ++iz) {
          const Real ph = row[iz];
          g0 += ph * dxy * w[2][iz];
          g1 += ph * xdy * w[2][iz];
          g2 += ph * wxy * dw[2][iz];
        }
      }
      p0[ix] = g0;
      p1[ix] = g1;
      p2[ix] = g2;
    }
    // the eight-lane kernel's xor tree (lanes 5-7 hold zeros)
    const Real g0 = ((p0[0] + p0[4]) + p0[2]) + (p0[1] + p0[3]);
    const Real g1 = ((p1[0] + p1[4]) + p1[2]) + (p1[1] + p1[3]);
    const Real g2 = ((p2[0] + p2[4]) + p2[2]) + (p2[1] + p2[3]);
    const double gd[3] = {(double)g0 * a.nx, (double)g1 * a.ny, (double)g2 * a.nz};
    for (int c = 0; c < 3; ++c) {
      const double f = -qd * (gd[0] * a.recip[0][c] + gd[1] * a.recip[1][c] + gd[2] * a.recip[2][c]);
      add_fixed(a.force + (long long)c * a.n_atoms + atom, to_fixed(f, kForceScale));
    }
    }
    __syncthreads();  // the list is refilled by the next chunk
  }
}

}  // namespace

void launch_pme_brick_ranges(const NlistArgs& a, const PmeBricks& b, cudaStream_t s) {
  const int n = a.n_cols * b.nb[2];
  brick_ranges_kernel<<<ceil_div(n, 128), 128, 0, s>>>(a, b);
}

template <class Real>
void launch_pme_brick_stencils(const PmeArgs<Real>& a, const PmeBricks& b, const NlistArgs& nl,
                               cudaStream_t s) {
  brick_stencils_kernel<Real><<<ceil_div(b.n_slots, 256), 256, 0, s>>>(a, b, nl);
}
template void launch_pme_brick_stencils<float>(const PmeArgs<float>&, const PmeBricks&,
                                               const NlistArgs&, cudaStream_t);
template void launch_pme_brick_stencils<double>(const PmeArgs<double>&, const PmeBricks&,
                                                const NlistArgs&, cudaStream_t);

template <class Real>
void launch_pme_gather_bricks(const PmeArgs<Real>& a, const PmeBricks& b, const NlistArgs& nl,
                              cudaStream_t s) {
  const int bytes = (int)(sizeof(Real) * kBrickHalo);  // the FP64 halo exceeds 48 KB with the rest
  cudaFuncSetAttribute(gather_bricks_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       bytes);
  gather_bricks_kernel<Real><<<b.nb[0] * b.nb[1] * b.nb[2], kBrickThreads, bytes, s>>>(a, b, nl);
}

template void launch_pme_gather_bricks<float>(const PmeArgs<float>&, const PmeBricks&,
                                              const NlistArgs&, cudaStream_t);
template void launch_pme_gather_bricks<double>(const PmeArgs<double>&, const PmeBricks&,
                                               const NlistArgs&, cudaStream_t);

}  // namespace ommb200
