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
// accumulation uses native 32-bit atomics on a split of each 64-bit fixed-point value,
// v = hi 2^20 + lo with 0 <= lo < 2^20: at most 64 contributions per cell keep both partial
// sums inside 32 bits (for |q| < 16 e), and hi_sum 2^20 + lo_sum recovers the exact 64-bit
// total, so the integer grid is identical to direct spreading.  A CTA whose box exceeds
// kSpreadCells (it straddles a periodic edge of the column order) or that holds a larger
// charge spreads directly.
constexpr int kSpreadAtoms = 64;
constexpr int kSpreadCells = 4096;

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
    if (fabs(qd) >= 16.0) s_big = 1;  // the 32-bit partial sums need |q| < 16 e
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
    c_lo[c] = 0u;
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
          const long long v = to_fixed(qxy * w[2][iz], gscale);
          atomicAdd(&c_hi[row + iz], (int)(v >> 20));
          atomicAdd(&c_lo[row + iz], (unsigned int)(v & 0xFFFFF));
        }
      }
    }
  }
  __syncthreads();
  for (int c = tid; c < nc; c += 2 * kSpreadAtoms) {
    const long long v = (long long)c_hi[c] * (1ll << 20) + (long long)c_lo[c];
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

}  // namespace

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

}  // namespace ommb200
