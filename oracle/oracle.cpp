// f64 CPU oracle for the openmm-rs hot path.  TEST INFRASTRUCTURE ONLY: loaded by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline arm, never by the product.
//
// Every routine restates the reference algorithm (crates/openmm-core/src/..., cited per
// function) in plain double precision, in the reference's own summation order when run with
// one thread, so that it can stand in for the reference (which cannot be compiled here: no
// Rust toolchain).  Build with -ffp-contract=off so products and sums round as in Rust.
//
// Parity pinning: no golden vectors exist for this path; the oracle is pinned by the
// reference's analytic known-answer and finite-difference tests (tests/test_oracle.py) and
// PME is checked against the direct Ewald sum below.
#include "oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <set>
#include <array>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;
// nonbonded.rs:16
constexpr double ONE_4PI_EPS0 = 138.93545764438198;
// integrators/langevin.rs:13
const double BOLTZMANN = 1.380649e-23 * 6.02214076e23 / 1000.0;
// gbsa_obc.rs:8-9
constexpr double DIELECTRIC_OFFSET = 0.009;
constexpr double PROBE_RADIUS = 0.14;

// harmonic_bond.rs:152-159: reduced-triclinic minimum image, delta = r_j - r_i.
inline void min_image(double d[3], const double* bv) {
  for (int k = 2; k >= 0; --k) {
    double shift = std::floor(d[k] / bv[3 * k + k] + 0.5);
    for (int a = 0; a <= k; ++a) d[a] -= shift * bv[3 * k + a];
  }
}

// pme.rs:176-199
void reciprocal_box(const double* bv, double recip[3][3], double* volume) {
  auto cross = [](const double* a, const double* b, double* out) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
  };
  const double* a = bv;
  const double* b = bv + 3;
  const double* c = bv + 6;
  double bc[3], ca[3], ab[3];
  cross(b, c, bc);
  cross(c, a, ca);
  cross(a, b, ab);
  double v = 0.0;
  for (int i = 0; i < 3; ++i) v += a[i] * bc[i];
  for (int i = 0; i < 3; ++i) {
    recip[0][i] = bc[i] / v;
    recip[1][i] = ca[i] / v;
    recip[2][i] = ab[i] / v;
  }
  *volume = v;
}

// ---------------------------------------------------------------------------------------
// Cell list: neighbors.rs:23-181.  visit() calls pair(i, j) for candidate pairs with j > i in
// the reference's order (cell heads hold the last inserted atom, offsets dx,dy,dz nested).
// ---------------------------------------------------------------------------------------
struct Geometry {
  long long dims[3];
  double origin[3];
  bool periodic;
  double recip[3][3];
  double inverse_cutoff;

  Geometry(int n, const double* pos, double cutoff, const double* box) {
    inverse_cutoff = 1.0 / cutoff;
    if (box) {
      periodic = true;
      double vol;
      reciprocal_box(box, recip, &vol);
      for (int a = 0; a < 3; ++a) {
        double norm = std::sqrt(recip[a][0] * recip[a][0] + recip[a][1] * recip[a][1] +
                                recip[a][2] * recip[a][2]);
        double d = std::floor(1.0 / (cutoff * norm));
        d = std::min(std::max(d, 1.0), 1e9);
        dims[a] = (long long)d;
        origin[a] = 0.0;
      }
    } else {
      periodic = false;
      double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
          mn[a] = std::min(mn[a], pos[3 * i + a]);
          mx[a] = std::max(mx[a], pos[3 * i + a]);
        }
      for (int a = 0; a < 3; ++a) {
        dims[a] = (long long)std::floor((mx[a] - mn[a]) * inverse_cutoff) + 1;
        origin[a] = mn[a];
      }
    }
  }
  std::array<long long, 3> key(const double* p) const {
    std::array<long long, 3> k;
    for (int a = 0; a < 3; ++a) {
      if (periodic) {
        double f = 0.0;
        for (int d = 0; d < 3; ++d) f += p[d] * recip[a][d];
        long long c = (long long)std::floor((f - std::floor(f)) * (double)dims[a]);
        k[a] = std::min(c, dims[a] - 1);
      } else {
        k[a] = (long long)std::floor((p[a] - origin[a]) * inverse_cutoff);
      }
    }
    return k;
  }
  int n_offsets(int axis, long long* out) const {
    if (periodic && dims[axis] == 1) {
      out[0] = 0;
      return 1;
    }
    if (periodic && dims[axis] == 2) {
      out[0] = 0;
      out[1] = 1;
      return 2;
    }
    out[0] = -1;
    out[1] = 0;
    out[2] = 1;
    return 3;
  }
};

template <class F>
void visit_cells(int n, const double* pos, double cutoff, const double* box, F&& pair) {
  if (n < 2) return;
  Geometry g(n, pos, cutoff, box);
  long long full_span = box ? 3 : 2;
  if (g.dims[0] <= full_span && g.dims[1] <= full_span && g.dims[2] <= full_span) {
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) pair(i, j);
    return;
  }
  const uint32_t EMPTY = 0xffffffffu;
  std::vector<uint32_t> next(n, EMPTY);
  std::map<std::array<long long, 3>, uint32_t> heads;  // order-independent lookup
  std::vector<std::array<long long, 3>> keys(n);
  for (int i = 0; i < n; ++i) {
    keys[i] = g.key(pos + 3 * i);
    auto it = heads.find(keys[i]);
    uint32_t prev = EMPTY;
    if (it != heads.end()) {
      prev = it->second;
      it->second = (uint32_t)i;
    } else {
      heads.emplace(keys[i], (uint32_t)i);
    }
    next[i] = prev;
  }
  long long off[3][3];
  int noff[3];
  for (int a = 0; a < 3; ++a) noff[a] = g.n_offsets(a, off[a]);
  for (int i = 0; i < n; ++i) {
    const auto& c = keys[i];
    for (int ix = 0; ix < noff[0]; ++ix)
      for (int iy = 0; iy < noff[1]; ++iy)
        for (int iz = 0; iz < noff[2]; ++iz) {
          std::array<long long, 3> k = {c[0] + off[0][ix], c[1] + off[1][iy], c[2] + off[2][iz]};
          if (g.periodic) {
            for (int a = 0; a < 3; ++a) {
              long long m = k[a] % g.dims[a];
              if (m < 0) m += g.dims[a];
              k[a] = m;
            }
          } else {
            bool out = false;
            for (int a = 0; a < 3; ++a) out |= (k[a] < 0 || k[a] >= g.dims[a]);
            if (out) continue;
          }
          auto it = heads.find(k);
          uint32_t j = it == heads.end() ? EMPTY : it->second;
          while (j != EMPTY) {
            if ((int)j > i) pair(i, (int)j);
            j = next[j];
          }
        }
  }
}

// ---------------------------------------------------------------------------------------
// Pair kernels: nonbonded.rs:1194-1288.  All return (E, dE/dr / r).
// ---------------------------------------------------------------------------------------
inline void lj_pair(double sigma, double epsilon, double r2, double* e, double* f) {
  if (epsilon == 0.0) {
    *e = 0.0;
    *f = 0.0;
    return;
  }
  double sr2 = (sigma * sigma) / r2;
  double sr6 = sr2 * sr2 * sr2;
  double sr12 = sr6 * sr6;
  *e = 4.0 * epsilon * (sr12 - sr6);
  *f = 4.0 * epsilon * (-12.0 * sr12 + 6.0 * sr6) / r2;
}
inline void coulomb_pair(double qq, double r, double r2, double* e, double* f) {
  if (qq == 0.0) {
    *e = 0.0;
    *f = 0.0;
    return;
  }
  *e = ONE_4PI_EPS0 * qq / r;
  *f = -ONE_4PI_EPS0 * qq / (r2 * r);
}
inline void reaction_field(double qq, double r, double r2, double rc, double eps_rf, double* e,
                           double* f) {
  if (qq == 0.0) {
    *e = 0.0;
    *f = 0.0;
    return;
  }
  double rc3 = rc * rc * rc, krf, crf;
  if (std::isinf(eps_rf)) {
    krf = 0.5 / rc3;
    crf = 1.5 / rc;
  } else {
    krf = (eps_rf - 1.0) / (2.0 * eps_rf + 1.0) / rc3;
    crf = (3.0 * eps_rf) / (2.0 * eps_rf + 1.0) / rc;
  }
  *e = ONE_4PI_EPS0 * qq * (1.0 / r + krf * r2 - crf);
  *f = ONE_4PI_EPS0 * qq * (-1.0 / (r2 * r) + 2.0 * krf);
}
inline void screened_coulomb(double qq, double r, double r2, double alpha, double* e,
                             double* f) {
  if (qq == 0.0) {
    *e = 0.0;
    *f = 0.0;
    return;
  }
  double erfc_v = std::erfc(alpha * r);
  double coefficient = ONE_4PI_EPS0 * qq;
  *e = coefficient * erfc_v / r;
  *f = -coefficient * (erfc_v / r + 2.0 * alpha / std::sqrt(kPi) * std::exp(-alpha * alpha * r2)) /
       r2;
}
inline void reciprocal_pair(double qq, double r, double r2, double alpha, double* e, double* f) {
  double coefficient = ONE_4PI_EPS0 * qq;
  if (alpha * r < 1e-6) {
    *e = coefficient * 2.0 * alpha / std::sqrt(kPi) * (1.0 - alpha * alpha * r2 / 3.0);
    *f = -coefficient * 4.0 * alpha * alpha * alpha / (3.0 * std::sqrt(kPi));
    return;
  }
  double erf_v = std::erf(alpha * r);
  *e = coefficient * erf_v / r;
  *f = coefficient * (2.0 * alpha / std::sqrt(kPi) * std::exp(-alpha * alpha * r2) - erf_v / r) /
       r2;
}

// nonbonded.rs:1290-1336: adaptive Simpson quadrature.
template <class F>
double simpson_recurse(const F& f, double a, double b, double fa, double fm, double fb,
                       double estimate, double tol, int depth) {
  double m = 0.5 * (a + b);
  double fl = f(0.5 * (a + m));
  double fr = f(0.5 * (m + b));
  double left = (m - a) / 6.0 * (fa + 4.0 * fl + fm);
  double right = (b - m) / 6.0 * (fm + 4.0 * fr + fb);
  double diff = left + right - estimate;
  if (depth == 0 || std::fabs(diff) <= 15.0 * tol) return left + right + diff / 15.0;
  return simpson_recurse(f, a, m, fa, fl, fm, left, 0.5 * tol, depth - 1) +
         simpson_recurse(f, m, b, fm, fr, fb, right, 0.5 * tol, depth - 1);
}
template <class F>
double integrate(const F& f, double a, double b) {
  double fa = f(a), fm = f(0.5 * (a + b)), fb = f(b);
  double est = (b - a) / 6.0 * (fa + 4.0 * fm + fb);
  return simpson_recurse(f, a, b, fa, fm, fb, est, 1e-11 * std::max(std::fabs(est), 1e-12), 20);
}

// ---------------------------------------------------------------------------------------
// Mixed-radix complex FFT (stands in for rustfft 6.4.1, pme.rs:230-238, 271-303).  Forward
// uses exp(-2 pi i jk/n), inverse exp(+2 pi i jk/n), both unnormalized, as rustfft does.
// ---------------------------------------------------------------------------------------
struct Fft1d {
  int n;
  std::vector<int> factors;
  std::vector<cplx> tw_fwd, tw_inv;
  explicit Fft1d(int n_) : n(n_) {
    int m = n;
    for (int p = 2; p * p <= m; ++p)
      while (m % p == 0) {
        factors.push_back(p);
        m /= p;
      }
    if (m > 1) factors.push_back(m);
    tw_fwd.resize(n);
    tw_inv.resize(n);
    for (int t = 0; t < n; ++t) {
      double ang = 2.0 * kPi * (double)t / (double)n;
      tw_fwd[t] = cplx(std::cos(ang), -std::sin(ang));
      tw_inv[t] = cplx(std::cos(ang), std::sin(ang));
    }
  }
  void run(cplx* data, bool inverse, std::vector<cplx>& buf) const {
    buf.assign(data, data + n);
    rec_safe(buf.data(), 1, data, n, 0, inverse ? tw_inv : tw_fwd);
  }
  void rec_safe(const cplx* in, int stride, cplx* out, int len, int level,
                const std::vector<cplx>& tw) const {
    if (len == 1) {
      out[0] = in[0];
      return;
    }
    int p = factors[level];
    int m = len / p;
    for (int r = 0; r < p; ++r) rec_safe(in + r * stride, stride * p, out + r * m, m, level + 1, tw);
    int twstep = n / len;
    std::vector<cplx> res(len);
    for (int k = 0; k < m; ++k)
      for (int q = 0; q < p; ++q) {
        cplx acc = 0.0;
        for (int r = 0; r < p; ++r) {
          long long t = ((long long)r * (k + (long long)q * m)) % len;
          acc += out[r * m + k] * tw[(size_t)(t * twstep)];
        }
        res[q * m + k] = acc;
      }
    for (int i = 0; i < len; ++i) out[i] = res[i];
  }
};

// pme.rs:151-174: order-5 cardinal B-spline weights and derivatives.
void spline5(double fraction, double w[5], double dw[5]) {
  for (int i = 0; i < 5; ++i) {
    w[i] = 0.0;
    dw[i] = 0.0;
  }
  w[0] = 1.0 - fraction;
  w[1] = fraction;
  for (int order = 3; order <= 5; ++order) {
    if (order == 5) {
      dw[0] = -w[0];
      for (int i = 1; i < 5; ++i) dw[i] = w[i - 1] - w[i];
    }
    double den = (double)(order - 1);
    w[order - 1] = fraction * w[order - 2] / den;
    for (int i = order - 2; i >= 1; --i)
      w[i] = ((fraction + (double)(order - 1 - i)) * w[i - 1] + ((double)(i + 1) - fraction) * w[i]) /
             den;
    w[0] *= (1.0 - fraction) / den;
  }
}

// pme.rs:201-218
void stencil(const double* p, const double recip[3][3], const int dims[3], int idx[3],
             double w[3][5], double dw[3][5]) {
  for (int a = 0; a < 3; ++a) {
    double f = 0.0;
    for (int j = 0; j < 3; ++j) f += p[j] * recip[a][j];
    double coord = (f - std::floor(f)) * (double)dims[a];
    idx[a] = (int)((size_t)std::floor(coord) % (size_t)dims[a]);
    spline5(coord - std::floor(coord), w[a], dw[a]);
  }
}

// pme.rs:240-259: |b(k)|^2 moduli with the < 1e-7 fix-up.
std::vector<double> bspline_moduli(int n) {
  double w[5], dw[5];
  spline5(0.0, w, dw);
  std::vector<double> v(n);
  for (int k = 0; k < n; ++k) {
    cplx s = 0.0;
    for (int i = 0; i < 5; ++i) s += std::polar(w[i], 2.0 * kPi * (double)k * (double)i / (double)n);
    v[k] = std::norm(s);
  }
  for (int k = 0; k < n; ++k)
    if (v[k] < 1e-7) v[k] = 0.5 * (v[(k + n - 1) % n] + v[(k + 1) % n]);
  return v;
}

// pme.rs:271-303: z rows, then y lines, then x lines.
void transform3d(std::vector<cplx>& grid, const int dims[3], bool inverse) {
  const int nx = dims[0], ny = dims[1], nz = dims[2];
  Fft1d fx(nx), fy(ny), fz(nz);
#pragma omp parallel
  {
    std::vector<cplx> buf, line(std::max(nx, std::max(ny, nz)));
#pragma omp for
    for (int r = 0; r < nx * ny; ++r) fz.run(&grid[(size_t)r * nz], inverse, buf);
#pragma omp for
    for (int xz = 0; xz < nx * nz; ++xz) {
      int x = xz / nz, z = xz % nz;
      for (int y = 0; y < ny; ++y) line[y] = grid[((size_t)x * ny + y) * nz + z];
      fy.run(line.data(), inverse, buf);
      for (int y = 0; y < ny; ++y) grid[((size_t)x * ny + y) * nz + z] = line[y];
    }
#pragma omp for
    for (int yz = 0; yz < ny * nz; ++yz) {
      int y = yz / nz, z = yz % nz;
      for (int x = 0; x < nx; ++x) line[x] = grid[((size_t)x * ny + y) * nz + z];
      fx.run(line.data(), inverse, buf);
      for (int x = 0; x < nx; ++x) grid[((size_t)x * ny + y) * nz + z] = line[x];
    }
  }
}

double pme_reciprocal(int n, const double* pos, const double* q, const double* box, double alpha,
                      const int dims[3], double* forces, double* virial) {
  double recip[3][3], volume;
  reciprocal_box(box, recip, &volume);
  const int nx = dims[0], ny = dims[1], nz = dims[2];
  std::vector<cplx> grid((size_t)nx * ny * nz, cplx(0.0, 0.0));
  // pme.rs:315-330 spread
  for (int i = 0; i < n; ++i) {
    if (q[i] == 0.0) continue;
    int idx[3];
    double w[3][5], dw[3][5];
    stencil(pos + 3 * i, recip, dims, idx, w, dw);
    for (int ix = 0; ix < 5; ++ix)
      for (int iy = 0; iy < 5; ++iy)
        for (int iz = 0; iz < 5; ++iz) {
          size_t index = (((size_t)(idx[0] + ix) % nx) * ny + (size_t)(idx[1] + iy) % ny) * nz +
                         (size_t)(idx[2] + iz) % nz;
          grid[index] += q[i] * w[0][ix] * w[1][iy] * w[2][iz];
        }
  }
  transform3d(grid, dims, false);
  std::vector<double> mod[3] = {bspline_moduli(nx), bspline_moduli(ny), bspline_moduli(nz)};
  auto freq = [](int k, int n) { return k < (n + 1) / 2 ? (double)k : (double)k - (double)n; };
  // pme.rs:340-372 influence function and energy
  double energy = 0.0;
  double vir[6] = {0, 0, 0, 0, 0, 0};
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        size_t index = ((size_t)x * ny + y) * nz + z;
        if (index == 0) {
          grid[index] = 0.0;
          continue;
        }
        double modes[3] = {freq(x, nx), freq(y, ny), freq(z, nz)};
        double kv[3];
        double k2 = 0.0;
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int d = 0; d < 3; ++d) s += modes[d] * recip[d][a];
          kv[a] = s;
          k2 += s * s;
        }
        double moduli = mod[0][x] * mod[1][y] * mod[2][z];
        double influence =
            ONE_4PI_EPS0 * std::exp(-kPi * kPi * k2 / (alpha * alpha)) / (kPi * volume * k2 * moduli);
        double e = 0.5 * influence * std::norm(grid[index]);
        energy += e;
        if (virial) {
          double c = 2.0 * (1.0 + kPi * kPi * k2 / (alpha * alpha)) / k2;
          vir[0] += e * (1.0 - c * kv[0] * kv[0]);
          vir[1] += e * (1.0 - c * kv[1] * kv[1]);
          vir[2] += e * (1.0 - c * kv[2] * kv[2]);
          vir[3] += e * (-c * kv[0] * kv[1]);
          vir[4] += e * (-c * kv[0] * kv[2]);
          vir[5] += e * (-c * kv[1] * kv[2]);
        }
        grid[index] *= influence;
      }
  transform3d(grid, dims, true);
  // pme.rs:377-425 gather
#pragma omp parallel for
  for (int i = 0; i < n; ++i) {
    if (q[i] == 0.0) continue;
    int idx[3];
    double w[3][5], dw[3][5];
    stencil(pos + 3 * i, recip, dims, idx, w, dw);
    double g[3] = {0, 0, 0};
    for (int ix = 0; ix < 5; ++ix)
      for (int iy = 0; iy < 5; ++iy)
        for (int iz = 0; iz < 5; ++iz) {
          size_t index = (((size_t)(idx[0] + ix) % nx) * ny + (size_t)(idx[1] + iy) % ny) * nz +
                         (size_t)(idx[2] + iz) % nz;
          double phi = grid[index].real();
          g[0] += phi * dw[0][ix] * w[1][iy] * w[2][iz];
          g[1] += phi * w[0][ix] * dw[1][iy] * w[2][iz];
          g[2] += phi * w[0][ix] * w[1][iy] * dw[2][iz];
        }
    for (int a = 0; a < 3; ++a) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) s += g[d] * (double)dims[d] * recip[d][a];
      forces[3 * i + a] -= q[i] * s;
    }
  }
  if (virial) {
    virial[0] += vir[0];
    virial[4] += vir[1];
    virial[8] += vir[2];
    virial[1] += vir[3];
    virial[3] += vir[3];
    virial[2] += vir[4];
    virial[6] += vir[4];
    virial[5] += vir[5];
    virial[7] += vir[5];
  }
  return energy;
}

inline void add_pair_virial(double* vir, double f_over_r, const double d[3]) {
  // W_ab = -sum f_over_r d_a d_b  (W = -dU/d strain, atomic scaling)
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) vir[3 * a + b] -= f_over_r * d[a] * d[b];
}

inline int64_t key_of(int i, int j) { return ((int64_t)std::min(i, j) << 32) | (int64_t)std::max(i, j); }

}  // namespace

extern "C" {

void orc_pme_parameters(double cutoff, double tolerance, const double box[9], double* alpha,
                        int dims[3]) {
  // nonbonded.rs:647-658
  double a = std::sqrt(-std::log(2.0 * tolerance)) / cutoff;
  *alpha = a;
  for (int axis = 0; axis < 3; ++axis) {
    double d = std::ceil(2.0 * a * box[3 * axis + axis] / (3.0 * std::pow(tolerance, 0.2)));
    dims[axis] = (int)std::max(d, 6.0);
  }
}

double orc_dispersion_coefficient(int n, const double* sigma, const double* epsilon,
                                  double cutoff, int use_switching, double switching_distance) {
  // nonbonded.rs:660-719 (without parameter offsets)
  double moments[13] = {0}, diagonal[13] = {0};
  for (int i = 0; i < n; ++i) {
    double power = 1.0;
    for (int k = 0; k <= 12; ++k) {
      moments[k] += std::sqrt(epsilon[i]) * power;
      diagonal[k] += epsilon[i] * power;
      power *= sigma[i];
    }
  }
  auto pair_moment = [&](int power) {
    double coefficient = 1.0, sum = 0.0;
    for (int k = 0; k <= power; ++k) {
      sum += coefficient * moments[k] * moments[power - k];
      coefficient *= (double)(power - k) / (double)(k + 1);
    }
    return sum / std::pow(2.0, power) + diagonal[power];
  };
  auto integral = [&](int power) {
    double tail = std::pow(cutoff, 3 - power) / (double)(power - 3);
    if (!use_switching) return tail;
    auto f = [&](double r) {
      double t = (r - switching_distance) / (cutoff - switching_distance);
      return t * t * t * (10.0 + t * (-15.0 + 6.0 * t)) * std::pow(r, 2 - power);
    };
    return tail + integrate(f, switching_distance, cutoff);
  };
  double nn = (double)n;
  return 8.0 * kPi * nn / (nn + 1.0) * (pair_moment(12) * integral(12) - pair_moment(6) * integral(6));
}

double orc_pme_reciprocal(int n, const double* pos, const double* charge, const double box[9],
                          double alpha, const int dims[3], double* forces, double* virial) {
  return pme_reciprocal(n, pos, charge, box, alpha, dims, forces, virial);
}

double orc_ewald_reciprocal(int n, const double* pos, const double* q, const double box[9],
                            double alpha, int kmax, double* forces) {
  double recip[3][3], volume;
  reciprocal_box(box, recip, &volume);
  double energy = 0.0;
  std::vector<double> fx(3 * (size_t)n, 0.0);
  for (int mx = -kmax; mx <= kmax; ++mx)
    for (int my = -kmax; my <= kmax; ++my)
      for (int mz = -kmax; mz <= kmax; ++mz) {
        if (mx == 0 && my == 0 && mz == 0) continue;
        double k[3];
        for (int a = 0; a < 3; ++a) k[a] = mx * recip[0][a] + my * recip[1][a] + mz * recip[2][a];
        double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        double c = std::exp(-kPi * kPi * k2 / (alpha * alpha)) / k2;
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
          double th = 2.0 * kPi * (k[0] * pos[3 * j] + k[1] * pos[3 * j + 1] + k[2] * pos[3 * j + 2]);
          sr += q[j] * std::cos(th);
          si += q[j] * std::sin(th);
        }
        double pref = ONE_4PI_EPS0 / (2.0 * kPi * volume);
        energy += pref * c * (sr * sr + si * si);
        for (int j = 0; j < n; ++j) {
          double th = 2.0 * kPi * (k[0] * pos[3 * j] + k[1] * pos[3 * j + 1] + k[2] * pos[3 * j + 2]);
          // Im(conj(S) e^{i th}) = sr sin th - si cos th
          double im = sr * std::sin(th) - si * std::cos(th);
          for (int a = 0; a < 3; ++a) fx[3 * j + a] += pref * c * 4.0 * kPi * q[j] * k[a] * im;
        }
      }
  if (forces)
    for (size_t i = 0; i < fx.size(); ++i) forces[i] += fx[i];
  return energy;
}

int orc_nonbonded(int n, const double* pos, const double* charge, const double* sigma,
                  const double* epsilon, int n_exc, const int* exc_i, const int* exc_j,
                  const double* exc_qq, const double* exc_sigma, const double* exc_eps,
                  const orc_nonbonded_options* opt, const double* box, double* forces,
                  double* energy_out, double* virial, int threads) {
  const int method = opt->method;
  if (method == ORC_EWALD || method < 0 || method > ORC_PME) return -1;
  const bool use_cutoff = method != ORC_NO_CUTOFF;
  const bool use_pbc = method == ORC_CUTOFF_PERIODIC || method == ORC_PME;
  const double rc = opt->cutoff;
  const double cutoff2 = rc * rc;
  if (use_pbc) {
    if (!box) return -1;
    for (int a = 0; a < 3; ++a)
      if (!(2.0 * rc <= box[3 * a + a] + 1e-12)) return -2;
  }
  if (use_cutoff && opt->use_switching &&
      !(opt->switching_distance >= 0.0 && opt->switching_distance < rc))
    return -3;
  double alpha = 0.0;
  int dims[3] = {0, 0, 0};
  const bool pme = method == ORC_PME;
  if (pme) {
    if (opt->pme_alpha > 0.0) {
      alpha = opt->pme_alpha;
      for (int a = 0; a < 3; ++a) dims[a] = opt->pme_grid[a];
    } else {
      orc_pme_parameters(rc, opt->ewald_tolerance, box, &alpha, dims);
    }
  }
  std::fill(forces, forces + 3 * (size_t)n, 0.0);
  double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::set<int64_t> excluded;
  for (int e = 0; e < n_exc; ++e) excluded.insert(key_of(exc_i[e], exc_j[e]));

  const bool sw = use_cutoff && opt->use_switching;
  const double rs = opt->switching_distance;
#ifdef _OPENMP
  int nthreads = threads > 0 ? threads : omp_get_max_threads();
#else
  int nthreads = 1;
  (void)threads;
#endif
  double energy = 0.0;
  // nonbonded.rs:842-924 (evaluate_pair)
  auto evaluate_pair = [&](int i, int j, double* f, double* e, double* w) {
    if (excluded.count(key_of(i, j))) return;
    double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                   pos[3 * j + 2] - pos[3 * i + 2]};
    if (use_pbc) min_image(d, box);
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (use_cutoff && r2 >= cutoff2) return;
    double r = std::sqrt(r2);
    double lje, ljf;
    lj_pair(0.5 * (sigma[i] + sigma[j]), std::sqrt(epsilon[i] * epsilon[j]), r2, &lje, &ljf);
    if (sw && r > rs) {
      double t = (r - rs) / (rc - rs);
      double s = 1.0 + t * t * t * (-10.0 + t * (15.0 - 6.0 * t));
      double ds = -30.0 * t * t * (1.0 - t) * (1.0 - t) / (rc - rs);
      ljf = s * ljf + lje * ds / r;
      lje *= s;
    }
    double qq = charge[i] * charge[j];
    double ee, ef;
    if (pme)
      screened_coulomb(qq, r, r2, alpha, &ee, &ef);
    else if (use_cutoff)
      reaction_field(qq, r, r2, rc, opt->reaction_field_dielectric, &ee, &ef);
    else
      coulomb_pair(qq, r, r2, &ee, &ef);
    double fo = ljf + ef;
    *e += lje + ee;
    for (int a = 0; a < 3; ++a) {
      double fa = fo * d[a];
      f[3 * i + a] += fa;
      f[3 * j + a] -= fa;
    }
    if (w) add_pair_virial(w, fo, d);
  };
  if (opt->include_direct) {
    if (nthreads <= 1) {
      auto cb = [&](int i, int j) { evaluate_pair(i, j, forces, &energy, virial ? vir : nullptr); };
      if (use_cutoff && opt->use_neighbor_cells && n > 32)
        visit_cells(n, pos, rc, use_pbc ? box : nullptr, cb);
      else
        for (int i = 0; i < n; ++i)
          for (int j = i + 1; j < n; ++j) cb(i, j);
    } else {
      // Multithreaded form for the CPU baseline: candidate pairs collected per i-row, rows
      // split across threads, per-thread accumulators reduced in thread order.
      std::vector<std::vector<int>> rows(n);
      if (use_cutoff && opt->use_neighbor_cells && n > 32)
        visit_cells(n, pos, rc, use_pbc ? box : nullptr, [&](int i, int j) { rows[i].push_back(j); });
      std::vector<std::vector<double>> tf(nthreads, std::vector<double>(3 * (size_t)n, 0.0));
      std::vector<double> te(nthreads, 0.0);
      std::vector<std::array<double, 9>> tw(nthreads);
      for (auto& x : tw) x.fill(0.0);
      const bool all_pairs = !(use_cutoff && opt->use_neighbor_cells && n > 32);
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
      {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (int i = 0; i < n; ++i) {
          if (all_pairs) {
            for (int j = i + 1; j < n; ++j)
              evaluate_pair(i, j, tf[t].data(), &te[t], virial ? tw[t].data() : nullptr);
          } else {
            for (int j : rows[i]) evaluate_pair(i, j, tf[t].data(), &te[t], virial ? tw[t].data() : nullptr);
          }
        }
      }
      for (int t = 0; t < nthreads; ++t) {
        for (size_t k = 0; k < 3 * (size_t)n; ++k) forces[k] += tf[t][k];
        energy += te[t];
        for (int k = 0; k < 9; ++k) vir[k] += tw[t][k];
      }
    }
  }
  double volume = 0.0;
  if (use_pbc) {
    double recip[3][3];
    reciprocal_box(box, recip, &volume);
  }
  if (opt->include_reciprocal && pme) {
    energy += pme_reciprocal(n, pos, charge, box, alpha, dims, forces, virial ? vir : nullptr);
    // nonbonded.rs:965-972 self + neutralising plasma
    double q2 = 0.0, qt = 0.0;
    for (int i = 0; i < n; ++i) q2 += charge[i] * charge[i];
    for (int i = 0; i < n; ++i) qt += charge[i];
    double plasma = ONE_4PI_EPS0 * kPi * qt * qt / (2.0 * alpha * alpha * volume);
    energy -= ONE_4PI_EPS0 * (alpha / std::sqrt(kPi) * q2 + kPi * qt * qt / (2.0 * alpha * alpha * volume));
    // W = -dE/d strain of -plasma/V-like term: E_n = -plasma, dE_n/de_ab = plasma delta_ab
    vir[0] -= plasma;
    vir[4] -= plasma;
    vir[8] -= plasma;
  }
  if (opt->include_direct && use_pbc && opt->use_dispersion_correction) {
    double c = orc_dispersion_coefficient(n, sigma, epsilon, rc, opt->use_switching, rs);
    double ed = c / volume;
    energy += ed;
    vir[0] += ed;
    vir[4] += ed;
    vir[8] += ed;
  }
  // nonbonded.rs:995-1036 exceptions
  if (opt->include_direct) {
    for (int k = 0; k < n_exc; ++k) {
      int i = exc_i[k], j = exc_j[k];
      double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                     pos[3 * j + 2] - pos[3 * i + 2]};
      if (use_pbc && opt->exceptions_use_pbc) min_image(d, box);
      double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double r = std::sqrt(r2);
      double e1, f1, e2, f2;
      lj_pair(exc_sigma[k], exc_eps[k], r2, &e1, &f1);
      coulomb_pair(exc_qq[k], r, r2, &e2, &f2);
      double e = e1 + e2, fo = f1 + f2;
      if (pme) {
        double ce, cf;
        reciprocal_pair(charge[i] * charge[j], r, r2, alpha, &ce, &cf);
        e -= ce;
        fo -= cf;
      }
      energy += e;
      for (int a = 0; a < 3; ++a) {
        double fa = fo * d[a];
        forces[3 * i + a] += fa;
        forces[3 * j + a] -= fa;
      }
      add_pair_virial(vir, fo, d);
    }
  }
  *energy_out = energy;
  if (virial)
    for (int k = 0; k < 9; ++k) virial[k] = vir[k];
  return 0;
}

int64_t orc_pair_set(int n, const double* pos, double cutoff, const double* box, int use_pbc,
                     int n_exc, const int* exc_i, const int* exc_j, int use_cells,
                     int64_t max_pairs, int32_t* pairs) {
  std::set<int64_t> excluded;
  for (int e = 0; e < n_exc; ++e) excluded.insert(key_of(exc_i[e], exc_j[e]));
  const double c2 = cutoff * cutoff;
  int64_t count = 0;
  auto cb = [&](int i, int j) {
    if (excluded.count(key_of(i, j))) return;
    double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                   pos[3 * j + 2] - pos[3 * i + 2]};
    if (use_pbc) min_image(d, box);
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 >= c2) return;
    if (count < max_pairs && pairs) {
      pairs[2 * count] = i;
      pairs[2 * count + 1] = j;
    }
    ++count;
  };
  if (use_cells && n > 32)
    visit_cells(n, pos, cutoff, use_pbc ? box : nullptr, cb);
  else
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) cb(i, j);
  return count;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// GBSA OBC: gbsa_obc.rs:151-309
// ---------------------------------------------------------------------------------------
namespace {
struct GbParticle {
  double q, radius, scale;
};
double descreening(const GbParticle& i, const GbParticle& j, double r) {
  double radius = i.radius - DIELECTRIC_OFFSET;
  double scaled = (j.radius - DIELECTRIC_OFFSET) * j.scale;
  if (radius >= r + scaled) return 0.0;
  double lower = 1.0 / std::max(radius, std::fabs(r - scaled));
  double upper = 1.0 / (r + scaled);
  double inverse = 1.0 / r;
  double value = lower - upper + 0.25 * r * (upper * upper - lower * lower) +
                 0.5 * inverse * std::log(upper / lower) +
                 0.25 * scaled * scaled * inverse * (lower * lower - upper * upper);
  if (radius < scaled - r) value += 2.0 * (1.0 / radius - lower);
  return value;
}
double descreening_gradient(const GbParticle& i, const GbParticle& j, double r) {
  double radius = i.radius - DIELECTRIC_OFFSET;
  double scaled = (j.radius - DIELECTRIC_OFFSET) * j.scale;
  if (radius >= r + scaled) return 0.0;
  double lower = 1.0 / std::max(radius, std::fabs(r - scaled));
  double upper = 1.0 / (r + scaled);
  double inverse = 1.0 / r;
  return (0.125 * (1.0 + scaled * scaled * inverse * inverse) * (lower * lower - upper * upper) +
          0.25 * std::log(upper / lower) * inverse * inverse) *
         inverse;
}
}  // namespace

extern "C" int orc_gbsa_obc(int n, const double* pos, const double* charge, const double* radius,
                            const double* scale, int method, double cutoff,
                            double solvent_dielectric, double solute_dielectric,
                            double surface_area_energy, const double* box, double* forces,
                            double* energy_out, double* born_out, double* virial) {
  // method: 0 NoCutoff, 1 CutoffNonPeriodic, 2 CutoffPeriodic (gbsa_obc.rs:11-17)
  const bool periodic = method == 2;
  if (periodic) {
    if (!box) return -1;
    for (int i = 0; i < 3; ++i)
      if (!(box[3 * i + i] >= 2.0 * cutoff)) return -2;
  }
  std::vector<GbParticle> p(n);
  for (int i = 0; i < n; ++i) p[i] = {charge[i], radius[i], scale[i]};
  std::vector<double> born(n, 0.0), chain(n, 0.0), deriv(n, 0.0);
  std::fill(forces, forces + 3 * (size_t)n, 0.0);
  double vir[9] = {0};
  // gbsa_obc.rs:151-183 visit_pairs
  auto visit = [&](auto&& fn) {
    auto one = [&](int i, int j) {
      double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                     pos[3 * j + 2] - pos[3 * i + 2]};
      if (periodic) min_image(d, box);
      double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (method == 0 || r <= cutoff) fn(i, j, d, r);
    };
    if (method == 0) {
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) one(i, j);
    } else {
      visit_cells(n, pos, cutoff, periodic ? box : nullptr, one);
    }
  };
  visit([&](int i, int j, const double*, double r) {
    born[i] += descreening(p[i], p[j], r);
    born[j] += descreening(p[j], p[i], r);
  });
  double prefactor = (solute_dielectric != 0.0 && solvent_dielectric != 0.0)
                         ? -ONE_4PI_EPS0 * (1.0 / solute_dielectric - 1.0 / solvent_dielectric)
                         : 0.0;
  double surface = 4.0 * kPi * surface_area_energy;
  double energy = 0.0;
  for (int i = 0; i < n; ++i) {
    double offset = p[i].radius - DIELECTRIC_OFFSET;
    double psi = 0.5 * offset * born[i];
    double t = std::tanh(psi - 0.8 * psi * psi + 4.85 * psi * psi * psi);
    born[i] = 1.0 / (1.0 / offset - t / p[i].radius);
    chain[i] = offset * (1.0 - 1.6 * psi + 14.55 * psi * psi) * (1.0 - t * t) / p[i].radius;
    double self_energy = 0.5 * prefactor * p[i].q * p[i].q / std::fabs(born[i]);
    energy += self_energy;
    deriv[i] = -self_energy / born[i];
    if (born[i] > 0.0) {
      double area = surface * std::pow(p[i].radius + PROBE_RADIUS, 2) * std::pow(p[i].radius / born[i], 6);
      energy += area;
      deriv[i] -= 6.0 * area / born[i];
    }
  }
  visit([&](int i, int j, const double* d, double r) {
    double product = born[i] * born[j];
    double dd = r * r / (4.0 * product);
    double ex = std::exp(-dd);
    double den2 = r * r + product * ex;
    double coefficient = prefactor * p[i].q * p[j].q;
    double pe = coefficient / std::sqrt(den2);
    energy += (method == 0) ? pe : pe - coefficient / cutoff;
    double radial = -pe * (1.0 - 0.25 * ex) / den2;
    double bd = -0.5 * pe * ex * (1.0 + dd) / den2;
    deriv[i] += bd * born[j];
    deriv[j] += bd * born[i];
    for (int a = 0; a < 3; ++a) {
      double f = radial * d[a];
      forces[3 * i + a] += f;
      forces[3 * j + a] -= f;
    }
    add_pair_virial(vir, radial, d);
  });
  for (int i = 0; i < n; ++i) deriv[i] *= born[i] * born[i] * chain[i];
  visit([&](int i, int j, const double* d, double r) {
    double radial = -(deriv[i] * descreening_gradient(p[i], p[j], r) +
                      deriv[j] * descreening_gradient(p[j], p[i], r));
    for (int a = 0; a < 3; ++a) {
      double f = radial * d[a];
      forces[3 * i + a] += f;
      forces[3 * j + a] -= f;
    }
    add_pair_virial(vir, radial, d);
  });
  *energy_out = energy;
  if (born_out)
    for (int i = 0; i < n; ++i) born_out[i] = born[i];
  if (virial)
    for (int k = 0; k < 9; ++k) virial[k] = vir[k];
  return 0;
}

// ---------------------------------------------------------------------------------------
// Learned Born radii (no reference counterpart; the OBC terms follow gbsa_obc.rs:184-309).
// The HCT integral is split as I_i = I_short_i + tail_i:
//   I_short_i = sum_j H(r_ij; rho_i, s_j) S(r_ij), S the quintic switch from rs to rc;
//   tail_i    = the network's prediction from radial symmetry functions (Behler & Parrinello,
//               Phys. Rev. Lett. 98, 146401 (2007)) G_if = sum_j exp(-eta (r_ij - mu_f)^2)
//               fc(r_ij) over r_ij < rf, fc(r) = (cos(pi r / rf) + 1) / 2, mu_f = mu0 + f dmu.
// Forces follow from dE/dI_i and dI_i/dr_ij = Phi'_ij(r) with
//   Phi_ij(r) = H(r; i, j) S(r) + sum_f (d tail_i / d G_if) g_f(r).
// ---------------------------------------------------------------------------------------
namespace {
double switch_value(double r, double rs, double rc, double* deriv) {
  if (r <= rs) {
    *deriv = 0.0;
    return 1.0;
  }
  if (r >= rc) {
    *deriv = 0.0;
    return 0.0;
  }
  const double w = rc - rs, t = (r - rs) / w;
  *deriv = -30.0 * t * t * (1.0 - t) * (1.0 - t) / w;
  return 1.0 + t * t * t * (-10.0 + t * (15.0 - 6.0 * t));
}
// g_f(r) and g_f'(r) for all features; zero beyond rc.
void radial_functions(double r, int nf, double mu0, double dmu, double eta, double rc,
                      double* g, double* dg) {
  if (r >= rc) {
    for (int f = 0; f < nf; ++f) g[f] = dg[f] = 0.0;
    return;
  }
  const double fc = 0.5 * (std::cos(kPi * r / rc) + 1.0);
  const double dfc = -0.5 * kPi / rc * std::sin(kPi * r / rc);
  for (int f = 0; f < nf; ++f) {
    const double x = r - (mu0 + f * dmu);
    const double e = std::exp(-eta * x * x);
    g[f] = e * fc;
    dg[f] = e * (-2.0 * eta * x * fc + dfc);
  }
}
}  // namespace

extern "C" int orc_radial_features(int n, const double* pos, int nf, double mu0, double dmu,
                                   double eta, double rc, double* features) {
  if (nf <= 0 || nf > 64) return -1;
  std::fill(features, features + (size_t)n * nf, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    double g[64], dg[64];
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
      const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r >= rc) continue;
      radial_functions(r, nf, mu0, dmu, eta, rc, g, dg);
      for (int f = 0; f < nf; ++f) features[(size_t)i * nf + f] += g[f];
    }
  }
  return 0;
}

extern "C" int orc_learned_gbsa(int n, const double* pos, const double* charge,
                                const double* radius, const double* scale,
                                double solvent_dielectric, double solute_dielectric,
                                double surface_area_energy, double rs, double rc, double rf,
                                int nf, double mu0, double dmu, double eta, const double* tail,
                                const double* dtail_dg, double* forces, double* energy_out,
                                double* born_out, double* short_out, double* full_out) {
  if (nf <= 0 || nf > 64 || !(rs < rc) || !(rf > 0.0)) return -1;
  std::vector<GbParticle> p(n);
  for (int i = 0; i < n; ++i) p[i] = {charge[i], radius[i], scale[i]};
  std::vector<double> integral(n, 0.0), full(n, 0.0), born(n), dedi(n, 0.0);
  std::fill(forces, forces + 3 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
      const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double hij = descreening(p[i], p[j], r), hji = descreening(p[j], p[i], r);
      full[i] += hij;
      full[j] += hji;
      double ds;
      const double sw = switch_value(r, rs, rc, &ds);
      integral[i] += hij * sw;
      integral[j] += hji * sw;
    }
  if (short_out)
    for (int i = 0; i < n; ++i) short_out[i] = integral[i];
  if (full_out)
    for (int i = 0; i < n; ++i) full_out[i] = full[i];
  for (int i = 0; i < n; ++i) integral[i] += tail[i];
  const double prefactor = (solute_dielectric != 0.0 && solvent_dielectric != 0.0)
                               ? -ONE_4PI_EPS0 * (1.0 / solute_dielectric - 1.0 / solvent_dielectric)
                               : 0.0;
  const double surface = 4.0 * kPi * surface_area_energy;
  double energy = 0.0;
  std::vector<double> dridi(n);
  for (int i = 0; i < n; ++i) {  // gbsa_obc.rs:214-237
    const double offset = p[i].radius - DIELECTRIC_OFFSET;
    const double psi = 0.5 * offset * integral[i];
    const double t = std::tanh(psi - 0.8 * psi * psi + 4.85 * psi * psi * psi);
    born[i] = 1.0 / (1.0 / offset - t / p[i].radius);
    // dR/dI = R^2 (1 - t^2)(1 - 1.6 psi + 14.55 psi^2) / rho * offset / 2
    dridi[i] = born[i] * born[i] * (1.0 - t * t) * (1.0 - 1.6 * psi + 14.55 * psi * psi) /
               p[i].radius * 0.5 * offset;
    const double self_energy = 0.5 * prefactor * p[i].q * p[i].q / std::fabs(born[i]);
    energy += self_energy;
    dedi[i] = -self_energy / born[i];
    if (born[i] > 0.0) {
      const double area = surface * std::pow(p[i].radius + PROBE_RADIUS, 2) *
                          std::pow(p[i].radius / born[i], 6);
      energy += area;
      dedi[i] -= 6.0 * area / born[i];
    }
  }
  for (int i = 0; i < n; ++i)  // gbsa_obc.rs:239-260 (NoCutoff)
    for (int j = i + 1; j < n; ++j) {
      const double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const double product = born[i] * born[j];
      const double dd = r2 / (4.0 * product);
      const double ex = std::exp(-dd);
      const double den2 = r2 + product * ex;
      const double pe = prefactor * p[i].q * p[j].q / std::sqrt(den2);
      energy += pe;
      const double radial = -pe * (1.0 - 0.25 * ex) / den2;
      const double bd = -0.5 * pe * ex * (1.0 + dd) / den2;
      dedi[i] += bd * born[j];
      dedi[j] += bd * born[i];
      for (int a = 0; a < 3; ++a) {
        forces[3 * i + a] += radial * d[a];
        forces[3 * j + a] -= radial * d[a];
      }
    }
  for (int i = 0; i < n; ++i) dedi[i] *= dridi[i];  // dE/dI_i
  std::vector<double> g(nf), dg(nf);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
      const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r >= rc) continue;
      double ds;
      const double sw = switch_value(r, rs, rc, &ds);
      // dH/dr = -2 r descreening_gradient (gbsa_obc.rs:297-309)
      double phi_ij = -2.0 * r * descreening_gradient(p[i], p[j], r) * sw +
                      descreening(p[i], p[j], r) * ds;
      double phi_ji = -2.0 * r * descreening_gradient(p[j], p[i], r) * sw +
                      descreening(p[j], p[i], r) * ds;
      radial_functions(r, nf, mu0, dmu, eta, rf, g.data(), dg.data());
      for (int f = 0; f < nf; ++f) {
        phi_ij += dtail_dg[(size_t)i * nf + f] * dg[f];
        phi_ji += dtail_dg[(size_t)j * nf + f] * dg[f];
      }
      const double radial = (dedi[i] * phi_ij + dedi[j] * phi_ji) / r;
      for (int a = 0; a < 3; ++a) {
        forces[3 * i + a] += radial * d[a];
        forces[3 * j + a] -= radial * d[a];
      }
    }
  *energy_out = energy;
  if (born_out)
    for (int i = 0; i < n; ++i) born_out[i] = born[i];
  return 0;
}

// ---------------------------------------------------------------------------------------
// Bonded terms: harmonic_bond.rs:102-144, harmonic_angle.rs:102-175
// ---------------------------------------------------------------------------------------
extern "C" double orc_harmonic_bond(int nb, const int* bi, const int* bj, const double* length,
                                    const double* k, const double* pos, int use_pbc,
                                    const double* box, double* forces, double* virial) {
  double energy = 0.0;
  for (int b = 0; b < nb; ++b) {
    int i = bi[b], j = bj[b];
    double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                   pos[3 * j + 2] - pos[3 * i + 2]};
    if (use_pbc && box) min_image(d, box);
    double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double dr = r - length[b];
    energy += 0.5 * k[b] * dr * dr;
    double fm = k[b] * dr / r;
    for (int a = 0; a < 3; ++a) {
      double f = fm * d[a];
      forces[3 * i + a] += f;
      forces[3 * j + a] -= f;
    }
    if (virial) add_pair_virial(virial, fm, d);
  }
  return energy;
}

extern "C" double orc_harmonic_angle(int na, const int* ai, const int* aj, const int* ak,
                                     const double* angle, const double* kk, const double* pos,
                                     int use_pbc, const double* box, double* forces,
                                     double* virial) {
  double energy = 0.0;
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  for (int t = 0; t < na; ++t) {
    int i = ai[t], j = aj[t], k = ak[t];
    double rji[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    double rjk[3] = {pos[3 * k] - pos[3 * j], pos[3 * k + 1] - pos[3 * j + 1], pos[3 * k + 2] - pos[3 * j + 2]};
    if (use_pbc && box) {
      min_image(rji, box);
      min_image(rjk, box);
    }
    double li = std::sqrt(dot(rji, rji));
    double lk = std::sqrt(dot(rjk, rjk));
    double c = std::min(std::max(dot(rji, rjk) / (li * lk), -1.0), 1.0);
    double theta = std::acos(c);
    double dt = theta - angle[t];
    energy += 0.5 * kk[t] * dt * dt;
    double s = std::max(std::sqrt(1.0 - c * c), 1e-8);
    double de = kk[t] * dt;
    double fi[3], fk[3];
    for (int d = 0; d < 3; ++d) {
      fi[d] = de * (c * rji[d] / li - rjk[d] / lk) / (li * s);
      fk[d] = de * (c * rjk[d] / lk - rji[d] / li) / (lk * s);
      forces[3 * i + d] -= fi[d];
      forces[3 * k + d] -= fk[d];
      forces[3 * j + d] += fi[d] + fk[d];
    }
    if (virial)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) virial[3 * a + b] += -fi[a] * rji[b] - fk[a] * rjk[b];
  }
  return energy;
}

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11) and Box-Muller normals.
// ---------------------------------------------------------------------------------------
extern "C" void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                  uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

extern "C" void orc_gaussian_noise(uint64_t seed, uint64_t stream, uint64_t step, int n,
                                   double* out) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int a = 0; a < n; ++a) {
    const uint32_t ctr[4] = {(uint32_t)a, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)stream};
    uint32_t r[4];
    orc_philox4x32_10(ctr, key, r);
    double u[4];
    for (int k = 0; k < 4; ++k) u[k] = ((double)r[k] + 0.5) * 2.3283064365386962890625e-10;
    double m0 = std::sqrt(-2.0 * std::log(u[0]));
    double m1 = std::sqrt(-2.0 * std::log(u[2]));
    out[3 * a + 0] = m0 * std::cos(2.0 * kPi * u[1]);
    out[3 * a + 1] = m0 * std::sin(2.0 * kPi * u[1]);
    out[3 * a + 2] = m1 * std::cos(2.0 * kPi * u[3]);
  }
}

// ---------------------------------------------------------------------------------------
// Constraints: constraints.rs:81-156
// ---------------------------------------------------------------------------------------
extern "C" int orc_constraints_solve(int nc, const int* ci, const int* cj, const double* distance,
                                     const double* masses, const double* reference,
                                     double* values, int velocities, double tolerance) {
  if (!(std::isfinite(tolerance) && tolerance > 0.0 && tolerance < 1.0)) return -5;
  struct Prep {
    int i, j;
    double wi, wj, d2;
    double dir[3];
  };
  std::vector<Prep> cs;
  for (int c = 0; c < nc; ++c) {
    int i = ci[c], j = cj[c];
    if (masses[i] == 0.0) continue;
    Prep p;
    p.i = i;
    p.j = j;
    p.wi = 1.0 / masses[i];
    p.wj = 1.0 / masses[j];
    p.d2 = distance[c] * distance[c];
    for (int a = 0; a < 3; ++a) p.dir[a] = reference[3 * i + a] - reference[3 * j + a];
    cs.push_back(p);
  }
  for (int it = 0; it < 1000; ++it) {
    bool converged = true;
    for (const Prep& c : cs) {
      double delta[3];
      for (int a = 0; a < 3; ++a) delta[a] = values[3 * c.i + a] - values[3 * c.j + a];
      double dot = delta[0] * c.dir[0] + delta[1] * c.dir[1] + delta[2] * c.dir[2];
      double mult;
      if (velocities) {
        double norm = c.dir[0] * c.dir[0] + c.dir[1] * c.dir[1] + c.dir[2] * c.dir[2];
        if (norm == 0.0 || !std::isfinite(norm)) return -4;
        double corr = -dot / ((c.wi + c.wj) * norm);
        if (std::fabs(corr) <= tolerance) continue;
        mult = corr;
      } else {
        double norm = delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2];
        double ratio = std::sqrt(norm / c.d2);
        if (std::isfinite(ratio) && std::fabs(ratio - 1.0) <= tolerance) continue;
        double den = 2.0 * (c.wi + c.wj) * dot;
        if (std::fabs(den) < 2.2250738585072014e-308 || !std::isfinite(den)) return -2;
        mult = (c.d2 - norm) / den;
      }
      if (!std::isfinite(mult)) return -3;
      converged = false;
      for (int a = 0; a < 3; ++a) {
        double corr = mult * c.dir[a];
        values[3 * c.i + a] += c.wi * corr;
        values[3 * c.j + a] -= c.wj * corr;
      }
    }
    if (converged) return 0;
  }
  return -1;
}

// ---------------------------------------------------------------------------------------
// SETTLE for rigid 3-site water, written from Miyamoto & Kollman (1992).  The constraint
// displacements lie in the plane of the old (reference) molecule, so in a frame whose z axis
// is that plane's normal every atom keeps its unconstrained z; the canonical triangle is tilted
// by phi (about x) and psi (about y) to reproduce those z values, then rotated in-plane by the
// theta that makes the mass-weighted torque of the displacements about z vanish.
// ---------------------------------------------------------------------------------------
namespace {
inline void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void normalize3(double* a) {
  double s = 1.0 / std::sqrt(dot3(a, a));
  a[0] *= s;
  a[1] *= s;
  a[2] *= s;
}
}  // namespace

extern "C" int orc_settle_positions(int nw, const int* atoms, double d_oh, double d_hh,
                                    const double* masses, const double* ref, double* x) {
  for (int w = 0; w < nw; ++w) {
    const int o = atoms[3 * w], h1 = atoms[3 * w + 1], h2 = atoms[3 * w + 2];
    const double mo = masses[o], mh = masses[h1];
    const double mt = mo + 2.0 * mh;
    const double rc = 0.5 * d_hh;
    const double hgt = std::sqrt(d_oh * d_oh - rc * rc);
    const double ra = 2.0 * mh * hgt / mt;
    const double rb = hgt - ra;
    double com[3];
    for (int a = 0; a < 3; ++a) com[a] = (mo * x[3 * o + a] + mh * x[3 * h1 + a] + mh * x[3 * h2 + a]) / mt;
    double a1[3], b1[3], c1[3], u[3], v[3];
    for (int a = 0; a < 3; ++a) {
      a1[a] = x[3 * o + a] - com[a];
      b1[a] = x[3 * h1 + a] - com[a];
      c1[a] = x[3 * h2 + a] - com[a];
      u[a] = ref[3 * h1 + a] - ref[3 * o + a];
      v[a] = ref[3 * h2 + a] - ref[3 * o + a];
    }
    double ez[3], ex[3], ey[3];
    cross3(u, v, ez);
    cross3(a1, ez, ex);
    cross3(ez, ex, ey);
    normalize3(ez);
    normalize3(ex);
    normalize3(ey);
    // old geometry (relative to O) and new positions (relative to COM) in the frame
    const double xb0 = dot3(u, ex), yb0 = dot3(u, ey);
    const double xc0 = dot3(v, ex), yc0 = dot3(v, ey);
    const double za1 = dot3(a1, ez);
    const double xb1 = dot3(b1, ex), yb1 = dot3(b1, ey), zb1 = dot3(b1, ez);
    const double xc1 = dot3(c1, ex), yc1 = dot3(c1, ey), zc1 = dot3(c1, ez);
    const double sphi = za1 / ra;
    const double cphi2 = 1.0 - sphi * sphi;
    if (!(cphi2 > 0.0)) return -2;
    const double cphi = std::sqrt(cphi2);
    const double spsi = (zb1 - zc1) / (2.0 * rc * cphi);
    const double cpsi2 = 1.0 - spsi * spsi;
    if (!(cpsi2 > 0.0)) return -2;
    const double cpsi = std::sqrt(cpsi2);
    // tilted canonical triangle, in-plane components
    const double ya2 = ra * cphi;
    const double xb2 = -rc * cpsi;
    const double yb2 = -rb * cphi - rc * spsi * sphi;
    const double yc2 = -rb * cphi + rc * spsi * sphi;
    const double xc2 = rc * cpsi;
    // alpha sin(theta) + beta cos(theta) = gamma over the two hydrogens
    const double alpha = xb0 * xb2 + yb0 * yb2 + xc0 * xc2 + yc0 * yc2;
    const double beta = xb0 * yb2 - yb0 * xb2 + xc0 * yc2 - yc0 * xc2;
    const double gamma = xb0 * yb1 - yb0 * xb1 + xc0 * yc1 - yc0 * xc1;
    const double ab2 = alpha * alpha + beta * beta;
    const double disc = ab2 - gamma * gamma;
    if (!(disc >= 0.0)) return -2;
    const double sth = (alpha * gamma - beta * std::sqrt(disc)) / ab2;
    const double cth = std::sqrt(1.0 - sth * sth);
    const double p3[3][3] = {
        {-ya2 * sth, ya2 * cth, za1},
        {xb2 * cth - yb2 * sth, xb2 * sth + yb2 * cth, zb1},
        {xc2 * cth - yc2 * sth, xc2 * sth + yc2 * cth, zc1},
    };
    const int idx[3] = {o, h1, h2};
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a)
        x[3 * idx[k] + a] = com[a] + p3[k][0] * ex[a] + p3[k][1] * ey[a] + p3[k][2] * ez[a];
  }
  return 0;
}

extern "C" int orc_settle_velocities(int nw, const int* atoms, const double* masses,
                                     const double* x, double* v) {
  // Exact projection: find lambda_k (k = O-H1, O-H2, H1-H2) with v_p += lambda d / m_p,
  // v_q -= lambda d / m_q (d = x_p - x_q) such that d_k . (v_p - v_q) = 0 for all k.
  for (int w = 0; w < nw; ++w) {
    const int at[3] = {atoms[3 * w], atoms[3 * w + 1], atoms[3 * w + 2]};
    const int cp[3] = {0, 0, 1}, cq[3] = {1, 2, 2};
    double d[3][3], inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0 / masses[at[k]];
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) d[k][a] = x[3 * at[cp[k]] + a] - x[3 * at[cq[k]] + a];
    double A[3][3], b[3];
    for (int k = 0; k < 3; ++k) {
      double rel[3];
      for (int a = 0; a < 3; ++a) rel[a] = v[3 * at[cp[k]] + a] - v[3 * at[cq[k]] + a];
      b[k] = -dot3(d[k], rel);
      for (int l = 0; l < 3; ++l) {
        // change of (v_p(k) - v_q(k)) per unit lambda_l, along d_l
        double s = 0.0;
        if (cp[l] == cp[k]) s += inv[cp[k]];
        if (cq[l] == cp[k]) s -= inv[cp[k]];
        if (cp[l] == cq[k]) s -= inv[cq[k]];
        if (cq[l] == cq[k]) s += inv[cq[k]];
        A[k][l] = s * dot3(d[k], d[l]);
      }
    }
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                 A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                 A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return -4;
    double lam[3];
    for (int c = 0; c < 3; ++c) {
      double M[3][3];
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) M[r][q] = (q == c) ? b[r] : A[r][q];
      lam[c] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) /
               det;
    }
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) {
        v[3 * at[cp[k]] + a] += lam[k] * d[k][a] * inv[cp[k]];
        v[3 * at[cq[k]] + a] -= lam[k] * d[k][a] * inv[cq[k]];
      }
  }
  return 0;
}

// ---------------------------------------------------------------------------------------
// LangevinMiddleIntegrator: langevin.rs:103-141 (host update) and 216-278 (constrained),
// integrators/mod.rs:232-268 (velocity correction).
// ---------------------------------------------------------------------------------------
extern "C" int orc_lfmiddle_step(int n, double* pos, double* vel, const double* forces,
                                 const double* masses, double dt, double temperature,
                                 double friction, const double* noise, int nc, const int* ci,
                                 const int* cj, const double* distance, double tolerance,
                                 int constraint_mode, int nw, const int* waters, double d_oh,
                                 double d_hh) {
  const double half_dt = 0.5 * dt;
  const double decay = std::exp(-friction * dt);
  const double variance = BOLTZMANN * temperature * -std::expm1(-2.0 * friction * dt);
  const bool constrained = (constraint_mode == 0 && nc > 0) || (constraint_mode == 1 && nw > 0);
  auto host_update = [&](bool kick) {
    for (int atom = 0; atom < n; ++atom) {
      double m = masses[atom];
      if (m == 0.0) continue;
      double im = 1.0 / m;
      double ns = std::sqrt(variance * im);
      for (int a = 0; a < 3; ++a) {
        int i = 3 * atom + a;
        if (kick) vel[i] += forces[i] * im * dt;
        double mid = pos[i] + half_dt * vel[i];
        vel[i] = decay * vel[i] + ns * noise[i];
        pos[i] = mid + half_dt * vel[i];
      }
    }
  };
  if (!constrained) {
    host_update(true);
    return 0;
  }
  std::vector<double> previous(pos, pos + 3 * (size_t)n);
  for (int atom = 0; atom < n; ++atom) {
    double m = masses[atom];
    if (m == 0.0) continue;
    double im = 1.0 / m;
    for (int a = 0; a < 3; ++a) vel[3 * atom + a] += forces[3 * atom + a] * im * dt;
  }
  int rc;
  if (constraint_mode == 0)
    rc = orc_constraints_solve(nc, ci, cj, distance, masses, pos, vel, 1, tolerance);
  else
    rc = orc_settle_velocities(nw, waters, masses, pos, vel);
  if (rc) return rc;
  host_update(false);
  std::vector<double> proposed(pos, pos + 3 * (size_t)n);
  if (constraint_mode == 0)
    rc = orc_constraints_solve(nc, ci, cj, distance, masses, previous.data(), pos, 0, tolerance);
  else
    rc = orc_settle_positions(nw, waters, d_oh, d_hh, masses, previous.data(), pos);
  if (rc) return rc;
  for (int atom = 0; atom < n; ++atom) {
    if (masses[atom] == 0.0) continue;
    for (int a = 0; a < 3; ++a) {
      int i = 3 * atom + a;
      vel[i] += (pos[i] - proposed[i]) / dt;
    }
  }
  return 0;
}

extern "C" double orc_kinetic_energy(int n, const double* vel, const double* masses) {
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    s += masses[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
  return 0.5 * s;
}

extern "C" double orc_wtime(void) {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

extern "C" int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
