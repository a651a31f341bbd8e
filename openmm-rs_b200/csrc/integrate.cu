// Fused LangevinMiddle step with constraints, in f64.
//
// Per particle this is integrators/langevin.rs:216-278: kick v += F/m dt, velocity constraint
// projection, x += dt/2 v, v = a v + sqrt(kT (1 - a^2) / m) xi, x += dt/2 v, position
// constraints against the start-of-step positions, v += (x_constrained - x_proposed) / dt.
// Rigid 3-site waters use analytic SETTLE (Miyamoto & Kollman 1992) and the exact rigid-body
// velocity projection, which are the converged limits of the reference's SHAKE / RATTLE
// (constraints.rs:81-156); other constraint clusters run the reference's Gauss-Seidel SHAKE /
// RATTLE, one thread per cluster.  Unconstrained particles take the plain update
// (langevin.rs:103-141); massless particles are never moved.
//
// Gaussian numbers come from Philox4x32-10 keyed by the seed and counted by (particle, step),
// so the stream is reproducible and independent of the launch shape.  Failures set the status
// word instead of trapping; the host turns it into OMMB200_ERR_CONSTRAINT / _NONFINITE.
#include "kernels.h"

namespace ommb200 {
namespace {

__device__ __forceinline__ void ld3(const double* p, int i, double o[3]) {
  o[0] = p[3 * i];
  o[1] = p[3 * i + 1];
  o[2] = p[3 * i + 2];
}
__device__ __forceinline__ void st3(double* p, int i, const double o[3]) {
  p[3 * i] = o[0];
  p[3 * i + 1] = o[1];
  p[3 * i + 2] = o[2];
}
__device__ __forceinline__ void force3(const long long* f, int n, int i, double o[3]) {
  o[0] = (double)f[i] * kForceScaleInv;
  o[1] = (double)f[n + i] * kForceScaleInv;
  o[2] = (double)f[2 * n + i] * kForceScaleInv;
}
// The force of `atom` for this step's kick; zeroed behind the read when the step owns the
// clearing for the next evaluation.
__device__ __forceinline__ void consume_force(const IntegrateArgs& a, int n, int atom, double o[3]) {
  force3(a.force, n, atom, o);
  if (a.zero_force) {
    a.force[atom] = 0;
    a.force[n + atom] = 0;
    a.force[2 * n + atom] = 0;
  }
}


__device__ __forceinline__ double dot(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ void unit(double* a) {
  const double s = rsqrt(dot(a, a));
  a[0] *= s;
  a[1] *= s;
  a[2] *= s;
}

// SETTLE: x[0..2] (O, H1, H2) are unconstrained new positions, r[0..2] the reference ones.
// The constraint displacements lie in the reference plane, so in a frame with z along that
// plane's normal every atom keeps its unconstrained z; the canonical triangle is tilted
// (phi about x, psi about y) to match, then turned in-plane by the theta that zeroes the
// mass-weighted torque of the displacements.  Returns false if no rigid solution exists.
__device__ bool settle_positions(const WaterGeometry& g, const double r[3][3], double x[3][3]) {
  const double mt = g.m_o + 2.0 * g.m_h;
  const double rc = 0.5 * g.d_hh;
  const double hgt = sqrt(g.d_oh * g.d_oh - rc * rc);
  const double ra = 2.0 * g.m_h * hgt / mt;
  const double rb = hgt - ra;
  double com[3], a1[3], b1[3], c1[3], u[3], v[3];
  for (int d = 0; d < 3; ++d) {
    com[d] = (g.m_o * x[0][d] + g.m_h * x[1][d] + g.m_h * x[2][d]) / mt;
    a1[d] = x[0][d] - com[d];
    b1[d] = x[1][d] - com[d];
    c1[d] = x[2][d] - com[d];
    u[d] = r[1][d] - r[0][d];
    v[d] = r[2][d] - r[0][d];
  }
  double ez[3], ex[3], ey[3];
  cross(u, v, ez);
  cross(a1, ez, ex);
  cross(ez, ex, ey);
  unit(ez);
  unit(ex);
  unit(ey);
  const double xb0 = dot(u, ex), yb0 = dot(u, ey), xc0 = dot(v, ex), yc0 = dot(v, ey);
  const double za1 = dot(a1, ez);
  const double xb1 = dot(b1, ex), yb1 = dot(b1, ey), zb1 = dot(b1, ez);
  const double xc1 = dot(c1, ex), yc1 = dot(c1, ey), zc1 = dot(c1, ez);
  const double sphi = za1 / ra;
  const double cphi2 = 1.0 - sphi * sphi;
  if (!(cphi2 > 0.0)) return false;
  const double cphi = sqrt(cphi2);
  const double spsi = (zb1 - zc1) / (2.0 * rc * cphi);
  const double cpsi2 = 1.0 - spsi * spsi;
  if (!(cpsi2 > 0.0)) return false;
  const double cpsi = sqrt(cpsi2);
  const double ya2 = ra * cphi;
  const double xb2 = -rc * cpsi, yb2 = -rb * cphi - rc * spsi * sphi;
  const double xc2 = rc * cpsi, yc2 = -rb * cphi + rc * spsi * sphi;
  const double alpha = xb0 * xb2 + yb0 * yb2 + xc0 * xc2 + yc0 * yc2;
  const double beta = xb0 * yb2 - yb0 * xb2 + xc0 * yc2 - yc0 * xc2;
  const double gamma = xb0 * yb1 - yb0 * xb1 + xc0 * yc1 - yc0 * xc1;
  const double ab2 = alpha * alpha + beta * beta;
  const double disc = ab2 - gamma * gamma;
  if (!(disc >= 0.0)) return false;
  const double sth = (alpha * gamma - beta * sqrt(disc)) / ab2;
  const double cth = sqrt(1.0 - sth * sth);
  const double p[3][3] = {{-ya2 * sth, ya2 * cth, za1},
                          {xb2 * cth - yb2 * sth, xb2 * sth + yb2 * cth, zb1},
                          {xc2 * cth - yc2 * sth, xc2 * sth + yc2 * cth, zc1}};
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < 3; ++d) x[k][d] = com[d] + p[k][0] * ex[d] + p[k][1] * ey[d] + p[k][2] * ez[d];
  return true;
}

// Exact velocity projection of a rigid water: solve for the three multipliers so that every
// bond's relative velocity is perpendicular to the bond (the limit RATTLE converges to).
__device__ bool settle_velocities(const double x[3][3], const double im[3], double v[3][3]) {
  const int cp[3] = {0, 0, 1}, cq[3] = {1, 2, 2};
  double d[3][3], A[3][3], b[3];
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) d[k][c] = x[cp[k]][c] - x[cq[k]][c];
  for (int k = 0; k < 3; ++k) {
    const double rel[3] = {v[cp[k]][0] - v[cq[k]][0], v[cp[k]][1] - v[cq[k]][1], v[cp[k]][2] - v[cq[k]][2]};
    b[k] = -dot(d[k], rel);
    for (int l = 0; l < 3; ++l) {
      double s = 0.0;
      if (cp[l] == cp[k]) s += im[cp[k]];
      if (cq[l] == cp[k]) s -= im[cp[k]];
      if (cp[l] == cq[k]) s -= im[cq[k]];
      if (cq[l] == cq[k]) s += im[cq[k]];
      A[k][l] = s * dot(d[k], d[l]);
    }
  }
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
  double lam[3];
  for (int c = 0; c < 3; ++c) {
    double M[3][3];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) M[r][q] = (q == c) ? b[r] : A[r][q];
    lam[c] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
              M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
              M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) / det;
  }
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) {
      v[cp[k]][c] += lam[k] * d[k][c] * im[cp[k]];
      v[cq[k]][c] -= lam[k] * d[k][c] * im[cq[k]];
    }
  return true;
}

__device__ __forceinline__ bool finite3(const double a[3]) {
  return isfinite(a[0]) && isfinite(a[1]) && isfinite(a[2]);
}

// What a particle's end-of-step bookkeeping reads (neighbour-list and prune reference
// positions, slot, lattice image, block centre), loaded at the start of the step so that the
// loads overlap the arithmetic instead of following the stores of x and v.
struct StepTail {
  double ref[3], prune_ref[3], img[3];
  const double* center;
  int slot;
};

__device__ __forceinline__ void load_tail(const IntegrateArgs& a, int atom, StepTail& t) {
  if (a.pos_ref) ld3(a.pos_ref, atom, t.ref);
  if (a.pos_prune) ld3(a.pos_prune, atom, t.prune_ref);
  if (a.posq) {
    t.slot = a.atom_slot[atom];
    t.img[0] = a.image[3 * atom];
    t.img[1] = a.image[3 * atom + 1];
    t.img[2] = a.image[3 * atom + 2];
    t.center = a.block_center + 3 * (t.slot >> 5);
  }
}

__device__ __forceinline__ void check_rebuild(const IntegrateArgs& a, const StepTail& t,
                                              const double x[3]) {
  if (!a.pos_ref) return;
  const double dx = x[0] - t.ref[0], dy = x[1] - t.ref[1], dz = x[2] - t.ref[2];
  if (dx * dx + dy * dy + dz * dz > a.half_skin2) *a.rebuild = 1;
  if (!a.pos_prune) return;
  const double px = x[0] - t.prune_ref[0], py = x[1] - t.prune_ref[1], pz = x[2] - t.prune_ref[2];
  if (px * px + py * py + pz * pz > a.half_margin2) *a.prune = 1;
}

// The pair kernel's packed coordinates of `atom` at its new position x (periodic lists; the
// same block-local arithmetic as the pack kernel); `q` = its scaled charge.
__device__ __forceinline__ void write_packed(const IntegrateArgs& a, const StepTail& t, double q,
                                             const double x[3]) {
  if (!a.posq) return;
  double r[3];
  block_local(x, t.img[0], t.img[1], t.img[2], t.center, a.pbox, r);
  if (a.posq_double)
    reinterpret_cast<double4*>(a.posq)[t.slot] = make_double4(r[0], r[1], r[2], q);
  else
    reinterpret_cast<float4*>(a.posq)[t.slot] =
        make_float4((float)r[0], (float)r[1], (float)r[2], (float)q);
}

// drift / thermostat / drift for one particle (langevin.rs:121-134 without the kick)
__device__ __forceinline__ void ou_update(const IntegrateArgs& a, int atom, double im, uint64_t step,
                                          double x[3], double v[3]) {
  double xi[3];
  gaussian3(a.seed, 0, step, (uint32_t)atom, xi);
  const double ns = sqrt(a.noise_var * im);
  const double h = 0.5 * a.dt;
  for (int c = 0; c < 3; ++c) {
    const double mid = x[c] + h * v[c];
    v[c] = a.decay * v[c] + ns * xi[c];
    x[c] = mid + h * v[c];
  }
}

// One rigid water on four lanes: lane k < 3 loads, kicks, draws the noise for and stores atom
// k (the Gaussian draws, the longest part of the chain, run side by side); the two SETTLE
// solves (velocity projection after the kick, positions after the drift) run on all four
// lanes from shuffled copies of the three atoms.
__device__ __forceinline__ void share3(double (&o)[3][3], const double mine[3], unsigned gmask) {
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) o[k][c] = __shfl_sync(gmask, mine[c], k, 4);
}

// o = m[k] without indexing the array by a run-time value (keeps m in registers)
__device__ __forceinline__ void pick3(const double (&m)[3][3], int k, double o[3]) {
#pragma unroll
  for (int q = 0; q < 3; ++q)
    if (q == k)
      for (int c = 0; c < 3; ++c) o[c] = m[q][c];
}

__device__ void water_step_lanes(const IntegrateArgs& a, int w, int k, uint64_t step, int n,
                                 unsigned gmask) {
  const int4 idx = a.water[w];
  const int atom = k == 0 ? idx.x : k == 1 ? idx.y : idx.z;
  const double im[3] = {1.0 / a.geom.m_o, 1.0 / a.geom.m_h, 1.0 / a.geom.m_h};
  const double imk = k == 0 ? im[0] : im[1];
  double rk[3] = {0, 0, 0}, vk[3] = {0, 0, 0};
  StepTail tail{};
  double qk = 0.0;
  if (k < 3) {
    ld3(a.pos, atom, rk);
    ld3(a.vel, atom, vk);
    load_tail(a, atom, tail);
    if (a.posq) qk = a.qscaled[atom];
    double f[3];
    consume_force(a, n, atom, f);
    for (int c = 0; c < 3; ++c) vk[c] += f[c] * imk * a.dt;
  }
  double r[3][3], v[3][3], x[3][3];
  share3(r, rk, gmask);
  share3(v, vk, gmask);
  bool ok = settle_velocities(r, im, v);
  double xk[3] = {rk[0], rk[1], rk[2]};
  double wk[3] = {0, 0, 0};
  if (k < 3) {
    pick3(v, k, wk);
    ou_update(a, atom, imk, step, xk, wk);
  }
  share3(x, xk, gmask);
  ok = ok && settle_positions(a.geom, r, x);
  if (k == 3) return;
  const double inv_dt = 1.0 / a.dt;
  double xo[3];
  pick3(x, k, xo);
  for (int c = 0; c < 3; ++c) wk[c] += (xo[c] - xk[c]) * inv_dt;
  if (k == 0 && !ok) report_status(a.status, kStatusConstraint);
  if (!(finite3(xo) && finite3(wk))) report_status(a.status, kStatusNonfinite);
  st3(a.pos, atom, xo);
  st3(a.vel, atom, wk);
  write_packed(a, tail, qk, xo);
  check_rebuild(a, tail, xo);
}

__device__ void free_step(const IntegrateArgs& a, int atom, uint64_t step, int n) {
  const double im = a.inv_mass[atom];
  double x[3], v[3], f[3];
  ld3(a.pos, atom, x);
  ld3(a.vel, atom, v);
  StepTail tail{};
  load_tail(a, atom, tail);
  const double q = a.posq ? a.qscaled[atom] : 0.0;
  consume_force(a, n, atom, f);
  for (int c = 0; c < 3; ++c) v[c] += f[c] * im * a.dt;
  ou_update(a, atom, im, step, x, v);
  if (!(finite3(x) && finite3(v))) report_status(a.status, kStatusNonfinite);
  st3(a.pos, atom, x);
  st3(a.vel, atom, v);
  write_packed(a, tail, q, x);
  check_rebuild(a, tail, x);
}

// constraints.rs:81-156 restricted to one cluster.  `values` are positions (velocities=false,
// reference = start-of-step positions) or velocities (reference = current positions).  When
// `vel_from_pos` is set, every position correction is also added to the velocity / dt.
__device__ bool cluster_solve(const IntegrateArgs& a, int c, const double* reference,
                              double* values, bool velocities, double* vel_from_pos) {
  const int c0 = a.cluster_start[c], c1 = a.cluster_start[c + 1];
  for (int it = 0; it < 1000; ++it) {
    bool converged = true;
    for (int k = c0; k < c1; ++k) {
      const int i = a.cluster_pairs[k].x, j = a.cluster_pairs[k].y;
      const double wi = a.inv_mass[i], wj = a.inv_mass[j];
      double dir[3], delta[3];
      for (int q = 0; q < 3; ++q) {
        dir[q] = reference[3 * i + q] - reference[3 * j + q];
        delta[q] = values[3 * i + q] - values[3 * j + q];
      }
      const double dt = dot(delta, dir);
      double mult;
      if (velocities) {
        const double norm = dot(dir, dir);
        if (norm == 0.0 || !isfinite(norm)) return false;
        const double corr = -dt / ((wi + wj) * norm);
        if (fabs(corr) <= a.tolerance) continue;
        mult = corr;
      } else {
        const double norm = dot(delta, delta);
        const double ratio = sqrt(norm / a.cluster_dist2[k]);
        if (isfinite(ratio) && fabs(ratio - 1.0) <= a.tolerance) continue;
        const double den = 2.0 * (wi + wj) * dt;
        if (fabs(den) < 2.2250738585072014e-308 || !isfinite(den)) return false;
        mult = (a.cluster_dist2[k] - norm) / den;
      }
      if (!isfinite(mult)) return false;
      converged = false;
      for (int q = 0; q < 3; ++q) {
        const double corr = mult * dir[q];
        values[3 * i + q] += wi * corr;
        values[3 * j + q] -= wj * corr;
        if (vel_from_pos) {
          vel_from_pos[3 * i + q] += wi * corr / a.dt;
          vel_from_pos[3 * j + q] -= wj * corr / a.dt;
        }
      }
    }
    if (converged) return true;
  }
  return false;
}

__device__ void cluster_step(const IntegrateArgs& a, int c, uint64_t step, int n) {
  const int s0 = a.cluster_atom_start[c], s1 = a.cluster_atom_start[c + 1];
  for (int s = s0; s < s1; ++s) {
    const int atom = a.cluster_atoms[s];
    const double im = a.inv_mass[atom];
    double f[3];
    consume_force(a, n, atom, f);
    if (im == 0.0) continue;
    for (int q = 0; q < 3; ++q) a.vel[3 * atom + q] += f[q] * im * a.dt;
  }
  bool ok = cluster_solve(a, c, a.pos, a.vel, true, nullptr);
  for (int s = s0; s < s1; ++s) {
    const int atom = a.cluster_atoms[s];
    const double im = a.inv_mass[atom];
    double x[3], v[3];
    ld3(a.pos, atom, x);
    st3(a.scratch, atom, x);  // start-of-step reference
    if (im == 0.0) continue;
    ld3(a.vel, atom, v);
    ou_update(a, atom, im, step, x, v);
    st3(a.pos, atom, x);
    st3(a.vel, atom, v);
  }
  ok = ok && cluster_solve(a, c, a.scratch, a.pos, false, a.vel);
  if (!ok) report_status(a.status, kStatusConstraint);
  for (int s = s0; s < s1; ++s) {
    const int atom = a.cluster_atoms[s];
    double x[3], v[3];
    ld3(a.pos, atom, x);
    ld3(a.vel, atom, v);
    if (!(finite3(x) && finite3(v))) report_status(a.status, kStatusNonfinite);
    StepTail tail{};
    load_tail(a, atom, tail);
    write_packed(a, tail, a.posq ? a.qscaled[atom] : 0.0, x);
    check_rebuild(a, tail, x);
  }
}

__global__ void integrate_kernel(const IntegrateArgs a, int n) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t step = *a.rng_step + (uint64_t)a.step_offset;
  if (t < 4 * a.n_water) {
    const int lane = threadIdx.x & 31;
    water_step_lanes(a, t >> 2, t & 3, step, n, 0xFu << (lane & ~3));
    return;
  }
  t -= 4 * a.n_water;
  if (t < a.n_free) {
    free_step(a, a.free_atoms[t], step, n);
    return;
  }
  t -= a.n_free;
  if (t < a.n_clusters) cluster_step(a, t, step, n);
}

__global__ void constrain_positions_kernel(const IntegrateArgs a, const double* reference) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.n_water) {
    const int4 idx = a.water[t];
    const int at[3] = {idx.x, idx.y, idx.z};
    double r[3][3], x[3][3];
    for (int k = 0; k < 3; ++k) {
      ld3(reference, at[k], r[k]);
      ld3(a.pos, at[k], x[k]);
    }
    if (!settle_positions(a.geom, r, x)) {
      report_status(a.status, kStatusConstraint);
      return;
    }
    for (int k = 0; k < 3; ++k) st3(a.pos, at[k], x[k]);
    return;
  }
  t -= a.n_water + a.n_free;
  if (t >= 0 && t < a.n_clusters)
    if (!cluster_solve(a, t, reference, a.pos, false, nullptr)) report_status(a.status, kStatusConstraint);
}

__global__ void constrain_velocities_kernel(const IntegrateArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.n_water) {
    const int4 idx = a.water[t];
    const int at[3] = {idx.x, idx.y, idx.z};
    const double im[3] = {1.0 / a.geom.m_o, 1.0 / a.geom.m_h, 1.0 / a.geom.m_h};
    double x[3][3], v[3][3];
    for (int k = 0; k < 3; ++k) {
      ld3(a.pos, at[k], x[k]);
      ld3(a.vel, at[k], v[k]);
    }
    if (!settle_velocities(x, im, v)) {
      report_status(a.status, kStatusConstraint);
      return;
    }
    for (int k = 0; k < 3; ++k) st3(a.vel, at[k], v[k]);
    return;
  }
  t -= a.n_water + a.n_free;
  if (t >= 0 && t < a.n_clusters)
    if (!cluster_solve(a, t, a.pos, a.vel, true, nullptr)) report_status(a.status, kStatusConstraint);
}

__global__ void advance_kernel(unsigned long long* c, int by) { *c += (unsigned long long)by; }

// Barostat volume move (context.rs:976-1028): every position coordinate times `scale`, or
// (rigid) each molecule shifted by (scale - 1) times its centroid, the unweighted mean of its
// particles summed in molecule order.
__global__ void scale_positions_kernel(double* pos, int n_atoms, const int* mol_start,
                                       const int* mol_atoms, int n_molecules, double scale,
                                       int rigid) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!rigid) {
    if (t < 3 * n_atoms) pos[t] = scale * pos[t];
    return;
  }
  if (t >= n_molecules) return;
  const int a0 = mol_start[t], a1 = mol_start[t + 1];
  double c[3] = {0.0, 0.0, 0.0};
  for (int k = a0; k < a1; ++k)
    for (int d = 0; d < 3; ++d) c[d] += pos[3 * mol_atoms[k] + d];
  const double inv = 1.0 / (double)(a1 - a0);
  const double f = scale - 1.0;
  double off[3];
  for (int d = 0; d < 3; ++d) off[d] = f * (c[d] * inv);
  for (int k = a0; k < a1; ++k)
    for (int d = 0; d < 3; ++d) pos[3 * mol_atoms[k] + d] += off[d];
}

int threads_needed(const IntegrateArgs& a) { return a.n_water + a.n_free + a.n_clusters; }

}  // namespace

void launch_integrate(const IntegrateArgs& a, cudaStream_t s) {
  const int t = threads_needed(a) + 3 * a.n_water;  // four lanes per water
  if (t == 0) return;
  integrate_kernel<<<ceil_div(t, 128), 128, 0, s>>>(a, a.n_atoms);
}

void launch_scale_positions(double* pos, int n_atoms, const int* mol_start, const int* mol_atoms,
                            int n_molecules, double scale, bool rigid, cudaStream_t s) {
  const int n = rigid ? n_molecules : 3 * n_atoms;
  if (n <= 0) return;
  scale_positions_kernel<<<ceil_div(n, 128), 128, 0, s>>>(pos, n_atoms, mol_start, mol_atoms,
                                                         n_molecules, scale, rigid ? 1 : 0);
}

void launch_advance_counter(unsigned long long* counter, int by, cudaStream_t s) {
  advance_kernel<<<1, 1, 0, s>>>(counter, by);
}

void launch_constrain_positions(const IntegrateArgs& a, const double* reference, cudaStream_t s) {
  const int t = threads_needed(a);
  if (t == 0) return;
  constrain_positions_kernel<<<ceil_div(t, 128), 128, 0, s>>>(a, reference);
}

void launch_constrain_velocities(const IntegrateArgs& a, cudaStream_t s) {
  const int t = threads_needed(a);
  if (t == 0) return;
  constrain_velocities_kernel<<<ceil_div(t, 128), 128, 0, s>>>(a);
}

}  // namespace ommb200
