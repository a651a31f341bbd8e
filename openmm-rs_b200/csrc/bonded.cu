// Exceptions (forces/nonbonded.rs:995-1036, 1194-1198, 1275-1288) and harmonic bonds/angles
// (forces/harmonic_bond.rs:102-144, forces/harmonic_angle.rs:102-175), in f64: these are the
// PME exclusion corrections, which cancel large reciprocal-space terms and so keep f64.
#include "kernels.h"

namespace ommb200 {
namespace {

__device__ __forceinline__ void commit_pair(long long* force, int n, int i, int j, double fo,
                                            const double d[3]) {
  for (int c = 0; c < 3; ++c) {
    const long long v = to_fixed(fo * d[c], kForceScale);
    add_fixed(force + (long long)c * n + i, v);
    add_fixed(force + (long long)c * n + j, -v);
  }
}

// `seg`: the term's system in a batch (energy at energy[8 * seg]), or -1 for a single
// system, whose warp sums are committed once.
__device__ __forceinline__ void reduce_commit(long long* energy, double e, const double w[6],
                                              int seg) {
  if (seg >= 0) {
    long long* dst = energy + 8 * seg;
    const long long ef = to_fixed(e, kEnergyScale);
    if (ef) add_fixed(dst, ef);
    for (int c = 0; c < 6; ++c) {
      const long long wf = to_fixed(w[c], kEnergyScale);
      if (wf) add_fixed(dst + 1 + c, wf);
    }
    return;
  }
  long long ef = to_fixed(e, kEnergyScale);
  long long wf[6];
  for (int c = 0; c < 6; ++c) wf[c] = to_fixed(w[c], kEnergyScale);
  for (int off = 16; off > 0; off >>= 1) {
    ef += __shfl_xor_sync(0xffffffffu, ef, off);
    for (int c = 0; c < 6; ++c) wf[c] += __shfl_xor_sync(0xffffffffu, wf[c], off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (ef) add_fixed(energy, ef);
    for (int c = 0; c < 6; ++c)
      if (wf[c]) add_fixed(energy + 1 + c, wf[c]);
  }
}

__device__ __forceinline__ void pair_virial(double w[6], double fo, const double d[3]) {
  w[0] -= fo * d[0] * d[0];
  w[1] -= fo * d[1] * d[1];
  w[2] -= fo * d[2] * d[2];
  w[3] -= fo * d[0] * d[1];
  w[4] -= fo * d[0] * d[2];
  w[5] -= fo * d[1] * d[2];
}

template <bool kEnergy>
__global__ void exceptions_kernel(const ExceptionArgs a, int n_atoms) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double en = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  int seg = a.atom_segment ? 0 : -1;
  if (e < a.n) {
    const int2 p = a.pairs[e];
    if (a.atom_segment) seg = a.atom_segment[p.x];
    const double4 prm = a.params[e];
    double d[3] = {a.pos[3 * p.y] - a.pos[3 * p.x], a.pos[3 * p.y + 1] - a.pos[3 * p.x + 1],
                   a.pos[3 * p.y + 2] - a.pos[3 * p.x + 2]};
    if (a.use_pbc) min_image_exact(d[0], d[1], d[2], a.box);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r = sqrt(r2);
    double ee = 0.0, fo = 0.0;
    if (prm.z != 0.0) {  // lj_pair
      const double sr2 = prm.y * prm.y / r2;
      const double sr6 = sr2 * sr2 * sr2;
      ee += 4.0 * prm.z * (sr6 * sr6 - sr6);
      fo += 4.0 * prm.z * (-12.0 * sr6 * sr6 + 6.0 * sr6) / r2;
    }
    if (prm.x != 0.0) {  // coulomb_pair
      ee += prm.x / r;
      fo += -prm.x / (r2 * r);
    }
    if (a.ewald) {  // reciprocal_pair
      const double qq = prm.w;
      double ce, cf;
      if (a.alpha * r < 1e-6) {
        ce = qq * 2.0 * a.alpha / sqrt(kPiD) * (1.0 - a.alpha * a.alpha * r2 / 3.0);
        cf = -qq * 4.0 * a.alpha * a.alpha * a.alpha / (3.0 * sqrt(kPiD));
      } else {
        const double ef = erf(a.alpha * r);
        ce = qq * ef / r;
        cf = qq * (2.0 * a.alpha / sqrt(kPiD) * exp(-a.alpha * a.alpha * r2) - ef / r) / r2;
      }
      ee -= ce;
      fo -= cf;
    }
    commit_pair(a.force, n_atoms, p.x, p.y, fo, d);
    if (kEnergy) {
      en = ee;
      pair_virial(w, fo, d);
    }
  }
  if (kEnergy) reduce_commit(a.energy, en, w, seg);
}

template <bool kEnergy>
__global__ void bonded_kernel(const BondedArgs a, int n_atoms) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double en = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  int seg = a.atom_segment ? 0 : -1;
  if (t < a.n_bonds) {
    const int2 b = a.bonds[t];
    if (a.atom_segment) seg = a.atom_segment[b.x];
    const double2 prm = a.bond_params[t];
    double d[3] = {a.pos[3 * b.y] - a.pos[3 * b.x], a.pos[3 * b.y + 1] - a.pos[3 * b.x + 1],
                   a.pos[3 * b.y + 2] - a.pos[3 * b.x + 2]};
    if (a.bond_pbc) min_image_exact(d[0], d[1], d[2], a.box);
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double dr = r - prm.x;
    const double fm = prm.y * dr / r;
    commit_pair(a.force, n_atoms, b.x, b.y, fm, d);
    if (kEnergy) {
      en = 0.5 * prm.y * dr * dr;
      pair_virial(w, fm, d);
    }
  } else if (t < a.n_bonds + a.n_angles) {
    const int4 an = a.angles[t - a.n_bonds];
    const double2 prm = a.angle_params[t - a.n_bonds];
    const int i = an.x, j = an.y, k = an.z;
    if (a.atom_segment) seg = a.atom_segment[j];
    double rji[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1],
                     a.pos[3 * i + 2] - a.pos[3 * j + 2]};
    double rjk[3] = {a.pos[3 * k] - a.pos[3 * j], a.pos[3 * k + 1] - a.pos[3 * j + 1],
                     a.pos[3 * k + 2] - a.pos[3 * j + 2]};
    if (a.angle_pbc) {
      min_image_exact(rji[0], rji[1], rji[2], a.box);
      min_image_exact(rjk[0], rjk[1], rjk[2], a.box);
    }
    const double li = sqrt(rji[0] * rji[0] + rji[1] * rji[1] + rji[2] * rji[2]);
    const double lk = sqrt(rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
    double c = (rji[0] * rjk[0] + rji[1] * rjk[1] + rji[2] * rjk[2]) / (li * lk);
    c = fmin(fmax(c, -1.0), 1.0);
    const double theta = acos(c);
    const double dtheta = theta - prm.x;
    const double s = fmax(sqrt(1.0 - c * c), 1e-8);
    const double de = prm.y * dtheta;
    for (int d = 0; d < 3; ++d) {
      const double fi = de * (c * rji[d] / li - rjk[d] / lk) / (li * s);
      const double fk = de * (c * rjk[d] / lk - rji[d] / li) / (lk * s);
      const long long vi = to_fixed(fi, kForceScale), vk = to_fixed(fk, kForceScale);
      add_fixed(a.force + (long long)d * n_atoms + i, -vi);
      add_fixed(a.force + (long long)d * n_atoms + k, -vk);
      add_fixed(a.force + (long long)d * n_atoms + j, vi + vk);
      if (kEnergy) {
        // W_ab = sum_atoms F_a r_b, positions relative to the vertex
        if (d == 0) {
          w[0] += -fi * rji[0] - fk * rjk[0];
          w[3] += -fi * rji[1] - fk * rjk[1];
          w[4] += -fi * rji[2] - fk * rjk[2];
        } else if (d == 1) {
          w[1] += -fi * rji[1] - fk * rjk[1];
          w[5] += -fi * rji[2] - fk * rjk[2];
        } else {
          w[2] += -fi * rji[2] - fk * rjk[2];
        }
      }
    }
    if (kEnergy) en = 0.5 * prm.y * dtheta * dtheta;
  }
  if (kEnergy) reduce_commit(a.energy, en, w, seg);
}

}  // namespace

void launch_exceptions(const ExceptionArgs& a, bool energy, cudaStream_t s) {
  if (a.n == 0) return;
  const int n_atoms = a.n_atoms_for_force;
  if (energy)
    exceptions_kernel<true><<<ceil_div(a.n, 128), 128, 0, s>>>(a, n_atoms);
  else
    exceptions_kernel<false><<<ceil_div(a.n, 128), 128, 0, s>>>(a, n_atoms);
}

void launch_bonded(const BondedArgs& a, bool energy, cudaStream_t s) {
  const int total = a.n_bonds + a.n_angles;
  if (total == 0) return;
  if (energy)
    bonded_kernel<true><<<ceil_div(total, 128), 128, 0, s>>>(a, a.n_atoms_for_force);
  else
    bonded_kernel<false><<<ceil_div(total, 128), 128, 0, s>>>(a, a.n_atoms_for_force);
}

}  // namespace ommb200
