// GBSAOBCForce (forces/gbsa_obc.rs:184-309): OBC-II Born radii from the HCT descreening
// integral, generalized-Born pair energy, ACE surface term.
//
// Three pair passes over 32 x 32 tiles of particle blocks, separated by per-particle f64
// kernels:
//   pass 1  I_i = sum_j H(r_ij; rho_i - 0.009, s_j (rho_j - 0.009))    (both directions)
//   radii   R_i = 1 / (1/(rho_i - 0.009) - tanh(psi - 0.8 psi^2 + 4.85 psi^3) / rho_i),
//           self and ACE energies, dE/dR_i from them
//   pass 2  GB pair energy, radial forces, dE/dR_i += dE_ij/dR_i
//   chain   dE/dR_i *= R_i^2 dR_i/dI_i
//   pass 3  forces from the descreening gradient
// The pair arithmetic runs in `Real` (FP32 in the mixed form); every sum over pairs is
// committed in 64-bit fixed point (descreening sums in 2^-40 nm^-1, dE/dR in 2^-32 kJ/mol/nm,
// forces in 2^-32 kJ/mol/nm), so results are bit-identical run to run.
//
// Tiles pair blocks of the same segment (one segment per independent system in a batch), so
// many systems of uneven size run in the same launches.
#include "kernels.h"
#include "gb_math.cuh"
#include "pair_math.cuh"

namespace ommb200 {
namespace {

using namespace gb;

// kNb (pass 2 only): the NoCutoff NonbondedForce pair terms (bare Coulomb + LJ 12-6 with the
// tile's exclusion mask, energy and virial as the nonbonded pair kernel computes them) join the
// GB pair term, sharing the distance, 1/r and the force rotation.  Pass 2 reads each slot's
// Born radius with its reciprocal, so r^2 / (4 R_i R_j) needs no division, and needs r itself
// only for the cutoff (kCutoff) and 1/r only for the nonbonded terms.
template <class Real, int kPass, bool kEnergy, bool kCutoff, bool kNb = false>
__global__ void __launch_bounds__(128) gb_pass(const GbArgs a) {
  if (kPass != 2 && a.use_learned && *a.use_learned) return;  // the network replaces them
  using T4 = typename V4<Real>::T4;
  using T2 = typename V4<Real>::T2;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ T4 s_pos[4][32];
  __shared__ T2 s_par[4][32];
  __shared__ Real s_aux[4][32];
  __shared__ T2 s_born[kPass == 2 ? 4 : 1][32];  // pass 2: R, 1 / R
  __shared__ T4 s_nb[kNb ? 4 : 1][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const T4* posq = reinterpret_cast<const T4*>(a.posq);
  const T2* par = reinterpret_cast<const T2*>(a.params);
  const T2* born = reinterpret_cast<const T2*>(a.born_slot);
  const Real* dedr = reinterpret_cast<const Real*>(a.dedr_slot);
  for (int t = blockIdx.x * 4 + w; t < a.n_tiles; t += gridDim.x * 4) {
    const int2 tile = a.tiles[t];
    const int I = tile.x, J = tile.y;
    const bool self = I == J;
    const int si = 32 * I + lane, sj = 32 * J + lane;
    const int ai = a.slot_atom[si], aj = a.slot_atom[sj];
    const T4 pi = posq[si];
    const T2 qi = par[si];  // (offset radius, scaled radius)
    Real ri_aux = Real(0);
    T2 bi;
    bi.x = bi.y = Real(1);
    if (kPass == 2) {
      bi = born[si];
      s_born[w][lane] = born[sj];
    } else {
      s_par[w][lane] = par[sj];
    }
    if (kPass == 3) {
      ri_aux = dedr[si];
      s_aux[w][lane] = dedr[sj];
    }
    s_pos[w][lane] = posq[sj];
    T4 nbi;
    uint32_t excl = 0u;
    if constexpr (kNb) {
      const T4* nbp = reinterpret_cast<const T4*>(a.nb_params);
      nbi = nbp[si];
      s_nb[w][lane] = nbp[sj];
      const int4 nt = a.nb_tiles[t];
      if (nt.y & kTileHasMask) excl = a.nb_masks[32 * nt.z + lane];
    }
    const unsigned valid_j = __ballot_sync(FULL, aj >= 0);  // entries holding a particle
    const Real qsi = (Real)a.prefactor_sign * pi.w;
    __syncwarp();
    Real acc_i = 0, acc_j = 0;  // pass 1: descreening sums; pass 2: dE/dR
    Real fix = 0, fiy = 0, fiz = 0, fjx = 0, fjy = 0, fjz = 0;
    double e_tile = 0.0, e_nb = 0.0;
    double w_nb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int k = self ? 1 : 0; k < 32; ++k) {
      const int jl = (lane + k) & 31;
      const T4 pj = s_pos[w][jl];
      Real dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
      if (a.periodic) {
        if constexpr (sizeof(Real) == 4) min_image_fast(dx, dy, dz, a.boxf);
        else min_image_fast(dx, dy, dz, a.boxd);
      }
      const Real r2 = dx * dx + dy * dy + dz * dz;
      bool use = ai >= 0 && ((valid_j >> jl) & 1u);
      Real r = Real(1), inv_r = Real(1);
      if (kPass != 2 || kCutoff || kNb) {
        if constexpr (sizeof(Real) == 4) {  // SFU reciprocal square root in the FP32 kernel
          inv_r = rsqrt_r(use ? r2 : Real(1));
          r = (use ? r2 : Real(1)) * inv_r;
        } else {
          r = sqrt_r(use ? r2 : Real(1));
          inv_r = Real(1) / r;
        }
      }
      if (kCutoff) use = use && r <= (Real)a.cutoff;  // gbsa_obc.rs:169 (<=)
      Real fo = 0;
      if (kPass == 1) {
        if (use) {
          const T2 qj = s_par[w][jl];
          acc_i += descreening_pair(qi.x, qj.y, r, inv_r);
          if (!self) acc_j += descreening_pair(qj.x, qi.y, r, inv_r);
        }
      } else if (kPass == 2) {
        if (use) {
          // SFU forms (ex2, rsqrt) in the FP32 kernel, exact ones in FP64
          const T2 bj = s_born[w][jl];
          const Real product = bi.x * bj.x;
          const Real d = Real(0.25) * r2 * (bi.y * bj.y);
          const Real ex = exp2_r(Real(-1.4426950408889634) * d);
          const Real den2 = r2 + product * ex;
          const Real inv = rsqrt_r(den2), inv2 = inv * inv;
          // prefactor q_i q_j, with q stored as q sqrt|prefactor|
          const Real coefficient = qsi * pj.w;
          const Real pe = coefficient * inv;
          fo = -pe * (Real(1) - Real(0.25) * ex) * inv2;
          const Real bd = Real(-0.5) * pe * ex * (Real(1) + d) * inv2;
          acc_i += bd * bj.x;
          if (!self) acc_j += bd * bi.x;
          if (kEnergy) {
            const double e = kCutoff ? (double)pe - (double)coefficient / a.cutoff : (double)pe;
            e_tile += (self ? 0.5 : 1.0) * e;
          }
        }
        if constexpr (kNb) {
          if (use && ((excl >> jl) & 1u) == 0u) {
            const T4 nbj = s_nb[w][jl];
            PairArgs<Real> none{};
            Real f_nb, en_nb;
            pair_terms_r<Real, kElecCoulomb, kEnergy, false>(none, r2, inv_r, nbi.x * nbj.x,
                                                             nbi.y + nbj.y, nbi.z * nbj.z, f_nb,
                                                             en_nb);
            fo += f_nb;
            if (kEnergy) {
              const double scale = self ? 0.5 : 1.0;
              e_nb += scale * (double)en_nb;
              w_nb[0] -= scale * (double)(f_nb * dx * dx);
              w_nb[1] -= scale * (double)(f_nb * dy * dy);
              w_nb[2] -= scale * (double)(f_nb * dz * dz);
              w_nb[3] -= scale * (double)(f_nb * dx * dy);
              w_nb[4] -= scale * (double)(f_nb * dx * dz);
              w_nb[5] -= scale * (double)(f_nb * dy * dz);
            }
          }
        }
      } else {
        if (use) {
          const T2 qj = s_par[w][jl];
          const Real rj_aux = s_aux[w][jl];
          fo = -(ri_aux * descreening_gradient_pair(qi.x, qj.y, r, inv_r) +
                 rj_aux * descreening_gradient_pair(qj.x, qi.y, r, inv_r));
        }
      }
      if (kPass != 1) {
        // self tiles visit each pair from both sides; each visit moves only its own lane
        fix = fma(fo, dx, fix);
        fiy = fma(fo, dy, fiy);
        fiz = fma(fo, dz, fiz);
      }
      if (!self) {
        const int src = (lane + 1) & 31;
        if (kPass != 1) {
          fjx = fma(-fo, dx, fjx);
          fjy = fma(-fo, dy, fjy);
          fjz = fma(-fo, dz, fjz);
          fjx = __shfl_sync(FULL, fjx, src);
          fjy = __shfl_sync(FULL, fjy, src);
          fjz = __shfl_sync(FULL, fjz, src);
        }
        if (kPass != 3) acc_j = __shfl_sync(FULL, acc_j, src);
      }
    }
    if (kPass == 1) {
      if (ai >= 0) add_fixed(a.born_sum + ai, to_fixed((double)acc_i, kBornScale));
      if (!self && aj >= 0) add_fixed(a.born_sum + aj, to_fixed((double)acc_j, kBornScale));
    } else {
      const Real fs = Real(kForceScale);
      if (ai >= 0) {
        add_fixed(a.force + ai, to_fixed(fix, fs));
        add_fixed(a.force + a.n_atoms + ai, to_fixed(fiy, fs));
        add_fixed(a.force + 2 * a.n_atoms + ai, to_fixed(fiz, fs));
      }
      if (!self && aj >= 0) {
        add_fixed(a.force + aj, to_fixed(fjx, fs));
        add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fs));
        add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fs));
      }
      if (kPass == 2) {
        if (ai >= 0) add_fixed(a.dedr_sum + ai, to_fixed((double)acc_i, kForceScale));
        if (!self && aj >= 0) add_fixed(a.dedr_sum + aj, to_fixed((double)acc_j, kForceScale));
      }
    }
    if (kEnergy && kPass == 2) {
      for (int off = 16; off > 0; off >>= 1) e_tile += __shfl_xor_sync(FULL, e_tile, off);
      const long long ef = to_fixed(e_tile, kEnergyScale);
      if (lane == 0 && ef) add_fixed(a.energy + 8 * a.block_segment[I], ef);
      if constexpr (kNb) {  // rounded per tile on its own, as the nonbonded pair kernel does
        for (int off = 16; off > 0; off >>= 1) {
          e_nb += __shfl_xor_sync(FULL, e_nb, off);
          for (int c = 0; c < 6; ++c) w_nb[c] += __shfl_xor_sync(FULL, w_nb[c], off);
        }
        if (lane == 0) {
          long long* dst = a.energy + 8 * a.block_segment[I];
          add_fixed(dst, to_fixed(e_nb, kEnergyScale));
          for (int c = 0; c < 6; ++c) add_fixed(dst + 1 + c, to_fixed(w_nb[c], kEnergyScale));
        }
      }
    }
    __syncwarp();
  }
}

// gbsa_obc.rs:214-237: radii, chain factor, self + ACE energies, dE/dR from them.
template <class Real, bool kEnergy>
__global__ void gb_radii(const GbArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_slots) return;
  const int atom = a.slot_atom[s];
  typename V4<Real>::T2* born = reinterpret_cast<typename V4<Real>::T2*>(a.born_slot);
  if (atom < 0) {
    born[s].x = born[s].y = Real(1);
    return;
  }
  const double rho = a.radius[atom];
  const double offset = rho - kDielectricOffset;
  const double integral = (a.use_learned && *a.use_learned)
                              ? (double)a.short_sum[atom] * kBornScaleInv + (double)a.tail[atom] +
                                    (double)a.seg_offset[a.atom_segment[atom]]
                              : (double)a.born_sum[atom] * kBornScaleInv;
  const double psi = 0.5 * offset * integral;
  const double t = tanh(psi - 0.8 * psi * psi + 4.85 * psi * psi * psi);
  const double R = 1.0 / (1.0 / offset - t / rho);
  a.chain[atom] = offset * (1.0 - 1.6 * psi + 14.55 * psi * psi) * (1.0 - t * t) / rho;
  a.born_radius[atom] = R;
  born[s].x = (Real)R;
  born[s].y = (Real)(1.0 / R);
  const double q = a.charge[atom];
  const double self_energy = 0.5 * a.prefactor * q * q / fabs(R);
  double dedr = -self_energy / R;
  double e = self_energy;
  if (R > 0.0) {
    const double ratio = rho / R;
    const double r2 = ratio * ratio;
    const double area = a.surface * (rho + kProbeRadius) * (rho + kProbeRadius) * r2 * r2 * r2;
    e += area;
    dedr -= 6.0 * area / R;
  }
  a.dedr_self[atom] = dedr;
  if (kEnergy) add_fixed(a.energy + 8 * a.atom_segment[atom], to_fixed(e, kEnergyScale));
}

// gbsa_obc.rs:261-263
template <class Real>
__global__ void gb_chain(const GbArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_slots) return;
  const int atom = a.slot_atom[s];
  Real* dedr = reinterpret_cast<Real*>(a.dedr_slot);
  if (atom < 0) {
    dedr[s] = Real(0);
    return;
  }
  const double R = a.born_radius[atom];
  const double total = a.dedr_self[atom] + (double)a.dedr_sum[atom] * kForceScaleInv;
  dedr[s] = (Real)(total * R * R * a.chain[atom]);
}

template <class Real>
__global__ void gb_pack(const GbArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_slots) return;
  const int atom = a.slot_atom[s];
  typename V4<Real>::T4 p;
  typename V4<Real>::T2 q;
  if (atom < 0) {
    p.x = p.y = p.z = p.w = Real(0);
    q.x = q.y = Real(0);
  } else {
    p.x = (Real)a.pos[3 * atom];
    p.y = (Real)a.pos[3 * atom + 1];
    p.z = (Real)a.pos[3 * atom + 2];
    p.w = (Real)(a.charge[atom] * a.charge_scale);
    a.born_sum[atom] = 0;
    a.dedr_sum[atom] = 0;
    const double offset = a.radius[atom] - kDielectricOffset;
    q.x = (Real)offset;
    q.y = (Real)(offset * a.scale[atom]);
  }
  reinterpret_cast<typename V4<Real>::T4*>(a.posq)[s] = p;
  reinterpret_cast<typename V4<Real>::T2*>(a.params)[s] = q;
  if (a.nb_params) {
    typename V4<Real>::T4 nb;
    nb.x = nb.y = nb.z = nb.w = Real(0);
    if (atom >= 0) {
      nb.x = (Real)a.nb_charge[atom];
      nb.y = (Real)a.nb_half_sigma[atom];
      nb.z = (Real)a.nb_two_sqrt_eps[atom];
    }
    reinterpret_cast<typename V4<Real>::T4*>(a.nb_params)[s] = nb;
  }
}

}  // namespace

template <class Real, int kPass, bool kEnergy, bool kNb = false>
void launch_gb_pass(const GbArgs& a, int grid, cudaStream_t s) {
  if (a.use_cutoff)
    gb_pass<Real, kPass, kEnergy, true, kNb><<<grid, 128, 0, s>>>(a);
  else
    gb_pass<Real, kPass, kEnergy, false, kNb><<<grid, 128, 0, s>>>(a);
}

template <class Real>
void launch_gbsa_phase(const GbArgs& a, int phase, bool energy, int sm_count, cudaStream_t s) {
  const int tb = 256;
  const int gs = ceil_div(a.n_slots, tb);
  const int gt = (int)std::min<long long>((a.n_tiles + 3) / 4, (long long)sm_count * 16);
  switch (phase) {
    case kGbPack:
      gb_pack<Real><<<gs, tb, 0, s>>>(a);
      break;
    case kGbPass1:
      launch_gb_pass<Real, 1, false>(a, gt, s);
      break;
    case kGbRadii:
      if (energy)
        gb_radii<Real, true><<<gs, tb, 0, s>>>(a);
      else
        gb_radii<Real, false><<<gs, tb, 0, s>>>(a);
      break;
    case kGbPass2:
      if (a.fuse_nonbonded) {
        if (energy)
          launch_gb_pass<Real, 2, true, true>(a, gt, s);
        else
          launch_gb_pass<Real, 2, false, true>(a, gt, s);
      } else if (energy) {
        launch_gb_pass<Real, 2, true>(a, gt, s);
      } else {
        launch_gb_pass<Real, 2, false>(a, gt, s);
      }
      break;
    case kGbChain:
      gb_chain<Real><<<gs, tb, 0, s>>>(a);
      break;
    case kGbPass3:
      launch_gb_pass<Real, 3, false>(a, gt, s);
      break;
  }
}

template void launch_gbsa_phase<float>(const GbArgs&, int, bool, int, cudaStream_t);
template void launch_gbsa_phase<double>(const GbArgs&, int, bool, int, cudaStream_t);

}  // namespace ommb200
