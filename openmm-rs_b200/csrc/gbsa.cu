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
#include <type_traits>

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

// Pass 2 in FP32 for non-periodic systems without a cutoff (the batched-chain workloads), with
// two i-particles per lane and packed (f32x2) arithmetic: lane m of each 16-lane half of the
// warp holds i-slots m and m + 16 of block I and meets the half's 16 entries of block J in 16
// steps, so a warp evaluates 64 pairs per step; the entry's force and dE/dR rotate within the
// half and are back at the entry's lane after the 16 steps, and the two halves' partial sums of
// each i-slot are added at the end (lane ^ 16).  Tiles whose every pair is a valid particle pair
// without exclusion take a loop without masks; self tiles (each pair seen from both sides, i
// sums only, half energy), padded and excluded tiles apply bit masks kept in step order.
template <bool kEnergy, bool kNb>
__global__ void __launch_bounds__(128) gb_pairs_x2(const GbArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ float4 s_pos[4][32];                // x, y, z, q sqrt|prefactor|
  __shared__ float2 s_born[4][32];               // R, 1 / R
  __shared__ float4 s_nb[kNb ? 4 : 1][32];       // q sqrt(ke), sigma / 2, 2 sqrt(eps), 0
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const float4* posq = reinterpret_cast<const float4*>(a.posq);
  const float2* born = reinterpret_cast<const float2*>(a.born_slot);
  const float4* nbp = reinterpret_cast<const float4*>(a.nb_params);
  const int m = lane & 15, eb = lane & 16, i1 = m, i2 = m + 16;
  const int src = eb | ((m + 1) & 15);
  const float sign = (float)a.prefactor_sign;
  for (int t = blockIdx.x * 4 + w; t < a.n_tiles; t += gridDim.x * 4) {
    const int2 tile = a.tiles[t];
    const int I = tile.x, J = tile.y;
    const bool self = I == J;
    const int ai = a.slot_atom[32 * I + lane], aj = a.slot_atom[32 * J + lane];
    s_pos[w][lane] = posq[32 * J + lane];
    s_born[w][lane] = born[32 * J + lane];
    uint32_t excl = 0u;
    if constexpr (kNb) {
      s_nb[w][lane] = nbp[32 * J + lane];
      const int4 nt = a.nb_tiles[t];
      if (nt.y & kTileHasMask) excl = a.nb_masks[32 * nt.z + lane];
    }
    const unsigned valid_i = __ballot_sync(FULL, ai >= 0), valid_j = __ballot_sync(FULL, aj >= 0);
    // step-ordered masks: bit k (i1) and 16 + k (i2) stand for entry eb + ((m + k) mod 16)
    auto rot = [&](uint32_t bits) {
      const uint32_t x = (bits >> eb) & 0xffffu;
      return ((x >> m) | (x << (16 - m))) & 0xffffu;
    };
    uint32_t use_bits, ex_bits = 0u;
    {
      const uint32_t vj = rot(valid_j);
      uint32_t u1 = ((valid_i >> i1) & 1u) ? vj : 0u, u2 = ((valid_i >> i2) & 1u) ? vj : 0u;
      if (self) {  // the diagonal: entry eb + m at step 0 is i1 (eb = 0) or i2 (eb = 16)
        u1 &= eb == 0 ? ~1u : ~0u;
        u2 &= eb == 16 ? ~1u : ~0u;
      }
      use_bits = u1 | (u2 << 16);
      if (kNb) ex_bits = rot(__shfl_sync(FULL, excl, i1)) | (rot(__shfl_sync(FULL, excl, i2)) << 16);
    }
    const bool plain = __all_sync(FULL, use_bits == 0xffffffffu && ex_bits == 0u);
    const float4 p1 = posq[32 * I + i1], p2 = posq[32 * I + i2];
    const float2 b1 = born[32 * I + i1], b2 = born[32 * I + i2];
    float4 n1 = make_float4(0.f, 0.f, 0.f, 0.f), n2 = n1;
    if (kNb) {
      n1 = nbp[32 * I + i1];
      n2 = nbp[32 * I + i2];
    }
    __syncwarp();
    const float2 npx = make_float2(-p1.x, -p2.x), npy = make_float2(-p1.y, -p2.y),
                 npz = make_float2(-p1.z, -p2.z);
    const float2 qn = make_float2(-sign * p1.w, -sign * p2.w);  // minus the GB charge factor
    const float2 Ri = make_float2(b1.x, b2.x), Rq = make_float2(0.25f * b1.y, 0.25f * b2.y);
    const float2 nq = make_float2(n1.x, n2.x), ns = make_float2(n1.y, n2.y),
                 ne = make_float2(n1.z, n2.z);
    float2 fx = x2::bc(0.f), fy = x2::bc(0.f), fz = x2::bc(0.f), acc_i = x2::bc(0.f);
    float fjx = 0.f, fjy = 0.f, fjz = 0.f, acc_j = 0.f;
    double e_gb = 0.0, e_nb = 0.0;
    double w_nb[6] = {0, 0, 0, 0, 0, 0};
    auto steps = [&](auto masked_tag) {
      constexpr bool kMasked = decltype(masked_tag)::value;
      uint32_t ub = use_bits;
      [[maybe_unused]] uint32_t xb = ex_bits;
#pragma unroll 2
      for (int k = 0; k < 16; ++k) {
        const int jl = eb | ((m + k) & 15);
        const float4 pj = s_pos[w][jl];
        const float2 bj = s_born[w][jl];
        const float2 dx = x2::add(x2::bc(pj.x), npx), dy = x2::add(x2::bc(pj.y), npy),
                     dz = x2::add(x2::bc(pj.z), npz);
        float2 r2 = x2::fma(dz, dz, x2::fma(dy, dy, x2::mul(dx, dx)));
        bool u1 = true, u2 = true;
        if (kMasked) {
          u1 = (ub & 1u) != 0u;
          u2 = (ub & 0x10000u) != 0u;
          ub >>= 1;
          r2 = x2::select(u1, u2, r2, 1.f);
        }
        // GB pair (gbsa_obc.rs:239-260): pe = -qn q_j / sqrt(r^2 + R_i R_j exp(-d)), d = r^2 / (4 R_i R_j)
        const float2 product = x2::mul(Ri, x2::bc(bj.x));
        const float2 d = x2::mul(r2, x2::mul(Rq, x2::bc(bj.y)));
        const float2 ex = x2::exp2_approx(x2::mul(x2::bc(-1.4426950408889634f), d));
        const float2 inv = x2::rsqrt_approx(x2::fma(product, ex, r2));
        const float2 pen = x2::mul(x2::mul(qn, x2::bc(pj.w)), inv);  // -pe
        const float2 pi2 = x2::mul(pen, x2::mul(inv, inv));          // -pe / den^2
        float2 fo = x2::mul(pi2, x2::fma(x2::bc(-0.25f), ex, x2::bc(1.f)));
        float2 bd = x2::mul(x2::mul(pi2, ex), x2::fma(d, x2::bc(0.5f), x2::bc(0.5f)));
        if (kEnergy) {
          const double sc = self ? 0.5 : 1.0;
          if (u1) e_gb -= sc * (double)pen.x;
          if (u2) e_gb -= sc * (double)pen.y;
        }
        if constexpr (kNb) {
          bool x1 = true, x2v = true;  // not excluded
          if (kMasked) {
            x1 = (xb & 1u) == 0u;
            x2v = (xb & 0x10000u) == 0u;
            xb >>= 1;
          }
          const float4 nj = s_nb[w][jl];
          const float2 inv_r = x2::rsqrt_approx(r2), inv_r2 = x2::mul(inv_r, inv_r);
          const float2 sig = x2::add(ns, x2::bc(nj.y));
          const float2 s2 = x2::mul(x2::mul(sig, sig), inv_r2);
          const float2 s6 = x2::mul(x2::mul(s2, s2), s2);
          const float2 eps4 = x2::mul(ne, x2::bc(nj.z));
          const float2 e6 = x2::mul(eps4, s6);
          float2 f_lj = x2::mul(x2::mul(e6, x2::fma(x2::bc(-12.f), s6, x2::bc(6.f))), inv_r2);
          if (eps4.x == 0.f) f_lj.x = 0.f;
          if (eps4.y == 0.f) f_lj.y = 0.f;
          const float2 qq = x2::mul(nq, x2::bc(nj.x));
          float2 f_nb = x2::sub(f_lj, x2::mul(x2::mul(qq, inv_r), inv_r2));
          if (kMasked) f_nb = x2::select(u1 && x1, u2 && x2v, f_nb, 0.f);
          if (kEnergy) {
            const double sc = self ? 0.5 : 1.0;
            const float2 e_lj = x2::mul(e6, x2::add(s6, x2::bc(-1.f)));
            const float2 e_el = x2::mul(qq, inv_r);
            const float2 fdx = x2::mul(f_nb, dx), fdy = x2::mul(f_nb, dy);
            const float2 wxx = x2::mul(fdx, dx), wyy = x2::mul(fdy, dy),
                         wzz = x2::mul(x2::mul(f_nb, dz), dz), wxy = x2::mul(fdx, dy),
                         wxz = x2::mul(fdx, dz), wyz = x2::mul(fdy, dz);
            for (int h = 0; h < 2; ++h) {
              if (!(h ? (u2 && x2v) : (u1 && x1))) continue;
              const float elj = h ? (eps4.y == 0.f ? 0.f : e_lj.y) : (eps4.x == 0.f ? 0.f : e_lj.x);
              e_nb += sc * ((double)elj + (double)(h ? e_el.y : e_el.x));
              w_nb[0] -= sc * (double)(h ? wxx.y : wxx.x);
              w_nb[1] -= sc * (double)(h ? wyy.y : wyy.x);
              w_nb[2] -= sc * (double)(h ? wzz.y : wzz.x);
              w_nb[3] -= sc * (double)(h ? wxy.y : wxy.x);
              w_nb[4] -= sc * (double)(h ? wxz.y : wxz.x);
              w_nb[5] -= sc * (double)(h ? wyz.y : wyz.x);
            }
          }
          fo = x2::add(fo, f_nb);
        }
        if (kMasked) {
          fo = x2::select(u1, u2, fo, 0.f);
          bd = x2::select(u1, u2, bd, 0.f);
        }
        fx = x2::fma(fo, dx, fx);
        fy = x2::fma(fo, dy, fy);
        fz = x2::fma(fo, dz, fz);
        acc_i = x2::fma(bd, x2::bc(bj.x), acc_i);
        if (!self) {
          fjx = fmaf(-fo.x, dx.x, fjx);
          fjy = fmaf(-fo.x, dy.x, fjy);
          fjz = fmaf(-fo.x, dz.x, fjz);
          acc_j = fmaf(bd.x, Ri.x, acc_j);
          fjx = fmaf(-fo.y, dx.y, fjx);
          fjy = fmaf(-fo.y, dy.y, fjy);
          fjz = fmaf(-fo.y, dz.y, fjz);
          acc_j = fmaf(bd.y, Ri.y, acc_j);
          fjx = __shfl_sync(FULL, fjx, src);
          fjy = __shfl_sync(FULL, fjy, src);
          fjz = __shfl_sync(FULL, fjz, src);
          acc_j = __shfl_sync(FULL, acc_j, src);
        }
      }
    };
    if (plain && !self)
      steps(std::false_type{});
    else
      steps(std::true_type{});
    // the two halves' sums of this lane's i-slots; the lane commits i-slot `lane`
    fx.x += __shfl_xor_sync(FULL, fx.x, 16);
    fx.y += __shfl_xor_sync(FULL, fx.y, 16);
    fy.x += __shfl_xor_sync(FULL, fy.x, 16);
    fy.y += __shfl_xor_sync(FULL, fy.y, 16);
    fz.x += __shfl_xor_sync(FULL, fz.x, 16);
    fz.y += __shfl_xor_sync(FULL, fz.y, 16);
    acc_i.x += __shfl_xor_sync(FULL, acc_i.x, 16);
    acc_i.y += __shfl_xor_sync(FULL, acc_i.y, 16);
    const bool second = eb != 0;
    const float fs = float(kForceScale);
    if (ai >= 0) {
      add_fixed(a.force + ai, to_fixed(second ? fx.y : fx.x, fs));
      add_fixed(a.force + a.n_atoms + ai, to_fixed(second ? fy.y : fy.x, fs));
      add_fixed(a.force + 2 * a.n_atoms + ai, to_fixed(second ? fz.y : fz.x, fs));
      add_fixed(a.dedr_sum + ai, to_fixed((double)(second ? acc_i.y : acc_i.x), kForceScale));
    }
    if (!self && aj >= 0) {
      add_fixed(a.force + aj, to_fixed(fjx, fs));
      add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fs));
      add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fs));
      add_fixed(a.dedr_sum + aj, to_fixed((double)acc_j, kForceScale));
    }
    if (kEnergy) {
      for (int off = 16; off > 0; off >>= 1) e_gb += __shfl_xor_sync(FULL, e_gb, off);
      const long long ef = to_fixed(e_gb, kEnergyScale);
      if (lane == 0 && ef) add_fixed(a.energy + 8 * a.block_segment[I], ef);
      if constexpr (kNb) {
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
      if (sizeof(Real) == 4 && !a.use_cutoff && !a.periodic) {
        if (a.fuse_nonbonded) {
          if (energy)
            gb_pairs_x2<true, true><<<gt, 128, 0, s>>>(a);
          else
            gb_pairs_x2<false, true><<<gt, 128, 0, s>>>(a);
        } else if (energy) {
          gb_pairs_x2<true, false><<<gt, 128, 0, s>>>(a);
        } else {
          gb_pairs_x2<false, false><<<gt, 128, 0, s>>>(a);
        }
      } else if (a.fuse_nonbonded) {
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
