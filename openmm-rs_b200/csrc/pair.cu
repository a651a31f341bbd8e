// Real-space nonbonded pair kernel: LJ 12-6 (Lorentz-Berthelot, optional switching) plus
// Ewald-screened, reaction-field or bare Coulomb, following forces/nonbonded.rs:842-924 and
// the pair functions at nonbonded.rs:1194-1288.
//
// One warp evaluates one 32x32 tile.  Lane l owns i-particle l of block I; the j-particles
// of block J start in lane l and rotate one lane per step (warp shuffles) together with the
// force they accumulate, so after 32 steps every (i, j) pair was seen once and each j-force
// is back in its own lane.  Diagonal tiles (I == J) read partners by shuffle and keep only
// i-forces, visiting each pair twice at half energy.  Forces are summed in `Real` within the
// tile and committed as 64-bit fixed point, which makes the total independent of tile order.
//
// Pair membership reproduces the reference exactly: pairs whose squared distance falls
// within `band` of rc^2 are re-decided from the f64 master positions with the reference's
// minimum-image and r^2 < rc^2 arithmetic (explicitly rounded, no fused multiply-add).
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

__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float exp_r(float x) { return __expf(x); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float erfc_r(float x, float ex) { return erfc_fit(x, ex); }
__device__ __forceinline__ double erfc_r(double x, double) { return erfc(x); }

// The reference's cutoff decision for particles a, b (original indices).
__device__ __noinline__ bool exact_inside(const double* pos, int a, int b, int periodic,
                                          const Box<double>& box, double rc2) {
  const int i = a < b ? a : b, j = a < b ? b : a;
  double dx = __dsub_rn(pos[3 * j], pos[3 * i]);
  double dy = __dsub_rn(pos[3 * j + 1], pos[3 * i + 1]);
  double dz = __dsub_rn(pos[3 * j + 2], pos[3 * i + 2]);
  if (periodic) min_image_exact(dx, dy, dz, box);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return r2 < rc2;
}

template <class Real, int kElec, bool kEnergy>
struct PairResult {
  Real f_over_r;  // dE/dr / r
  Real energy;
};

template <class Real, int kElec, bool kEnergy>
__device__ __forceinline__ PairResult<Real, kElec, kEnergy> pair_terms(
    const PairArgs<Real>& a, Real r2, Real qq, Real sig, Real eps) {
  const Real inv_r = rsqrt_r(r2);
  const Real inv_r2 = inv_r * inv_r;
  // LJ 12-6 (nonbonded.rs:1203-1214)
  const Real s2 = sig * sig * inv_r2;
  const Real s6 = s2 * s2 * s2;
  const Real eps4 = Real(4) * eps;
  Real f_lj = eps4 * (Real(6) * s6 - Real(12) * s6 * s6) * inv_r2;
  Real e_lj = eps4 * (s6 * s6 - s6);
  if (eps == Real(0)) {
    f_lj = Real(0);
    e_lj = Real(0);
  }
  // switching (nonbonded.rs:888-900)
  if (a.use_switching) {
    const Real r = r2 * inv_r;
    if (r > a.switch_r) {
      const Real t = (r - a.switch_r) * a.switch_inv_width;
      const Real sw = Real(1) + t * t * t * (Real(-10) + t * (Real(15) - Real(6) * t));
      const Real dsw = Real(-30) * t * t * (Real(1) - t) * (Real(1) - t) * a.switch_inv_width;
      f_lj = sw * f_lj + e_lj * dsw * inv_r;
      e_lj *= sw;
    }
  }
  Real f_el, e_el;
  if (kElec == kElecEwald) {
    // screened_coulomb (nonbonded.rs:1263-1273)
    const Real r = r2 * inv_r;
    const Real ex = exp_r(-a.alpha2 * r2);
    const Real ec = erfc_r(a.alpha * r, ex);
    e_el = qq * ec * inv_r;
    f_el = -qq * (ec * inv_r + a.two_alpha_sqrtpi * ex) * inv_r2;
  } else if (kElec == kElecReactionField) {
    // reaction_field (nonbonded.rs:1222-1243)
    e_el = qq * (inv_r + a.krf * r2 - a.crf);
    f_el = qq * (Real(2) * a.krf - inv_r * inv_r2);
  } else {
    // coulomb_pair (nonbonded.rs:1186-1192)
    e_el = qq * inv_r;
    f_el = -qq * inv_r * inv_r2;
  }
  PairResult<Real, kElec, kEnergy> res;
  res.f_over_r = f_lj + f_el;
  res.energy = kEnergy ? e_lj + e_el : Real(0);
  return res;
}

template <class Real, int kElec, bool kEnergy, bool kDump>
__global__ void __launch_bounds__(128) pair_kernel(const PairArgs<Real> a) {
  using T4 = typename V4<Real>::T4;
  using T2 = typename V4<Real>::T2;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nt = min(*a.n_tiles, a.tile_capacity);
  const T4* posq = reinterpret_cast<const T4*>(a.posq);
  const T2* ljp = reinterpret_cast<const T2*>(a.ljp);
  const T4* shifts = reinterpret_cast<const T4*>(a.tile_shift);
  long long e_fixed = 0;
  long long w_fixed[6] = {0, 0, 0, 0, 0, 0};

  for (int t = warp; t < nt; t += nwarps) {
    const int4 tile = a.tiles[t];
    const int I = tile.x, J = tile.y;
    const int si = 32 * I + lane, sj = 32 * J + lane;
    const T4 pi = posq[si];
    const T2 li = ljp[si];
    T4 pj = posq[sj];
    T2 lj = ljp[sj];
    const T4 sh = shifts[t];
    pj.x += sh.x;
    pj.y += sh.y;
    pj.z += sh.z;
    const uint32_t excl = (tile.z & kTileHasMask) ? a.masks[32 * tile.w + lane] : 0u;
    const bool pair_image = (tile.z & kTilePairImage) != 0;
    const int ai = a.sorted_atom[si];
    Real fix = 0, fiy = 0, fiz = 0, fjx = 0, fjy = 0, fjz = 0;
    double e_tile = 0.0;
    double w_tile[6] = {0, 0, 0, 0, 0, 0};
    const bool diag = (I == J);
    for (int k = diag ? 1 : 0; k < 32; ++k) {
      const int jl = (lane + k) & 31;
      Real xj, yj, zj, qj, sj_, ej;
      if (diag) {
        xj = __shfl_sync(FULL, pj.x, jl);
        yj = __shfl_sync(FULL, pj.y, jl);
        zj = __shfl_sync(FULL, pj.z, jl);
        qj = __shfl_sync(FULL, pj.w, jl);
        sj_ = __shfl_sync(FULL, lj.x, jl);
        ej = __shfl_sync(FULL, lj.y, jl);
      } else {
        xj = pj.x;
        yj = pj.y;
        zj = pj.z;
        qj = pj.w;
        sj_ = lj.x;
        ej = lj.y;
      }
      Real dx = xj - pi.x, dy = yj - pi.y, dz = zj - pi.z;
      if (pair_image) min_image_fast(dx, dy, dz, a.box);
      Real r2 = dx * dx + dy * dy + dz * dz;
      bool use = ((excl >> jl) & 1u) == 0u;
      if (a.use_cutoff && use) {
        bool inside = r2 < a.cutoff2;
        if (fabs(r2 - a.cutoff2) < a.band) {
          const int aj = a.sorted_atom[32 * J + jl];
          inside = ai >= 0 && aj >= 0 &&
                   exact_inside(a.pos, ai, aj, a.periodic, a.box_exact, a.cutoff2_exact);
        }
        use = inside;
      }
      const int aj_dump = kDump ? a.sorted_atom[32 * J + jl] : 0;
      if (kDump && use && ai >= 0 && aj_dump >= 0 && (!diag || ai < aj_dump)) {
        const int aj = aj_dump;
        const unsigned long long slot = atomicAdd(a.pair_count, 1ull);
        if ((long long)slot < a.pair_capacity) {
          a.pair_dump[2 * slot] = ai < aj ? ai : aj;
          a.pair_dump[2 * slot + 1] = ai < aj ? aj : ai;
        }
      }
      if (!use) r2 = Real(1);
      const auto res = pair_terms<Real, kElec, kEnergy>(a, r2, pi.w * qj, li.x + sj_, li.y * ej);
      const Real fo = use ? res.f_over_r : Real(0);
      const Real fx = fo * dx, fy = fo * dy, fz = fo * dz;
      fix += fx;
      fiy += fy;
      fiz += fz;
      if (kEnergy && use) {
        const double scale = diag ? 0.5 : 1.0;
        e_tile += scale * (double)res.energy;
        w_tile[0] -= scale * (double)(fx * dx);
        w_tile[1] -= scale * (double)(fy * dy);
        w_tile[2] -= scale * (double)(fz * dz);
        w_tile[3] -= scale * (double)(fx * dy);
        w_tile[4] -= scale * (double)(fx * dz);
        w_tile[5] -= scale * (double)(fy * dz);
      }
      if (!diag) {
        fjx -= fx;
        fjy -= fy;
        fjz -= fz;
        const int src = (lane + 1) & 31;
        pj.x = __shfl_sync(FULL, pj.x, src);
        pj.y = __shfl_sync(FULL, pj.y, src);
        pj.z = __shfl_sync(FULL, pj.z, src);
        pj.w = __shfl_sync(FULL, pj.w, src);
        lj.x = __shfl_sync(FULL, lj.x, src);
        lj.y = __shfl_sync(FULL, lj.y, src);
        fjx = __shfl_sync(FULL, fjx, src);
        fjy = __shfl_sync(FULL, fjy, src);
        fjz = __shfl_sync(FULL, fjz, src);
      }
    }
    const Real fscale = Real(kForceScale);
    if (ai >= 0) {
      add_fixed(a.force + ai, to_fixed(fix, fscale));
      add_fixed(a.force + a.n_atoms + ai, to_fixed(fiy, fscale));
      add_fixed(a.force + 2 * a.n_atoms + ai, to_fixed(fiz, fscale));
    }
    if (!diag) {
      const int aj = a.sorted_atom[sj];
      if (aj >= 0) {
        add_fixed(a.force + aj, to_fixed(fjx, fscale));
        add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fscale));
        add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fscale));
      }
    }
    if (kEnergy) {
      e_fixed += to_fixed(e_tile, kEnergyScale);
      for (int c = 0; c < 6; ++c) w_fixed[c] += to_fixed(w_tile[c], kEnergyScale);
    }
  }
  if (kEnergy) {
    for (int off = 16; off > 0; off >>= 1) {
      e_fixed += __shfl_xor_sync(FULL, e_fixed, off);
      for (int c = 0; c < 6; ++c) w_fixed[c] += __shfl_xor_sync(FULL, w_fixed[c], off);
    }
    if (lane == 0) {
      add_fixed(a.energy, e_fixed);
      for (int c = 0; c < 6; ++c) add_fixed(a.energy + 1 + c, w_fixed[c]);
    }
  }
}

template <class Real>
__global__ void pack_kernel(int n_slots, const int* sorted_atom, const double* pos,
                            const int* image, const double* block_center, const double* qscaled,
                            typename V4<Real>::T4* posq, Box<double> b) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const int a = sorted_atom[s];
  typename V4<Real>::T4 out;
  if (a < 0) {
    out.x = out.y = out.z = out.w = Real(0);
  } else {
    const double n0 = image[3 * a], n1 = image[3 * a + 1], n2 = image[3 * a + 2];
    const double* c = block_center + 3 * (s >> 5);
    out.x = (Real)(pos[3 * a] - (n0 * b.ax + n1 * b.bx + n2 * b.cx) - c[0]);
    out.y = (Real)(pos[3 * a + 1] - (n1 * b.by + n2 * b.cy) - c[1]);
    out.z = (Real)(pos[3 * a + 2] - n2 * b.cz - c[2]);
    out.w = (Real)qscaled[a];
  }
  posq[s] = out;
}

template <class Real>
__global__ void pack_params_kernel(int n_slots, const int* sorted_atom, const double* half_sigma,
                                   const double* sqrt_eps, typename V4<Real>::T2* ljp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const int a = sorted_atom[s];
  typename V4<Real>::T2 out;
  out.x = a < 0 ? Real(0) : (Real)half_sigma[a];
  out.y = a < 0 ? Real(0) : (Real)sqrt_eps[a];
  ljp[s] = out;
}

}  // namespace

template <class Real>
void launch_pair(const PairArgs<Real>& a, int elec, bool energy, bool dump, int grid,
                 cudaStream_t s) {
#define OMMB200_PAIR(E, EN, D) pair_kernel<Real, E, EN, D><<<grid, 128, 0, s>>>(a)
  if (dump) {
    if (elec == kElecEwald) OMMB200_PAIR(kElecEwald, false, true);
    else if (elec == kElecReactionField) OMMB200_PAIR(kElecReactionField, false, true);
    else OMMB200_PAIR(kElecCoulomb, false, true);
    return;
  }
  if (energy) {
    if (elec == kElecEwald) OMMB200_PAIR(kElecEwald, true, false);
    else if (elec == kElecReactionField) OMMB200_PAIR(kElecReactionField, true, false);
    else OMMB200_PAIR(kElecCoulomb, true, false);
  } else {
    if (elec == kElecEwald) OMMB200_PAIR(kElecEwald, false, false);
    else if (elec == kElecReactionField) OMMB200_PAIR(kElecReactionField, false, false);
    else OMMB200_PAIR(kElecCoulomb, false, false);
  }
#undef OMMB200_PAIR
}

template <class Real>
void launch_pack(int n_slots, const int* sorted_atom, const double* pos, const int* image,
                 const double* block_center, const double* qscaled, void* posq,
                 const Box<double>& box, cudaStream_t s) {
  pack_kernel<Real><<<ceil_div(n_slots, 256), 256, 0, s>>>(
      n_slots, sorted_atom, pos, image, block_center, qscaled,
      reinterpret_cast<typename V4<Real>::T4*>(posq), box);
}

template <class Real>
void launch_pack_params(int n_slots, const int* sorted_atom, const double* half_sigma,
                        const double* sqrt_eps, void* ljp, cudaStream_t s) {
  pack_params_kernel<Real><<<ceil_div(n_slots, 256), 256, 0, s>>>(
      n_slots, sorted_atom, half_sigma, sqrt_eps, reinterpret_cast<typename V4<Real>::T2*>(ljp));
}

template void launch_pair<float>(const PairArgs<float>&, int, bool, bool, int, cudaStream_t);
template void launch_pair<double>(const PairArgs<double>&, int, bool, bool, int, cudaStream_t);
template void launch_pack<float>(int, const int*, const double*, const int*, const double*,
                                 const double*, void*, const Box<double>&, cudaStream_t);
template void launch_pack<double>(int, const int*, const double*, const int*, const double*,
                                  const double*, void*, const Box<double>&, cudaStream_t);
template void launch_pack_params<float>(int, const int*, const double*, const double*, void*,
                                        cudaStream_t);
template void launch_pack_params<double>(int, const int*, const double*, const double*, void*,
                                         cudaStream_t);

}  // namespace ommb200
