// Real-space nonbonded pair kernel: LJ 12-6 (Lorentz-Berthelot, optional switching) plus
// Ewald-screened, reaction-field or bare Coulomb, following forces/nonbonded.rs:842-924 and
// the pair functions at nonbonded.rs:1194-1288.
//
// One warp evaluates one tile: lane l owns i-particle l of block I; the tile's 32 j-entries
// are staged in shared memory and lane l visits entry (l + k) mod 32 at step k, so every
// (i, j) pair is seen once in 32 steps with conflict-free shared-memory reads.  The force on
// each j-entry travels with the entry: it is rotated one lane per step by a warp shuffle and
// is back in lane j after 32 steps.  Self tiles (entries = block I) visit each pair from both
// sides and keep only i-forces, at half energy.  "Halves" tiles hold 16 entries for each half
// of block I (gathered against that half's smaller box): each half-warp rotates its own 16
// entries in 16 steps.  Forces are summed in `Real` within a tile and
// committed as 64-bit fixed point, so the total does not depend on tile order.
//
// Pair membership reproduces the reference exactly: pairs whose squared distance falls
// within `band` of rc^2 are re-decided from the f64 master positions with the reference's
// minimum-image and r^2 < rc^2 arithmetic (explicitly rounded, no fused multiply-add).
#include "kernels.h"
#include "pair_math.cuh"

namespace ommb200 {
namespace {

constexpr int kPairWarps = 4;

template <class Real, int kElec, bool kEnergy, bool kDump, bool kSwitch>
__global__ void __launch_bounds__(32 * kPairWarps) pair_kernel(const PairArgs<Real> a) {
  using T4 = typename V4<Real>::T4;
  using T2 = typename V4<Real>::T2;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ T4 s_pos[kPairWarps][32];
  __shared__ T2 s_lj[kPairWarps][32];
  __shared__ int s_atom[kPairWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int warp = blockIdx.x * kPairWarps + w;
  const int nwarps = gridDim.x * kPairWarps;
  const int nt = min(*a.n_tiles, a.tile_capacity);
  const T4* posq = reinterpret_cast<const T4*>(a.posq);
  const T2* ljp = reinterpret_cast<const T2*>(a.ljp);
  const T4* entries = reinterpret_cast<const T4*>(a.entries);
  long long e_fixed = 0;
  long long w_fixed[6] = {0, 0, 0, 0, 0, 0};

  for (int t = warp; t < nt; t += nwarps) {
    const int4 tile = a.tiles[t];
    const int I = tile.x;
    const bool self = (tile.y & kTileSelf) != 0;
    const bool pair_image = (tile.y & kTilePairImage) != 0;
    const bool halves = (tile.y & kTileHalves) != 0;
    const int si = 32 * I + lane;
    const T4 pi = posq[si];
    const T2 li = ljp[si];
    const int ai = a.sorted_atom[si];
    const uint32_t excl = (tile.y & kTileHasMask) ? a.masks[32 * tile.z + lane] : 0u;
    int aj = ai;
    if (self) {
      s_pos[w][lane] = pi;
      s_lj[w][lane] = li;
    } else {
      const T4 e = entries[32 * t + lane];
      int slot;
      if constexpr (sizeof(Real) == 4) slot = __float_as_int(e.w);
      else slot = (int)e.w;
      T4 pj;
      T2 lj;
      if (slot >= 0) {
        pj = posq[slot];
        lj = ljp[slot];
        aj = a.sorted_atom[slot];
      } else {
        pj.x = pj.y = pj.z = pj.w = Real(0);
        lj.x = lj.y = Real(0);
        aj = -1;
      }
      pj.x += e.x;
      pj.y += e.y;
      pj.z += e.z;
      s_pos[w][lane] = pj;
      s_lj[w][lane] = lj;
    }
    s_atom[w][lane] = aj;
    __syncwarp();
    Real fix = 0, fiy = 0, fiz = 0, fjx = 0, fjy = 0, fjz = 0;
    double e_tile = 0.0;
    double w_tile[6] = {0, 0, 0, 0, 0, 0};
    // halves tiles: lanes 0-15 (first half of block I) meet entries 0-15 in 16 steps, lanes
    // 16-31 entries 16-31; otherwise every lane meets all 32 entries.  j-forces travel one
    // lane per step within their group and are back at their entry's lane at the end.
    const int hb = halves ? (lane & 16) : 0, kmask = halves ? 15 : 31;
    const int nsteps = halves ? 16 : 32;
    const int src = hb | ((lane + 1) & kmask);
#pragma unroll 4
    for (int k = self ? 1 : 0; k < nsteps; ++k) {
      const int jl = hb | ((lane + k) & kmask);
      const T4 pj = s_pos[w][jl];
      const T2 lj = s_lj[w][jl];
      Real dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
      if (pair_image) min_image_fast(dx, dy, dz, a.box);
      Real r2 = dx * dx + dy * dy + dz * dz;
      bool use = ((excl >> jl) & 1u) == 0u;
      if (a.use_cutoff) {
        bool inside = r2 < a.cutoff2;
        if (fabs(r2 - a.cutoff2) < a.band && use) {
          const int b = s_atom[w][jl];
          inside = ai >= 0 && b >= 0 &&
                   exact_inside(a.pos, ai, b, a.periodic, a.box_exact, a.cutoff2_exact);
        }
        use = use && inside;
      }
      if (kDump && use) {
        const int b = s_atom[w][jl];
        if (ai >= 0 && b >= 0 && (!self || ai < b)) {
          const unsigned long long slot = atomicAdd(a.pair_count, 1ull);
          if ((long long)slot < a.pair_capacity) {
            a.pair_dump[2 * slot] = ai < b ? ai : b;
            a.pair_dump[2 * slot + 1] = ai < b ? b : ai;
          }
        }
      }
      Real fo, en;
      pair_terms<Real, kElec, kEnergy, kSwitch>(a, use ? r2 : Real(1), pi.w * pj.w, li.x + lj.x,
                                                li.y * lj.y, fo, en);
      fo = use ? fo : Real(0);
      fix = fma(fo, dx, fix);
      fiy = fma(fo, dy, fiy);
      fiz = fma(fo, dz, fiz);
      if (kEnergy && use) {
        const double scale = self ? 0.5 : 1.0;
        e_tile += scale * (double)en;
        w_tile[0] -= scale * (double)(fo * dx * dx);
        w_tile[1] -= scale * (double)(fo * dy * dy);
        w_tile[2] -= scale * (double)(fo * dz * dz);
        w_tile[3] -= scale * (double)(fo * dx * dy);
        w_tile[4] -= scale * (double)(fo * dx * dz);
        w_tile[5] -= scale * (double)(fo * dy * dz);
      }
      if (!self) {
        fjx = fma(-fo, dx, fjx);
        fjy = fma(-fo, dy, fjy);
        fjz = fma(-fo, dz, fjz);
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
    if (!self && aj >= 0) {
      add_fixed(a.force + aj, to_fixed(fjx, fscale));
      add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fscale));
      add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fscale));
    }
    if (kEnergy) {
      // one fixed-point rounding per tile: reduce the tile's partial sums across the warp in
      // f64 first (a fixed order, so the result stays deterministic)
      for (int off = 16; off > 0; off >>= 1) {
        e_tile += __shfl_xor_sync(FULL, e_tile, off);
        for (int c = 0; c < 6; ++c) w_tile[c] += __shfl_xor_sync(FULL, w_tile[c], off);
      }
      if (a.block_segment) {  // a batch: each tile's energy goes to its own system
        if (lane == 0) {
          long long* dst = a.energy + 8 * a.block_segment[I];
          add_fixed(dst, to_fixed(e_tile, kEnergyScale));
          for (int c = 0; c < 6; ++c) add_fixed(dst + 1 + c, to_fixed(w_tile[c], kEnergyScale));
        }
      } else {
        e_fixed += to_fixed(e_tile, kEnergyScale);
        for (int c = 0; c < 6; ++c) w_fixed[c] += to_fixed(w_tile[c], kEnergyScale);
      }
    }
    __syncwarp();
  }
  if (kEnergy && !a.block_segment) {
    if (lane == 0) {
      add_fixed(a.energy, e_fixed);
      for (int c = 0; c < 6; ++c) add_fixed(a.energy + 1 + c, w_fixed[c]);
    }
  }
}

template <class Real>
__global__ void pack_kernel(int n_slots, const int* sorted_atom, const double* pos,
                            const int* image, const double* block_center, const double* qscaled,
                            const double* half_sigma, const double* two_sqrt_eps,
                            typename V4<Real>::T4* posq, typename V4<Real>::T2* ljp,
                            Box<double> b) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const int a = sorted_atom[s];
  typename V4<Real>::T4 out;
  typename V4<Real>::T2 lj;
  if (a < 0) {
    out.x = out.y = out.z = out.w = Real(0);
    lj.x = lj.y = Real(0);
  } else {
    const double n0 = image[3 * a], n1 = image[3 * a + 1], n2 = image[3 * a + 2];
    const double* c = block_center + 3 * (s >> 5);
    out.x = (Real)(pos[3 * a] - (n0 * b.ax + n1 * b.bx + n2 * b.cx) - c[0]);
    out.y = (Real)(pos[3 * a + 1] - (n1 * b.by + n2 * b.cy) - c[1]);
    out.z = (Real)(pos[3 * a + 2] - n2 * b.cz - c[2]);
    out.w = (Real)qscaled[a];
    lj.x = (Real)half_sigma[a];
    lj.y = (Real)two_sqrt_eps[a];
  }
  posq[s] = out;
  ljp[s] = lj;
}

}  // namespace

template <class Real>
void launch_pair(const PairArgs<Real>& a, int elec, bool energy, bool dump, int grid,
                 cudaStream_t s) {
#define OMMB200_PAIR(E, EN, D, SW) pair_kernel<Real, E, EN, D, SW><<<grid, 32 * kPairWarps, 0, s>>>(a)
#define OMMB200_PAIR_SW(E, EN, D)     \
  if (a.use_switching)                \
    OMMB200_PAIR(E, EN, D, true);     \
  else                                \
    OMMB200_PAIR(E, EN, D, false)
#define OMMB200_PAIR_E(EN, D)                                      \
  if (elec == kElecEwald) {                                        \
    OMMB200_PAIR_SW(kElecEwald, EN, D);                            \
  } else if (elec == kElecReactionField) {                         \
    OMMB200_PAIR_SW(kElecReactionField, EN, D);                    \
  } else {                                                         \
    OMMB200_PAIR_SW(kElecCoulomb, EN, D);                          \
  }
  if (dump) {
    OMMB200_PAIR_E(false, true)
  } else if (energy) {
    OMMB200_PAIR_E(true, false)
  } else {
    OMMB200_PAIR_E(false, false)
  }
#undef OMMB200_PAIR_E
#undef OMMB200_PAIR_SW
#undef OMMB200_PAIR
}

template <class Real>
void launch_pack(int n_slots, const int* sorted_atom, const double* pos, const int* image,
                 const double* block_center, const double* qscaled, const double* half_sigma,
                 const double* two_sqrt_eps, void* posq, void* ljp, const Box<double>& box,
                 cudaStream_t s) {
  pack_kernel<Real><<<ceil_div(n_slots, 256), 256, 0, s>>>(
      n_slots, sorted_atom, pos, image, block_center, qscaled, half_sigma, two_sqrt_eps,
      reinterpret_cast<typename V4<Real>::T4*>(posq), reinterpret_cast<typename V4<Real>::T2*>(ljp),
      box);
}

template void launch_pair<float>(const PairArgs<float>&, int, bool, bool, int, cudaStream_t);
template void launch_pair<double>(const PairArgs<double>&, int, bool, bool, int, cudaStream_t);
template void launch_pack<float>(int, const int*, const double*, const int*, const double*,
                                 const double*, const double*, const double*, void*, void*,
                                 const Box<double>&, cudaStream_t);
template void launch_pack<double>(int, const int*, const double*, const int*, const double*,
                                  const double*, const double*, const double*, void*, void*,
                                  const Box<double>&, cudaStream_t);

}  // namespace ommb200
