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
#include <type_traits>

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

// The FP32 form with two i-particles per lane and packed (f32x2) arithmetic.  The warp splits
// into groups of G lanes (G = 8 for halves tiles, 16 otherwise); a group owns G consecutive
// entries and the 2G i-slots that meet them, lane m of the group holding i-slots m and m + G
// of its half (halves) or of the block.  In G steps the lane meets each of the group's entries
// once, evaluating the pairs with both of its i-particles in the two lanes of the packed
// values; the entry's force (both pairs summed) rotates one lane per step within the group and
// is back at the entry's own lane after G steps.  Every i-slot is met by two groups, whose
// partial forces are summed at the end (lane ^ G), so each lane commits the i-slot equal to
// its lane index and the entry it loaded.  A warp evaluates 64 pair slots per step, against 32
// in the one-particle-per-lane form, with half the shuffles and shared-memory reads per pair.
// Entry data sit in shared memory already duplicated into both lanes of each packed value, so
// a step moves no register.  The cutoff (and with it the exact decision band) applies to the
// Ewald and reaction-field forms; the bare-Coulomb form is the no-cutoff method.
template <int kElec, bool kEnergy, bool kDump, bool kSwitch>
__global__ void __launch_bounds__(32 * kPairWarps, 6) pair_kernel_x2(const PairArgs<float> a) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr bool kCutoff = kElec != kElecCoulomb;
  __shared__ float4 s_j[kPairWarps][3][32];  // per entry (x, x, y, y), (z, z, q, q), (s, s, e, e)
  __shared__ int s_atom[kPairWarps][32];
  __shared__ float4 s_ipos[kPairWarps][32];
  __shared__ float2 s_ilj[kPairWarps][32];
  __shared__ int s_iatom[kPairWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int warp = blockIdx.x * kPairWarps + w;
  const int nwarps = gridDim.x * kPairWarps;
  const int nt = min(*a.n_tiles, a.tile_capacity);
  const float4* posq = reinterpret_cast<const float4*>(a.posq);
  const float2* ljp = reinterpret_cast<const float2*>(a.ljp);
  const float4* entries = reinterpret_cast<const float4*>(a.entries);
  long long e_fixed = 0;
  long long w_fixed[6] = {0, 0, 0, 0, 0, 0};

  for (int t = warp; t < nt; t += nwarps) {
    const int4 tile = a.tiles[t];
    const float4 e = entries[32 * t + lane];  // unused (unwritten) for self tiles
    const int I = tile.x;
    const bool self = (tile.y & kTileSelf) != 0;
    const bool pair_image = (tile.y & kTilePairImage) != 0;
    const bool halves = (tile.y & kTileHalves) != 0;
    const int si = 32 * I + lane;
    const float4 pi = posq[si];
    const float2 li = ljp[si];
    const int ai = a.sorted_atom[si];
    const uint32_t excl = (tile.y & kTileHasMask) ? a.masks[32 * tile.z + lane] : 0u;
    float4 pj = pi;
    float2 lj = li;
    int aj = ai;
    if (!self) {
      const int slot = __float_as_int(e.w);
      pj = make_float4(0.f, 0.f, 0.f, 0.f);
      lj = make_float2(0.f, 0.f);
      aj = -1;
      if (slot >= 0) {
        pj = posq[slot];
        lj = ljp[slot];
        aj = a.sorted_atom[slot];
      }
      pj.x += e.x;
      pj.y += e.y;
      pj.z += e.z;
    }
    s_j[w][0][lane] = make_float4(pj.x, pj.x, pj.y, pj.y);
    s_j[w][1][lane] = make_float4(pj.z, pj.z, pj.w, pj.w);
    s_j[w][2][lane] = make_float4(lj.x, lj.x, lj.y, lj.y);
    s_atom[w][lane] = aj;
    s_ipos[w][lane] = pi;
    s_ilj[w][lane] = li;
    s_iatom[w][lane] = ai;
    __syncwarp();
    const int G = halves ? 8 : 16, gm = G - 1;
    const int m = lane & gm, eb = lane & ~gm;
    const int i1 = (halves ? (lane & 16) : 0) + m, i2 = i1 + G;
    // exclusion/padding bits of the two i-slots in step order: bit k (i1) and bit 16 + k (i2)
    // stand for entry eb + ((m + k) mod G); a self tile also drops the diagonal
    uint32_t steps_mask;
    {
      const uint32_t gmask = (1u << G) - 1u;
      const uint32_t x1 = ((__shfl_sync(FULL, excl, i1) | (self ? 1u << i1 : 0u)) >> eb) & gmask;
      const uint32_t x2v = ((__shfl_sync(FULL, excl, i2) | (self ? 1u << i2 : 0u)) >> eb) & gmask;
      const uint32_t r1 = ((x1 >> m) | (x1 << (G - m))) & gmask;
      const uint32_t r2v = ((x2v >> m) | (x2v << (G - m))) & gmask;
      steps_mask = r1 | (r2v << 16);
    }
    const float4 p1 = s_ipos[w][i1], p2 = s_ipos[w][i2];
    const float2 l1 = s_ilj[w][i1], l2 = s_ilj[w][i2];
    const float2 npx = make_float2(-p1.x, -p2.x), npy = make_float2(-p1.y, -p2.y),
                 npz = make_float2(-p1.z, -p2.z);
    const float2 qi = make_float2(p1.w, p2.w), sgi = make_float2(l1.x, l2.x),
                 epi = make_float2(l1.y, l2.y);
    float2 fx = x2::bc(0.f), fy = x2::bc(0.f), fz = x2::bc(0.f);
    float fjx = 0.f, fjy = 0.f, fjz = 0.f;
    double e_tile = 0.0;
    double w_tile[6] = {0, 0, 0, 0, 0, 0};
    const int src = eb | ((m + 1) & gm);
    auto steps = [&](auto image_tag) {
      constexpr bool kImage = decltype(image_tag)::value;
      uint32_t sm = steps_mask;
#pragma unroll 2
      for (int k = 0; k < G; ++k) {
        const int jl = eb | ((m + k) & gm);
        const float4 jxy = s_j[w][0][jl], jzq = s_j[w][1][jl], jse = s_j[w][2][jl];
        float2 dx = x2::add(make_float2(jxy.x, jxy.y), npx);
        float2 dy = x2::add(make_float2(jxy.z, jxy.w), npy);
        float2 dz = x2::add(make_float2(jzq.x, jzq.y), npz);
        if (kImage) {
          min_image_fast(dx.x, dy.x, dz.x, a.box);
          min_image_fast(dx.y, dy.y, dz.y, a.box);
        }
        const float2 r2 = x2::fma(dz, dz, x2::fma(dy, dy, x2::mul(dx, dx)));
        bool u1 = (sm & 1u) == 0u, u2 = (sm & 0x10000u) == 0u;
        sm >>= 1;
        if (kCutoff) {
          bool in1 = r2.x < a.cutoff2, in2 = r2.y < a.cutoff2;
          const float2 d = x2::add(r2, x2::bc(-a.cutoff2));
          const bool b1 = fabsf(d.x) < a.band && u1, b2 = fabsf(d.y) < a.band && u2;
          if (b1 | b2) {  // within the band: the reference's decision from the f64 positions
            const int b = s_atom[w][jl];
            if (b1) {
              const int ia = s_iatom[w][i1];
              in1 = ia >= 0 && b >= 0 &&
                    exact_inside(a.pos, ia, b, a.periodic, a.box_exact, a.cutoff2_exact);
            }
            if (b2) {
              const int ia = s_iatom[w][i2];
              in2 = ia >= 0 && b >= 0 &&
                    exact_inside(a.pos, ia, b, a.periodic, a.box_exact, a.cutoff2_exact);
            }
          }
          u1 = u1 && in1;
          u2 = u2 && in2;
        }
        if (kDump) {
          const int b = s_atom[w][jl];
          for (int h = 0; h < 2; ++h) {
            const int ia = s_iatom[w][h ? i2 : i1];
            if ((h ? u2 : u1) && ia >= 0 && b >= 0 && (!self || ia < b)) {
              const unsigned long long slot = atomicAdd(a.pair_count, 1ull);
              if ((long long)slot < a.pair_capacity) {
                a.pair_dump[2 * slot] = ia < b ? ia : b;
                a.pair_dump[2 * slot + 1] = ia < b ? b : ia;
              }
            }
          }
        }
        float2 fo, en;
        pair_terms_x2<kElec, kEnergy, kSwitch>(
            a, x2::select(u1, u2, r2, 1.f), x2::mul(make_float2(jzq.z, jzq.w), qi),
            x2::add(make_float2(jse.x, jse.y), sgi), x2::mul(make_float2(jse.z, jse.w), epi), fo, en);
        fo = x2::select(u1, u2, fo, 0.f);
        fx = x2::fma(fo, dx, fx);
        fy = x2::fma(fo, dy, fy);
        fz = x2::fma(fo, dz, fz);
        if (kEnergy) {
          const double scale = self ? 0.5 : 1.0;
          const float2 fdx = x2::mul(fo, dx), fdy = x2::mul(fo, dy), fdz = x2::mul(fo, dz);
          const float2 wxx = x2::mul(fdx, dx), wyy = x2::mul(fdy, dy), wzz = x2::mul(fdz, dz),
                       wxy = x2::mul(fdx, dy), wxz = x2::mul(fdx, dz), wyz = x2::mul(fdy, dz);
          if (u1) {
            e_tile += scale * (double)en.x;
            w_tile[0] -= scale * (double)wxx.x;
            w_tile[1] -= scale * (double)wyy.x;
            w_tile[2] -= scale * (double)wzz.x;
            w_tile[3] -= scale * (double)wxy.x;
            w_tile[4] -= scale * (double)wxz.x;
            w_tile[5] -= scale * (double)wyz.x;
          }
          if (u2) {
            e_tile += scale * (double)en.y;
            w_tile[0] -= scale * (double)wxx.y;
            w_tile[1] -= scale * (double)wyy.y;
            w_tile[2] -= scale * (double)wzz.y;
            w_tile[3] -= scale * (double)wxy.y;
            w_tile[4] -= scale * (double)wxz.y;
            w_tile[5] -= scale * (double)wyz.y;
          }
        }
        if (!self) {
          fjx = fmaf(-fo.x, dx.x, fjx);
          fjy = fmaf(-fo.x, dy.x, fjy);
          fjz = fmaf(-fo.x, dz.x, fjz);
          fjx = fmaf(-fo.y, dx.y, fjx);
          fjy = fmaf(-fo.y, dy.y, fjy);
          fjz = fmaf(-fo.y, dz.y, fjz);
          fjx = __shfl_sync(FULL, fjx, src);
          fjy = __shfl_sync(FULL, fjy, src);
          fjz = __shfl_sync(FULL, fjz, src);
        }
      }
    };
    if (pair_image)
      steps(std::true_type{});
    else
      steps(std::false_type{});
    // the two groups that met this lane's i-slots combine; the lane commits i-slot `lane`
    fx.x += __shfl_xor_sync(FULL, fx.x, G);
    fx.y += __shfl_xor_sync(FULL, fx.y, G);
    fy.x += __shfl_xor_sync(FULL, fy.x, G);
    fy.y += __shfl_xor_sync(FULL, fy.y, G);
    fz.x += __shfl_xor_sync(FULL, fz.x, G);
    fz.y += __shfl_xor_sync(FULL, fz.y, G);
    const bool second = (lane & G) != 0;
    const float fs = float(kForceScale);
    if (ai >= 0) {
      add_fixed(a.force + ai, to_fixed(second ? fx.y : fx.x, fs));
      add_fixed(a.force + a.n_atoms + ai, to_fixed(second ? fy.y : fy.x, fs));
      add_fixed(a.force + 2 * a.n_atoms + ai, to_fixed(second ? fz.y : fz.x, fs));
    }
    if (!self && aj >= 0) {
      add_fixed(a.force + aj, to_fixed(fjx, fs));
      add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fs));
      add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fs));
    }
    if (kEnergy) {
      for (int off = 16; off > 0; off >>= 1) {
        e_tile += __shfl_xor_sync(FULL, e_tile, off);
        for (int c = 0; c < 6; ++c) w_tile[c] += __shfl_xor_sync(FULL, w_tile[c], off);
      }
      if (a.block_segment) {
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

// `only_after_rebuild` (may be null): pack only when that rebuild flag is set (the integrator
// writes the packed coordinates of the other steps).
template <class Real>
__global__ void pack_kernel(int n_slots, const int* sorted_atom, const double* pos,
                            const int* image, const double* block_center, const double* qscaled,
                            const double* half_sigma, const double* two_sqrt_eps,
                            typename V4<Real>::T4* posq, typename V4<Real>::T2* ljp,
                            Box<double> b, const int* only_after_rebuild) {
  if (only_after_rebuild && *only_after_rebuild == 0) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const int a = sorted_atom[s];
  typename V4<Real>::T4 out;
  typename V4<Real>::T2 lj;
  if (a < 0) {
    out.x = out.y = out.z = out.w = Real(0);
    lj.x = lj.y = Real(0);
  } else {
    const double x[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    double r[3];
    block_local(x, image[3 * a], image[3 * a + 1], image[3 * a + 2], block_center + 3 * (s >> 5),
                b, r);
    out.x = (Real)r[0];
    out.y = (Real)r[1];
    out.z = (Real)r[2];
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
#define OMMB200_PAIR(E, EN, D, SW)                                                  \
  if constexpr (sizeof(Real) == 4)                                                  \
    pair_kernel_x2<E, EN, D, SW><<<grid, 32 * kPairWarps, 0, s>>>(a);               \
  else                                                                              \
    pair_kernel<Real, E, EN, D, SW><<<grid, 32 * kPairWarps, 0, s>>>(a)
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
                 cudaStream_t s, const int* only_after_rebuild) {
  pack_kernel<Real><<<ceil_div(n_slots, 256), 256, 0, s>>>(
      n_slots, sorted_atom, pos, image, block_center, qscaled, half_sigma, two_sqrt_eps,
      reinterpret_cast<typename V4<Real>::T4*>(posq), reinterpret_cast<typename V4<Real>::T2*>(ljp),
      box, only_after_rebuild);
}

template void launch_pair<float>(const PairArgs<float>&, int, bool, bool, int, cudaStream_t);
template void launch_pair<double>(const PairArgs<double>&, int, bool, bool, int, cudaStream_t);
template void launch_pack<float>(int, const int*, const double*, const int*, const double*,
                                 const double*, const double*, const double*, void*, void*,
                                 const Box<double>&, cudaStream_t, const int*);
template void launch_pack<double>(int, const int*, const double*, const int*, const double*,
                                  const double*, const double*, const double*, void*, void*,
                                  const Box<double>&, cudaStream_t, const int*);

}  // namespace ommb200
