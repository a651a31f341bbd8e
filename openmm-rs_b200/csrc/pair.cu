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
__global__ void __launch_bounds__(32 * kPairWarps, 5) pair_kernel_x2(const PairArgs<float> a) {
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
      // 96 registers and no unrolling: at 80 registers the compiler re-read constants and
      // lane-dependent values inside the loop (23,958-atom box: 62.9 -> 58.8 us)
#pragma unroll 1
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

// ---- culling form -----------------------------------------------------------------------
// The packed FP32 form over a halves-tile list, with the entries culled at the current
// positions.  A warp takes a run of consecutive tiles of one block I (a sub-chunk: tiles
// [sub K, (sub + 1) K) of the block's range, the last sub-chunk taking the rest) and drops
// every entry that lies farther than the cutoff (plus the exact-decision band) from the
// bounding box of the current positions of its half of I: no pair of such an entry can be
// inside the cutoff, so the pair set is unchanged.  The surviving entries of each half queue in
// a ring in shared memory; whenever both halves hold 16, a round runs the halves-tile steps
// (groups of 8 lanes, two i-slots per lane) over 16 queued entries per half, and at the end of
// the sub-chunk the rest runs with dummy entries (masked for every i-slot) topping the rounds
// up.  Each round commits its entries' forces; the i-forces accumulate over the sub-chunk and
// are committed once.  Sub-chunks are fixed runs of a block's own tiles, whose order the
// builder fixes, so rounds, float sums and forces are the same run to run, whichever warp
// takes them: warps fetch sub-chunks from a counter (all blocks' first sub-chunks, then the
// second ones, ...), and the last warp to finish resets the counter for the next launch (no
// warp waits for another).  Self tiles and tiles that need a per-pair minimum image are staged
// and run directly, after the queue is drained; a self tile runs as two rounds (each half's
// i-slots with the entries of its own half, then of the other half).  Exclusion words are kept
// over all 32 i-slots of block I, an entry of a tile holding only its own half's bits.  The
// next tile's header, entry and mask word are loaded one tile ahead.
constexpr int kRing = 64;  // queued entries per half of block I, per warp (a power of two)

// 32 x 32 bit transpose across the warp: lane r holds row r (bit c = M[r][c]); the result in
// lane c is column c (bit r = M[r][c]).  Five butterfly stages of block swaps.
__device__ __forceinline__ uint32_t transpose_bits(uint32_t x, int lane) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const uint32_t lo = s == 16  ? 0x0000FFFFu
                        : s == 8 ? 0x00FF00FFu
                        : s == 4 ? 0x0F0F0F0Fu
                        : s == 2 ? 0x33333333u
                                 : 0x55555555u;
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, s);
    x = (lane & s) ? ((x & ~lo) | ((y >> s) & lo)) : ((x & lo) | ((y & lo) << s));
  }
  return x;
}

struct CullRing {
  float4 j[3][2 * kRing];  // per entry (x, x, y, y), (z, z, q, q), (s, s, e, e); half h owns
                           // [h kRing, (h + 1) kRing)
  uint32_t em[2 * kRing];  // exclusion/padding bits of the entry over the 32 i-slots of I
  int at[2 * kRing];       // particle of the entry, -1 for a dummy
  float4 ipos[32];         // block I
  float2 ilj[32];
  int iatom[32];
  float4 lo[2], hi[2];     // bounding box of the real particles of each half of block I
};

__device__ __forceinline__ void ring_put(CullRing& r, int f, float4 pj, float2 lj, uint32_t em,
                                         int at) {
  r.j[0][f] = make_float4(pj.x, pj.x, pj.y, pj.y);
  r.j[1][f] = make_float4(pj.z, pj.z, pj.w, pj.w);
  r.j[2][f] = make_float4(lj.x, lj.x, lj.y, lj.y);
  r.em[f] = em;
  r.at[f] = at;
}

// Rounds of the culling kernel, in the order a warp runs them.
enum CullRound : int {
  kRoundQueue = 0,  // 16 queued entries per half from the ring heads
  kRoundImage = 1,  // a staged tile whose pairs take the minimum image
  kRoundSelf0 = 2,  // a staged self tile: each half's i-slots with its own half
  kRoundSelf1 = 3,  // ... then with the other half
};

// One round: lane m of a group of 8 lanes meets the group's 8 entries, at ring slots
// base + ((m + k) mod 8), with its i-slots i1 and i2, in 8 steps.  The entry's force rotates
// one lane per step and ends in the lane whose m is the entry's position (self rounds keep no
// entry forces: every pair is met from both sides, at half energy).
template <int kElec, bool kEnergy, bool kDump, bool kSwitch>
__device__ __forceinline__ void cull_steps(const PairArgs<float>& a, const CullRing& r, int base,
                                           int m, int src, int i1, int i2, bool image, bool self,
                                           float2 npx, float2 npy, float2 npz, float2 qi,
                                           float2 sgi, float2 epi, float2& fx, float2& fy,
                                           float2& fz, float& fjx, float& fjy, float& fjz,
                                           double& e_acc, double (&w_acc)[6]) {
  constexpr unsigned FULL = 0xffffffffu;
#pragma unroll 1
  for (int k = 0; k < 8; ++k) {
    const int jf = base + ((m + k) & 7);
    const float4 jxy = r.j[0][jf], jzq = r.j[1][jf], jse = r.j[2][jf];
    const uint32_t em = r.em[jf];
    float2 dx = x2::add(make_float2(jxy.x, jxy.y), npx);
    float2 dy = x2::add(make_float2(jxy.z, jxy.w), npy);
    float2 dz = x2::add(make_float2(jzq.x, jzq.y), npz);
    if (image) {
      min_image_fast(dx.x, dy.x, dz.x, a.box);
      min_image_fast(dx.y, dy.y, dz.y, a.box);
    }
    const float2 r2 = x2::fma(dz, dz, x2::fma(dy, dy, x2::mul(dx, dx)));
    bool u1 = ((em >> i1) & 1u) == 0u, u2 = ((em >> i2) & 1u) == 0u;
    {
      bool in1 = r2.x < a.cutoff2, in2 = r2.y < a.cutoff2;
      const float2 d = x2::add(r2, x2::bc(-a.cutoff2));
      const bool c1 = fabsf(d.x) < a.band && u1, c2 = fabsf(d.y) < a.band && u2;
      if (c1 | c2) {  // within the band: the reference's decision from the f64 positions
        const int b = r.at[jf];
        if (c1) {
          const int ia = r.iatom[i1];
          in1 = ia >= 0 && b >= 0 &&
                exact_inside(a.pos, ia, b, a.periodic, a.box_exact, a.cutoff2_exact);
        }
        if (c2) {
          const int ia = r.iatom[i2];
          in2 = ia >= 0 && b >= 0 &&
                exact_inside(a.pos, ia, b, a.periodic, a.box_exact, a.cutoff2_exact);
        }
      }
      u1 = u1 && in1;
      u2 = u2 && in2;
    }
    if (kDump) {
      const int b = r.at[jf];
      for (int hh = 0; hh < 2; ++hh) {
        const int ia = r.iatom[hh ? i2 : i1];
        if ((hh ? u2 : u1) && ia >= 0 && b >= 0 && (!self || ia < b)) {
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
        e_acc += scale * (double)en.x;
        w_acc[0] -= scale * (double)wxx.x;
        w_acc[1] -= scale * (double)wyy.x;
        w_acc[2] -= scale * (double)wzz.x;
        w_acc[3] -= scale * (double)wxy.x;
        w_acc[4] -= scale * (double)wxz.x;
        w_acc[5] -= scale * (double)wyz.x;
      }
      if (u2) {
        e_acc += scale * (double)en.y;
        w_acc[0] -= scale * (double)wxx.y;
        w_acc[1] -= scale * (double)wyy.y;
        w_acc[2] -= scale * (double)wzz.y;
        w_acc[3] -= scale * (double)wxy.y;
        w_acc[4] -= scale * (double)wxz.y;
        w_acc[5] -= scale * (double)wyz.y;
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
}

template <int kElec, bool kEnergy, bool kDump, bool kSwitch>
__global__ void __launch_bounds__(32 * kPairWarps, 5) pair_kernel_cull(const PairArgs<float> a) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ CullRing s_ring[kPairWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  CullRing& rg = s_ring[w];
  const int nwarps = gridDim.x * kPairWarps;
  const int nt = min(*a.n_tiles, a.tile_capacity);
  const int per = a.cull_chunks, K = a.cull_tiles;
  const int nb = *a.n_blocks;
  const int n_items = nb * per;
  const float4* posq = reinterpret_cast<const float4*>(a.posq);
  const float2* ljp = reinterpret_cast<const float2*>(a.ljp);
  const float4* entries = reinterpret_cast<const float4*>(a.entries);
  // rounds: groups of 8 lanes (gsub: the group's first entry within its half's 16); lane m of
  // a group meets i-slots i1 = 16 h + m and i2 = i1 + 8 of its half h
  const int h = lane >> 4, m = lane & 7, gsub = lane & 8;
  const int i1 = (lane & 16) + m, i2 = i1 + 8;
  const int src8 = (lane & ~7) | ((m + 1) & 7);
  const float fs = float(kForceScale);
  long long e_fixed = 0;
  long long w_fixed[6] = {0, 0, 0, 0, 0, 0};

  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(a.cull_work, 1);
    it = __shfl_sync(FULL, it, 0);
    if (it >= n_items) break;
    const int sub = it / nb, I = it - sub * nb;
    const int tb = a.block_tiles[2 * I], tn = a.block_tiles[2 * I + 1];
    const int k0 = sub * K;
    if (tb < 0 || k0 >= tn) continue;  // uniform
    const int k1 = min(sub == per - 1 ? tn : min(tn, k0 + K), nt - tb);
    {
      const int si = 32 * I + lane;
      rg.ipos[lane] = posq[si];
      rg.ilj[lane] = ljp[si];
      rg.iatom[lane] = a.sorted_atom[si];
    }
    __syncwarp();
    float2 npx, npy, npz, qi, sgi, epi;
    {
      const float4 p1 = rg.ipos[i1], p2 = rg.ipos[i2];
      const float2 l1 = rg.ilj[i1], l2 = rg.ilj[i2];
      npx = make_float2(-p1.x, -p2.x);
      npy = make_float2(-p1.y, -p2.y);
      npz = make_float2(-p1.z, -p2.z);
      qi = make_float2(p1.w, p2.w);
      sgi = make_float2(l1.x, l2.x);
      epi = make_float2(l1.y, l2.y);
    }
    {  // bounding box of the real particles of each half (empty: nothing is kept)
      const float4 pi = rg.ipos[lane];
      const bool real = rg.iatom[lane] >= 0;
      float lox = real ? pi.x : INFINITY, loy = real ? pi.y : INFINITY,
            loz = real ? pi.z : INFINITY;
      float hix = real ? pi.x : -INFINITY, hiy = real ? pi.y : -INFINITY,
            hiz = real ? pi.z : -INFINITY;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        lox = fminf(lox, __shfl_xor_sync(FULL, lox, o));
        loy = fminf(loy, __shfl_xor_sync(FULL, loy, o));
        loz = fminf(loz, __shfl_xor_sync(FULL, loz, o));
        hix = fmaxf(hix, __shfl_xor_sync(FULL, hix, o));
        hiy = fmaxf(hiy, __shfl_xor_sync(FULL, hiy, o));
        hiz = fmaxf(hiz, __shfl_xor_sync(FULL, hiz, o));
      }
      if ((lane & 15) == 0) {
        rg.lo[h] = make_float4(lox, loy, loz, 0.f);
        rg.hi[h] = make_float4(hix, hiy, hiz, 0.f);
      }
      __syncwarp();
    }
    float2 fx = x2::bc(0.f), fy = x2::bc(0.f), fz = x2::bc(0.f);
    double e_acc = 0.0;
    double w_acc[6] = {0, 0, 0, 0, 0, 0};
    int hd0 = 0, tl0 = 0, hd1 = 0, tl1 = 0;  // ring cursors per half (heads: multiples of 16)
    int mode = kRoundQueue;                   // the next round's kind
    int n_rounds = 0;
    bool staged_image = false;                // the staged self tile's pairs take the image
    int k = k0;
    // tile k's header, entry and exclusion word; the next tile's are fetched one tile ahead,
    // so their latency overlaps this tile's rounds
    int4 tile = make_int4(0, 0, 0, 0);
    float4 ent = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t xw = 0u;
    if (k < k1) {
      tile = a.tiles[tb + k];
      ent = entries[32 * (tb + k) + lane];
      if (tile.y & kTileHasMask) xw = a.masks[32 * tile.z + lane];
    }
    for (;;) {
      // a round is due for a staged tile, for two full halves or a nearly full ring, or to
      // empty the queue before a tile that must be staged and at the end of the sub-chunk
      const int q0 = tl0 - hd0, q1 = tl1 - hd1;
      const bool special = k < k1 && (tile.y & (kTileSelf | kTilePairImage)) != 0;
      const bool due = mode != kRoundQueue || (q0 >= 16 && q1 >= 16) || q0 > kRing - 16 ||
                       q1 > kRing - 16 || ((k >= k1 || special) && (q0 > 0 || q1 > 0));
      if (due) {
        if (mode == kRoundQueue) {  // top each half up to 16 entries with dummies
          const int hd = h ? hd1 : hd0, q = h ? q1 : q0, e = lane & 15;
          if (e >= q)
            ring_put(rg, kRing * h + ((hd + e) & (kRing - 1)), make_float4(0.f, 0.f, 0.f, 0.f),
                     make_float2(0.f, 0.f), 0xFFFFFFFFu, -1);
          __syncwarp();
        }
        const bool self = mode >= kRoundSelf0;
        const int base = mode == kRoundQueue ? kRing * h + ((h ? hd1 : hd0) & (kRing - 1)) + gsub
                                             : kRing * (h ^ (mode == kRoundSelf1)) + gsub;
        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
        cull_steps<kElec, kEnergy, kDump, kSwitch>(
            a, rg, base, m, src8, i1, i2, mode == kRoundImage || (self && staged_image), self,
            npx, npy, npz, qi, sgi, epi, fx, fy, fz, fjx, fjy, fjz, e_acc, w_acc);
        ++n_rounds;
        if (!self) {
          const int aj = rg.at[base + m];
          if (aj >= 0) {
            add_fixed(a.force + aj, to_fixed(fjx, fs));
            add_fixed(a.force + a.n_atoms + aj, to_fixed(fjy, fs));
            add_fixed(a.force + 2 * a.n_atoms + aj, to_fixed(fjz, fs));
          }
        }
        if (mode == kRoundQueue) {
          hd0 += 16;
          hd1 += 16;
          tl0 = max(tl0, hd0);
          tl1 = max(tl1, hd1);
        } else if (mode == kRoundSelf0) {
          mode = kRoundSelf1;
        } else {
          mode = kRoundQueue;
          hd0 = tl0 = hd1 = tl1 = 0;
        }
        __syncwarp();
        continue;
      }
      if (k >= k1) break;
      int4 tile_n = make_int4(0, 0, 0, 0);
      float4 ent_n = make_float4(0.f, 0.f, 0.f, 0.f);
      uint32_t xw_n = 0u;
      if (k + 1 < k1) {
        tile_n = a.tiles[tb + k + 1];
        ent_n = entries[32 * (tb + k + 1) + lane];
        if (tile_n.y & kTileHasMask) xw_n = a.masks[32 * tile_n.z + lane];
      }
      // tile k (the queue is empty if it is special)
      uint32_t col = 0u;  // exclusion bits of entry `lane` over the 32 i-slots
      if (tile.y & kTileHasMask) col = transpose_bits(xw, lane);
      if (tile.y & kTileSelf) {
        ring_put(rg, kRing * h + (lane & 15), rg.ipos[lane], rg.ilj[lane], col | (1u << lane),
                 rg.iatom[lane]);
        mode = kRoundSelf0;
        staged_image = (tile.y & kTilePairImage) != 0;
      } else {
        const float4 e = ent;
        const int slot = __float_as_int(e.w);
        float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 lj = make_float2(0.f, 0.f);
        int aj = -1;
        if (slot >= 0) {
          pj = posq[slot];
          lj = ljp[slot];
          aj = a.sorted_atom[slot];
        }
        pj.x += e.x;
        pj.y += e.y;
        pj.z += e.z;
        const uint32_t hmask = 0xFFFFu << (lane & 16);  // the i-slots of this entry's half
        const uint32_t em = col & hmask;
        if (special) {  // a small box: every pair takes the minimum image, nothing is culled
          ring_put(rg, kRing * h + (lane & 15), pj, lj, slot >= 0 ? em : 0xFFFFFFFFu, aj);
          mode = kRoundImage;
        } else {
          // distance from the entry to its half's box with the pair distance's rounding
          // (monotone in each component, so never above any of the entry's pair r^2)
          const float4 blo = rg.lo[h], bhi = rg.hi[h];
          const float cx = fmaxf(fmaxf(blo.x - pj.x, pj.x - bhi.x), 0.f);
          const float cy = fmaxf(fmaxf(blo.y - pj.y, pj.y - bhi.y), 0.f);
          const float cz = fmaxf(fmaxf(blo.z - pj.z, pj.z - bhi.z), 0.f);
          const float d2 = fmaf(cz, cz, fmaf(cy, cy, cx * cx));
          const bool keep = slot >= 0 && d2 < a.cull2 && em != hmask;
          const unsigned kb = __ballot_sync(FULL, keep);
          if (keep) {
            const unsigned mine = (kb >> (lane & 16)) & 0xFFFFu;
            const int pos = (h ? tl1 : tl0) + __popc(mine & ((1u << (lane & 15)) - 1u));
            ring_put(rg, kRing * h + (pos & (kRing - 1)), pj, lj, em, aj);
          }
          tl0 += __popc(kb & 0xFFFFu);
          tl1 += __popc(kb >> 16);
        }
      }
      __syncwarp();
      ++k;
      tile = tile_n;
      ent = ent_n;
      xw = xw_n;
    }
    // the two groups of each half met the same i-slots; the lane commits i-slot `lane`
    fx.x += __shfl_xor_sync(FULL, fx.x, 8);
    fx.y += __shfl_xor_sync(FULL, fx.y, 8);
    fy.x += __shfl_xor_sync(FULL, fy.x, 8);
    fy.y += __shfl_xor_sync(FULL, fy.y, 8);
    fz.x += __shfl_xor_sync(FULL, fz.x, 8);
    fz.y += __shfl_xor_sync(FULL, fz.y, 8);
    if (lane == 0) atomicAdd(a.cull_rounds, (unsigned long long)n_rounds);
    const int ai = rg.iatom[lane];
    if (ai >= 0) {
      const bool second = gsub != 0;
      add_fixed(a.force + ai, to_fixed(second ? fx.y : fx.x, fs));
      add_fixed(a.force + a.n_atoms + ai, to_fixed(second ? fy.y : fy.x, fs));
      add_fixed(a.force + 2 * a.n_atoms + ai, to_fixed(second ? fz.y : fz.x, fs));
    }
    if (kEnergy) {
      for (int off = 16; off > 0; off >>= 1) {
        e_acc += __shfl_xor_sync(FULL, e_acc, off);
        for (int c = 0; c < 6; ++c) w_acc[c] += __shfl_xor_sync(FULL, w_acc[c], off);
      }
      e_fixed += to_fixed(e_acc, kEnergyScale);
      for (int c = 0; c < 6; ++c) w_fixed[c] += to_fixed(w_acc[c], kEnergyScale);
    }
    __syncwarp();
  }
  if (kEnergy && lane == 0) {
    add_fixed(a.energy, e_fixed);
    for (int c = 0; c < 6; ++c) add_fixed(a.energy + 1 + c, w_fixed[c]);
  }
  // a warp counts itself only after its last fetch returned (the fetch's value decided the
  // loop's exit), so when the last warp counts itself no fetch is left and it may reset both
  // counters for the next launch
  if (lane == 0) {
    if (atomicAdd(a.cull_work + 1, 1) == nwarps - 1) {
      a.cull_work[0] = 0;
      a.cull_work[1] = 0;
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
  if constexpr (sizeof(Real) == 4) {                                                \
    if constexpr (E != kElecCoulomb) {                                              \
      if (a.cull_tiles > 0) {                                                       \
        cudaFuncSetAttribute(pair_kernel_cull<E, EN, D, SW>,                        \
                             cudaFuncAttributePreferredSharedMemoryCarveout,        \
                             cudaSharedmemCarveoutMaxShared);                       \
        pair_kernel_cull<E, EN, D, SW><<<grid, 32 * kPairWarps, 0, s>>>(a);         \
        return;                                                                     \
      }                                                                             \
    }                                                                               \
    pair_kernel_x2<E, EN, D, SW><<<grid, 32 * kPairWarps, 0, s>>>(a);               \
  } else                                                                            \
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
