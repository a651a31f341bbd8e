// Neighbour tiles for periodic cutoff methods.
//
// The reference enumerates candidate pairs from a linked-list cell grid rebuilt at every
// evaluation (forces/neighbors.rs:96-181) and tests each pair against r^2 < rc^2
// (forces/nonbonded.rs:862).  Here the list is rebuilt only when some particle has moved
// more than skin/2 since the last rebuild (the integrator raises `rebuild`), so every pair
// inside the cutoff at any step in between is covered; the pair kernel applies the
// reference's exact cutoff test, which makes the interacting pair set the reference's.
//
// Sort: particles are binned into x-y columns about 0.62 nm wide and ordered by z inside
// each column; every column starts on a 32-slot block boundary, so a block is a compact
// ~0.6 x 0.6 x 0.7 nm brick.  Ties are broken by particle index, so the slot order (and with
// it every force sum) is deterministic.
//
// Tiles: for every block I, one self tile, then the particles of blocks J > I that lie within
// cutoff + skin of I's bounding box, packed 32 at a time into neighbour tiles.  Each entry
// stores the offset of its block's frame from I's frame, so the pair kernel works in small
// block-local coordinates.  Block pairs too close to a periodic image of themselves are kept
// whole and flagged for a per-pair minimum image.
//
// Every kernel returns at once unless `rebuild` is set, so the sequence can sit in a CUDA
// graph that is replayed every step.
#include <type_traits>

#include "kernels.h"

namespace ommb200 {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// atomicAdd(counter, 1) for every calling lane, as one atomic per distinct key among the warp's
// active lanes (a column's particles meet in few warps, so per-lane atomics on the same counter
// would serialise); returns the lane's old-value offset like atomicAdd would.
__device__ __forceinline__ int aggregated_add(int* counter, int key) {
  const unsigned peers = __match_any_sync(__activemask(), key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

__global__ void nl_columns(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    *a.n_tiles = 0;
    *a.n_masks = 0;
  }
  if (i >= a.n_atoms) return;
  double x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
  a.pos_ref[3 * i] = x;
  a.pos_ref[3 * i + 1] = y;
  a.pos_ref[3 * i + 2] = z;
  const Box<double>& b = a.box;
  const double n2 = floor(z * b.inv_cz);
  z -= n2 * b.cz;
  y -= n2 * b.cy;
  x -= n2 * b.cx;
  const double n1 = floor(y * b.inv_by);
  y -= n1 * b.by;
  x -= n1 * b.bx;
  const double n0 = floor(x * b.inv_ax);
  x -= n0 * b.ax;
  a.image[3 * i] = (int)n0;
  a.image[3 * i + 1] = (int)n1;
  a.image[3 * i + 2] = (int)n2;
  const int cx = min(max((int)(x * b.inv_ax * a.n_col[0]), 0), a.n_col[0] - 1);
  const int cy = min(max((int)(y * b.inv_by * a.n_col[1]), 0), a.n_col[1] - 1);
  const int col = cy * a.n_col[0] + cx;
  a.column[i] = col;
  a.zkey[i] = fmaxf((float)z, 0.0f);
  aggregated_add(&a.col_count[col], col);
}

// Single-CTA scan over the columns: padded slot starts, unpadded scatter starts, block count.
__global__ void __launch_bounds__(1024) nl_col_scan(NlistArgs a) {
  if (*a.rebuild == 0) return;
  __shared__ int ps[1024], pu[1024];
  const int t = threadIdx.x;
  const int chunk = (a.n_cols + 1023) / 1024;
  const int lo = min(t * chunk, a.n_cols), hi = min(lo + chunk, a.n_cols);
  int sp = 0, su = 0;
  for (int c = lo; c < hi; ++c) {
    const int n = a.col_count[c];
    if (n > a.col_max) report_status(a.status, kStatusTileOverflow);
    sp += (n + 31) & ~31;
    su += n;
  }
  ps[t] = sp;
  pu[t] = su;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int vp = t >= off ? ps[t - off] : 0, vu = t >= off ? pu[t - off] : 0;
    __syncthreads();
    ps[t] += vp;
    pu[t] += vu;
    __syncthreads();
  }
  int rp = ps[t] - sp, ru = pu[t] - su;
  for (int c = lo; c < hi; ++c) {
    a.col_start[c] = rp;
    a.col_scatter[c] = ru;
    const int n = a.col_count[c];
    rp += (n + 31) & ~31;
    ru += n;
  }
  const int total = min(ps[1023], a.slot_capacity);
  if (t == 0) {
    a.col_start[a.n_cols] = total;
    a.col_scatter[a.n_cols] = pu[1023];
    *a.n_blocks = total / 32;
  }
  for (int s = total + t; s < a.slot_capacity; s += 1024) a.sorted_atom[s] = -1;
}

__global__ void nl_col_scatter(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms) return;
  const int c = a.column[i];
  a.scratch_atoms[a.col_scatter[c] + aggregated_add(&a.col_cursor[c], c)] = i;
}

// One CTA per column: bitonic sort of (z, particle) keys in shared memory.
__global__ void __launch_bounds__(256) nl_col_sort(NlistArgs a) {
  if (*a.rebuild == 0) return;
  extern __shared__ unsigned long long keys[];
  const int c = blockIdx.x;
  const int n = a.col_count[c];
  if (n > a.col_max || n == 0) return;
  int m = 1;
  while (m < n) m <<= 1;
  const int s0 = a.col_scatter[c];
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    if (k < n) {
      const int atom = a.scratch_atoms[s0 + k];
      keys[k] = ((unsigned long long)__float_as_uint(a.zkey[atom]) << 32) | (unsigned)atom;
    } else {
      keys[k] = ~0ull;
    }
  }
  __syncthreads();
  for (int size = 2; size <= m; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int j = k ^ stride;
        if (j > k) {
          const bool up = (k & size) == 0;
          const unsigned long long x = keys[k], y = keys[j];
          if ((x > y) == up) {
            keys[k] = y;
            keys[j] = x;
          }
        }
      }
      __syncthreads();
    }
  const int base = a.col_start[c];
  const int padded = (n + 31) & ~31;
  for (int k = threadIdx.x; k < padded; k += blockDim.x) {
    if (base + k >= a.slot_capacity) break;
    if (k < n) {
      const int atom = (int)(keys[k] & 0xffffffffu);
      a.sorted_atom[base + k] = atom;
      a.atom_slot[atom] = base + k;
    } else {
      a.sorted_atom[base + k] = -1;
    }
  }
}

// One warp per block: bounding box of the wrapped rebuild positions.
__global__ void nl_bounds(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int lane = threadIdx.x & 31;
  const int blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (blk >= *a.n_blocks) return;
  const int atom = a.sorted_atom[32 * blk + lane];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (atom >= 0) {
    const Box<double>& b = a.box;
    const double n0 = a.image[3 * atom], n1 = a.image[3 * atom + 1], n2 = a.image[3 * atom + 2];
    const double w[3] = {a.pos_ref[3 * atom] - (n0 * b.ax + n1 * b.bx + n2 * b.cx),
                         a.pos_ref[3 * atom + 1] - (n1 * b.by + n2 * b.cy),
                         a.pos_ref[3 * atom + 2] - n2 * b.cz};
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = w[d];
    a.slot_wpos[32 * blk + lane] = make_double4(w[0], w[1], w[2], 0.0);
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(kFull, lo[d], off));
      hi[d] = fmax(hi[d], __shfl_xor_sync(kFull, hi[d], off));
    }
  if (lane == 0)
    for (int d = 0; d < 3; ++d) {
      const bool empty = lo[d] > hi[d];
      a.block_center[3 * blk + d] = empty ? 0.0 : 0.5 * (lo[d] + hi[d]);
      a.block_half[3 * blk + d] = empty ? 0.0 : 0.5 * (hi[d] - lo[d]);
    }
}

__device__ __forceinline__ double box_gap2(const double d[3], const double* hi, const double* hj) {
  double s = 0.0;
  for (int k = 0; k < 3; ++k) {
    double g = fabs(d[k]) - hi[k] - (hj ? hj[k] : 0.0);
    g = g > 0.0 ? g : 0.0;
    s += g * g;
  }
  return s;
}

// Exclusion partners of a lane's particle as slots, loaded once per block I: up to
// kCachedPartners in registers; a particle with more keeps reading its CSR row.
constexpr int kCachedPartners = 8;
struct Partners {
  int slot[kCachedPartners];
  int n;  // cached count, or -1 when the particle has more partners than fit
};

__device__ __forceinline__ Partners load_partners(const NlistArgs& a, int ai) {
  Partners p;
  p.n = 0;
#pragma unroll
  for (int k = 0; k < kCachedPartners; ++k) p.slot[k] = -2;
  if (ai < 0) return p;
  const int e0 = a.excl_start[ai], e1 = a.excl_start[ai + 1];
  if (e1 - e0 > kCachedPartners) {
    p.n = -1;
    return p;
  }
#pragma unroll
  for (int k = 0; k < kCachedPartners; ++k)
    if (e0 + k < e1) p.slot[k] = a.atom_slot[a.excl_list[e0 + k]];
  p.n = e1 - e0;
  return p;
}

// Mask of lane l over 32 entry slots: bit k set when entry k is padding or an exclusion
// partner of the lane's particle; all bits when the lane itself is padding.
__device__ __forceinline__ uint32_t entry_mask(const NlistArgs& a, int ai, const Partners& pt,
                                               const int* slots) {
  if (ai < 0) return kFull;
  uint32_t m = 0;
  for (int k = 0; k < 32; ++k) {
    const int sk = slots[k];
    bool hit = sk < 0;
#pragma unroll
    for (int q = 0; q < kCachedPartners; ++q) hit = hit || sk == pt.slot[q];
    if (hit) m |= 1u << k;
  }
  if (pt.n < 0) {
    for (int e = a.excl_start[ai]; e < a.excl_start[ai + 1]; ++e) {
      const int sp = a.atom_slot[a.excl_list[e]];
      for (int k = 0; k < 32; ++k)
        if (slots[k] == sp) m |= 1u << k;
    }
  }
  return m;
}

// entry_mask restricted to the 16 entries [kb, kb + 16) a lane meets in a halves tile (the
// other bits stay clear: the pair kernel never reads them).  The entries are read once; each
// cached partner is compared with all 16, and only as many partners as the particle has.
__device__ __forceinline__ uint32_t entry_mask_half(const NlistArgs& a, int ai, const Partners& pt,
                                                    const int* slots, int kb) {
  if (ai < 0) return kFull;
  int sk[16];
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    sk[k] = slots[kb + k];
    if (sk[k] < 0) m |= 1u << (kb + k);
  }
  if (pt.n < 0) {
    for (int e = a.excl_start[ai]; e < a.excl_start[ai + 1]; ++e) {
      const int sp = a.atom_slot[a.excl_list[e]];
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (sk[k] == sp) m |= 1u << (kb + k);
    }
    return m;
  }
#pragma unroll
  for (int q = 0; q < kCachedPartners; ++q) {
    if (q < pt.n) {
      const int sp = pt.slot[q];
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (sk[k] == sp) m |= 1u << (kb + k);
    }
  }
  return m;
}

// Position of set bit r (0-based, r < popc(m)) of m: a binary search on the population of the
// lower half of the remaining window, five steps without branches.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int r) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const int c = __popc(m & ((1u << w) - 1u));
    const bool up = r >= c;
    r -= up ? c : 0;
    m = up ? m >> w : m;
    pos += up ? w : 0;
  }
  return pos;
}

// Reserve a tile (and a mask slot if any lane needs one) and write its header and masks.
__device__ __forceinline__ int commit_tile(const NlistArgs& a, int I, int flags, uint32_t mask,
                                           int lane) {
  int t = 0;
  if (lane == 0) t = atomicAdd(a.n_tiles, 1);
  t = __shfl_sync(kFull, t, 0);
  if (t >= a.tile_capacity) {
    if (lane == 0) report_status(a.status, kStatusTileOverflow);
    return -1;
  }
  int slot = -1;
  if (__any_sync(kFull, mask != 0)) {
    if (lane == 0) slot = atomicAdd(a.n_masks, 1);
    slot = __shfl_sync(kFull, slot, 0);
    if (slot < a.mask_capacity) {
      a.masks[32 * slot + lane] = mask;
      flags |= kTileHasMask;
    } else {
      if (lane == 0) report_status(a.status, kStatusTileOverflow);
      slot = -1;
    }
  }
  if (lane == 0) a.tiles[t] = make_int4(I, flags, slot, 0);
  return t;
}

template <bool kDouble>
__device__ __forceinline__ void write_entry(const NlistArgs& a, int t, int lane, int slot,
                                            const double* sh) {
  if (kDouble)
    reinterpret_cast<double4*>(a.entries)[32 * t + lane] =
        make_double4(sh[0], sh[1], sh[2], (double)slot);
  else
    reinterpret_cast<float4*>(a.entries)[32 * t + lane] =
        make_float4((float)sh[0], (float)sh[1], (float)sh[2], __int_as_float(slot));
}

constexpr int kListWarps = 4;

// One warp per block I: self tile, then neighbour tiles of up to 32 gathered particles.
template <bool kDouble>
__global__ void __launch_bounds__(32 * kListWarps) nl_lists(NlistArgs a) {
  if (*a.rebuild == 0) return;
  __shared__ int s_slot[kListWarps][64];
  __shared__ int s_flag[kListWarps][64];
  __shared__ double s_shift[kListWarps][64][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nb = *a.n_blocks;
  const double reach = a.cutoff + a.skin;
  const double reach2 = reach * reach;
  const int warps = gridDim.x * kListWarps;
  for (int I = blockIdx.x * kListWarps + w; I < nb; I += warps) {
    const double ci[3] = {a.block_center[3 * I], a.block_center[3 * I + 1], a.block_center[3 * I + 2]};
    const double hi[3] = {a.block_half[3 * I], a.block_half[3 * I + 1], a.block_half[3 * I + 2]};
    const double ri = sqrt(hi[0] * hi[0] + hi[1] * hi[1] + hi[2] * hi[2]);
    const int ai = a.sorted_atom[32 * I + lane];
    const Partners partners = load_partners(a, ai);
    // self tile
    {
      s_slot[w][lane] = ai < 0 ? -1 : 32 * I + lane;
      __syncwarp();
      uint32_t m = entry_mask(a, ai, partners, s_slot[w]);
      const bool image = a.periodic && a.min_width < reach + 2.0 * ri;
      commit_tile(a, I, kTileSelf | (image ? kTilePairImage : 0), m, lane);
      __syncwarp();
    }
    int pending = 0;
    auto flush = [&](int count) {
      const int slot = lane < count ? s_slot[w][lane] : -1;
      const int f = __reduce_or_sync(kFull, lane < count ? s_flag[w][lane] : 0);
      if (lane >= count) s_slot[w][lane] = -1;
      __syncwarp();
      const uint32_t m = entry_mask(a, ai, partners, s_slot[w]);
      const int t = commit_tile(a, I, f, m, lane);
      double sh[3] = {0.0, 0.0, 0.0};
      if (lane < count)
        for (int d = 0; d < 3; ++d) sh[d] = s_shift[w][lane][d];
      if (t >= 0) write_entry<kDouble>(a, t, lane, slot, sh);
      __syncwarp();
    };
    // candidate blocks J in [j0, j1), 32 per pass
    auto scan = [&](int j0, int j1) {
      for (int base = j0; base < j1; base += 32) {
        const int J = base + lane;
        bool cand = false, unsafe = false;
        double d[3] = {0.0, 0.0, 0.0};
        if (J < j1) {
          const double* cj = a.block_center + 3 * J;
          const double* hj = a.block_half + 3 * J;
          d[0] = cj[0] - ci[0];
          d[1] = cj[1] - ci[1];
          d[2] = cj[2] - ci[2];
          double gap2 = 0.0;
          if (a.periodic) {
            min_image_fast(d[0], d[1], d[2], a.box);
            const double rj = sqrt(hj[0] * hj[0] + hj[1] * hj[1] + hj[2] * hj[2]);
            const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            // every other image is at least min_width - |d| away (reduced box); when that is
            // not enough to rule the other images out, all 27 images are tested
            unsafe = a.min_width - dist < reach + ri + rj;
          }
          gap2 = box_gap2(d, hi, hj);
          if (unsafe) {
            const Box<double>& b = a.box;
            for (int m0 = -1; m0 <= 1; ++m0)
              for (int m1 = -1; m1 <= 1; ++m1)
                for (int m2 = -1; m2 <= 1; ++m2) {
                  const double e[3] = {d[0] + m0 * b.ax + m1 * b.bx + m2 * b.cx,
                                       d[1] + m1 * b.by + m2 * b.cy, d[2] + m2 * b.cz};
                  gap2 = fmin(gap2, box_gap2(e, hi, hj));
                }
          }
          cand = gap2 < reach2;
        }
        unsigned cm = __ballot_sync(kFull, cand);
        // the candidate blocks' particles, one block ahead of the one being tested
        auto fetch = [&](int src, int* aj, double4* wp) {
          const int slot = 32 * (base + src) + lane;
          *aj = a.sorted_atom[slot];
          *wp = a.slot_wpos[slot];
        };
        int src = -1, aj_next = -1;
        double4 wp_next = make_double4(0.0, 0.0, 0.0, 0.0);
        if (cm) {
          src = __ffs(cm) - 1;
          cm &= cm - 1;
          fetch(src, &aj_next, &wp_next);
        }
        while (src >= 0) {
          const int Jc = base + src;
          const int aj = aj_next;
          const double4 wp = wp_next;
          const int cur = src;
          src = -1;
          if (cm) {
            src = __ffs(cm) - 1;
            cm &= cm - 1;
            fetch(src, &aj_next, &wp_next);
          }
          const double s0 = __shfl_sync(kFull, d[0], cur), s1 = __shfl_sync(kFull, d[1], cur),
                       s2 = __shfl_sync(kFull, d[2], cur);
          const bool un = __shfl_sync(kFull, unsafe, cur);
          bool in = false;
          if (aj >= 0) {
            const Box<double>& b = a.box;
            const double* cj = a.block_center + 3 * Jc;
            double rel[3] = {wp.x - cj[0] + s0, wp.y - cj[1] + s1, wp.z - cj[2] + s2};
            if (un) {
              // conservative: the nearest image of the particle to I's centre, against a
              // sphere that contains I's box
              min_image_fast(rel[0], rel[1], rel[2], b);
              const double r = sqrt(rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2]);
              in = r < reach + ri + 1e-6;
            } else {
              in = box_gap2(rel, hi, nullptr) < reach2;
            }
          }
          const unsigned im = __ballot_sync(kFull, in);
          if (in) {
            const int p = pending + __popc(im & ((1u << lane) - 1u));
            s_slot[w][p] = 32 * Jc + lane;
            s_flag[w][p] = un ? kTilePairImage : 0;
            s_shift[w][p][0] = s0;
            s_shift[w][p][1] = s1;
            s_shift[w][p][2] = s2;
          }
          pending += __popc(im);
          __syncwarp();
          if (pending >= 32) {
            flush(32);
            const int rest = pending - 32;
            int sl = 0, fl = 0;
            double sh0 = 0.0, sh1 = 0.0, sh2 = 0.0;
            if (lane < rest) {
              sl = s_slot[w][32 + lane];
              fl = s_flag[w][32 + lane];
              sh0 = s_shift[w][32 + lane][0];
              sh1 = s_shift[w][32 + lane][1];
              sh2 = s_shift[w][32 + lane][2];
            }
            __syncwarp();
            if (lane < rest) {
              s_slot[w][lane] = sl;
              s_flag[w][lane] = fl;
              s_shift[w][lane][0] = sh0;
              s_shift[w][lane][1] = sh1;
              s_shift[w][lane][2] = sh2;
            }
            pending = rest;
            __syncwarp();
          }
        }
      }
    };
    const Box<double>& bx = a.box;
    if (!a.periodic || bx.bx != 0.0 || bx.cx != 0.0 || bx.cy != 0.0 || a.sorted_atom[32 * I] < 0) {
      scan(I + 1, nb);  // triclinic: every later block is a candidate
    } else {
      // rectangular box: blocks lie inside their x-y column, so only columns whose x and y
      // ranges come within `reach` of I's column can hold candidates (a column k apart is at
      // least (k - 1) column widths away); the range covers every periodic image
      const int first = a.sorted_atom[32 * I];
      const int col = first >= 0 ? a.column[first] : 0;
      const int nx = a.n_col[0], ny = a.n_col[1];
      const int kx = (int)floor(reach * nx / bx.ax + 1e-6) + 1;
      const int ky = (int)floor(reach * ny / bx.by + 1e-6) + 1;
      const bool all_x = 2 * kx + 1 >= nx, all_y = 2 * ky + 1 >= ny;
      const int x0 = col % nx, y0 = col / nx;
      const int ny_iter = all_y ? ny : 2 * ky + 1, nx_iter = all_x ? nx : 2 * kx + 1;
      for (int oy = 0; oy < ny_iter; ++oy) {
        const int cy = all_y ? oy : (y0 + oy - ky + ny) % ny;
        for (int ox = 0; ox < nx_iter; ++ox) {
          const int cx = all_x ? ox : (x0 + ox - kx + nx) % nx;
          const int c = cy * nx + cx;
          const int j0 = max(a.col_start[c] / 32, I + 1), j1 = min(a.col_start[c + 1] / 32, nb);
          if (j0 < j1) scan(j0, j1);
        }
      }
    }
    if (pending > 0) flush(pending);
  }
}

// Rectangular boxes: one CTA of kCtaWarps warps per block I, in four phases.
//   A  candidate blocks J > I of I's column neighbourhood whose boxes come within reach (the
//      warps split the columns; two passes place every warp's candidates at fixed offsets)
//   B  per candidate, the 32-bit masks of its particles within reach of each half of I (slots
//      0-15 and 16-31; one warp per candidate; the conservative sphere test for blocks near a
//      periodic image of I)
//   C  prefix sums of the masks' populations pack each half's particles 16 to a half tile;
//      tile k carries the k-th 16 entries of both halves
//   D  each warp fills whole tiles: entries, flags, and exclusion masks
// Candidates, masks and prefix sums live in shared memory; I's tiles are reserved with one
// atomic, so they are contiguous.  The selected particles and their order are a function of
// the rebuild positions alone, so the tile contents are deterministic.
constexpr int kCtaWarps = 8;
constexpr int kStageRegs = 2;  // staged candidates per lane when phase A packs its regions

template <bool kDouble>
__global__ void __launch_bounds__(32 * kCtaWarps, 4) nl_lists_cta(NlistArgs a) {
  if (*a.rebuild == 0) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int cap = a.max_cand;
  double* c_d = reinterpret_cast<double*>(smem);                    // [3][cap]
  int* c_J = reinterpret_cast<int*>(c_d + 3 * (size_t)cap);          // [cap]
  int* c_un = c_J + cap;                                             // [cap]
  uint32_t* c_mask = reinterpret_cast<uint32_t*>(c_un + cap);        // [2][cap] per half of I
  int* c_pre = reinterpret_cast<int*>(c_mask + 2 * (size_t)cap);     // [2][cap + 1]
  __shared__ int s_wcount[kCtaWarps], s_wbase[kCtaWarps + 1];
  __shared__ int s_tile0, s_ntiles, s_spill;
  __shared__ int s_slots[kCtaWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nb = *a.n_blocks;
  const int I = blockIdx.x;
  if (I >= nb) return;
  const double reach = a.cutoff + a.skin;
  const double reach2 = reach * reach;
  const double ci[3] = {a.block_center[3 * I], a.block_center[3 * I + 1], a.block_center[3 * I + 2]};
  const double hi[3] = {a.block_half[3 * I], a.block_half[3 * I + 1], a.block_half[3 * I + 2]};
  const double ri = sqrt(hi[0] * hi[0] + hi[1] * hi[1] + hi[2] * hi[2]);
  const Box<double>& bx = a.box;
  // boxes of the two halves of I (slots 0-15 and 16-31), relative to I's centre
  double hc[3], hh[3];
  {
    const int ai0 = a.sorted_atom[32 * I + lane];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, up[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (ai0 >= 0) {
      const double4 wp = a.slot_wpos[32 * I + lane];
      lo[0] = up[0] = wp.x - ci[0];
      lo[1] = up[1] = wp.y - ci[1];
      lo[2] = up[2] = wp.z - ci[2];
    }
    for (int o = 8; o > 0; o >>= 1)
      for (int d = 0; d < 3; ++d) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(kFull, lo[d], o));
        up[d] = fmax(up[d], __shfl_xor_sync(kFull, up[d], o));
      }
    for (int d = 0; d < 3; ++d) {
      const bool empty = lo[d] > up[d];
      hc[d] = empty ? 0.0 : 0.5 * (lo[d] + up[d]);
      hh[d] = empty ? -1.0 : 0.5 * (up[d] - lo[d]);  // negative: the half holds no particle
    }
  }
  const double hcA[3] = {__shfl_sync(kFull, hc[0], 0), __shfl_sync(kFull, hc[1], 0), __shfl_sync(kFull, hc[2], 0)};
  const double hhA[3] = {__shfl_sync(kFull, hh[0], 0), __shfl_sync(kFull, hh[1], 0), __shfl_sync(kFull, hh[2], 0)};
  const double hcB[3] = {__shfl_sync(kFull, hc[0], 16), __shfl_sync(kFull, hc[1], 16), __shfl_sync(kFull, hc[2], 16)};
  const double hhB[3] = {__shfl_sync(kFull, hh[0], 16), __shfl_sync(kFull, hh[1], 16), __shfl_sync(kFull, hh[2], 16)};
  const int first = a.sorted_atom[32 * I];
  const int col = first >= 0 ? a.column[first] : 0;
  const int nx = a.n_col[0], ny = a.n_col[1];
  const int kx = (int)floor(reach * nx / bx.ax + 1e-6) + 1;
  const int ky = (int)floor(reach * ny / bx.by + 1e-6) + 1;
  const bool all_x = 2 * kx + 1 >= nx, all_y = 2 * ky + 1 >= ny;
  const int x0 = col % nx, y0 = col / nx;
  const int ny_iter = all_y ? ny : 2 * ky + 1, nx_iter = all_x ? nx : 2 * kx + 1;
  const int n_colq = nx_iter * ny_iter;
  // candidate test of block J (same arithmetic as the warp-per-block kernel)
  auto test = [&](int J, double d[3], bool* unsafe) {
    const double* cj = a.block_center + 3 * J;
    const double* hj = a.block_half + 3 * J;
    d[0] = cj[0] - ci[0];
    d[1] = cj[1] - ci[1];
    d[2] = cj[2] - ci[2];
    min_image_fast(d[0], d[1], d[2], bx);
    const double rj = sqrt(hj[0] * hj[0] + hj[1] * hj[1] + hj[2] * hj[2]);
    const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    *unsafe = a.min_width - dist < reach + ri + rj;
    double gap2 = box_gap2(d, hi, hj);
    if (*unsafe) {
      for (int m0 = -1; m0 <= 1; ++m0)
        for (int m1 = -1; m1 <= 1; ++m1)
          for (int m2 = -1; m2 <= 1; ++m2) {
            const double e[3] = {d[0] + m0 * bx.ax + m1 * bx.bx + m2 * bx.cx,
                                 d[1] + m1 * bx.by + m2 * bx.cy, d[2] + m2 * bx.cz};
            gap2 = fmin(gap2, box_gap2(e, hi, hj));
          }
    }
    return gap2 < reach2;
  };
  // phase A: the warps split I's columns.  In one pass each warp stages its candidates, in
  // test order, in its own region of the candidate arrays; the regions are then packed in
  // warp order (through registers, so no region is overwritten before it is read).  A warp
  // with more candidates than its region holds makes the CTA test again, placing every
  // candidate at its final offset.  Either way candidate c of warp w lands at
  // s_wbase[w] + c, the same order whichever way it was placed.
  const int region = min(cap / kCtaWarps, 32 * kStageRegs);
  auto scan_columns = [&](bool staged) {
    int n = 0;
    for (int q = w; q < n_colq; q += kCtaWarps) {
      const int oy = q / nx_iter, ox = q % nx_iter;
      const int cy = all_y ? oy : (y0 + oy - ky + ny) % ny;
      const int cx = all_x ? ox : (x0 + ox - kx + nx) % nx;
      const int c = cy * nx + cx;
      const int j0 = max(a.col_start[c] / 32, I + 1), j1 = min(a.col_start[c + 1] / 32, nb);
      for (int base = j0; base < j1; base += 32) {
        const int J = base + lane;
        double d[3] = {0.0, 0.0, 0.0};
        bool unsafe = false, cand = false;
        if (J < j1) cand = test(J, d, &unsafe);
        const unsigned m = __ballot_sync(kFull, cand);
        if (cand) {
          const int r = n + __popc(m & ((1u << lane) - 1u));
          const int k = staged ? (r < region ? w * region + r : cap) : s_wbase[w] + r;
          if (k < cap) {
            c_J[k] = J;
            c_un[k] = unsafe ? 1 : 0;
            c_d[k] = d[0];
            c_d[cap + k] = d[1];
            c_d[2 * cap + k] = d[2];
          }
        }
        n += __popc(m);
      }
    }
    return n;
  };
  if (threadIdx.x == 0) s_spill = 0;
  __syncthreads();
  {
    const int n = scan_columns(true);
    if (lane == 0) {
      s_wcount[w] = n;
      if (n > region) s_spill = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int u = 0; u < kCtaWarps; ++u) {
      s_wbase[u] = t;
      t += s_wcount[u];
    }
    s_wbase[kCtaWarps] = t;
  }
  __syncthreads();
  if (s_spill) {
    scan_columns(false);
  } else {
    const int nw = s_wcount[w];
    int rJ[kStageRegs], run[kStageRegs];
    double rd[kStageRegs][3];
#pragma unroll
    for (int u = 0; u < kStageRegs; ++u) {
      const int i = lane + 32 * u, k = w * region + i;
      if (i < nw) {
        rJ[u] = c_J[k];
        run[u] = c_un[k];
        rd[u][0] = c_d[k];
        rd[u][1] = c_d[cap + k];
        rd[u][2] = c_d[2 * cap + k];
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kStageRegs; ++u) {
      const int i = lane + 32 * u, k = s_wbase[w] + i;
      if (i < nw && k < cap) {
        c_J[k] = rJ[u];
        c_un[k] = run[u];
        c_d[k] = rd[u][0];
        c_d[cap + k] = rd[u][1];
        c_d[2 * cap + k] = rd[u][2];
      }
    }
  }
  __syncthreads();
  int n_cand = s_wbase[kCtaWarps];
  if (n_cand > cap) {  // cannot happen with the host-computed capacity
    if (threadIdx.x == 0) report_status(a.status, kStatusTileOverflow);
    n_cand = cap;
  }
  // phase B: one warp per candidate; a particle is kept for a half of I when it lies within
  // reach of that half's box (the conservative sphere around it near a periodic image)
  int aj_n = -1;
  double4 wp_n = make_double4(0.0, 0.0, 0.0, 0.0);
  if (w < n_cand) {  // this warp's first candidate, fetched ahead
    const int slot = 32 * c_J[w] + lane;
    aj_n = a.sorted_atom[slot];
    wp_n = a.slot_wpos[slot];
  }
  for (int c = w; c < n_cand; c += kCtaWarps) {
    const int J = c_J[c];
    const bool un = c_un[c] != 0;
    const int aj = aj_n;
    const double4 wp = wp_n;
    if (c + kCtaWarps < n_cand) {  // the next candidate's particles, in flight meanwhile
      const int slot = 32 * c_J[c + kCtaWarps] + lane;
      aj_n = a.sorted_atom[slot];
      wp_n = a.slot_wpos[slot];
    }
    bool in_a = false, in_b = false;
    if (aj >= 0) {
      const double* cj = a.block_center + 3 * J;
      const double rel[3] = {wp.x - cj[0] + c_d[c], wp.y - cj[1] + c_d[cap + c],
                             wp.z - cj[2] + c_d[2 * cap + c]};
      auto near_half = [&](const double* hcen, const double* hext) {
        if (hext[0] < 0.0) return false;
        double rh[3] = {rel[0] - hcen[0], rel[1] - hcen[1], rel[2] - hcen[2]};
        if (un) {
          min_image_fast(rh[0], rh[1], rh[2], bx);
          const double rad = sqrt(hext[0] * hext[0] + hext[1] * hext[1] + hext[2] * hext[2]);
          return sqrt(rh[0] * rh[0] + rh[1] * rh[1] + rh[2] * rh[2]) < reach + rad + 1e-6;
        }
        return box_gap2(rh, hext, nullptr) < reach2;
      };
      in_a = near_half(hcA, hhA);
      in_b = near_half(hcB, hhB);
    }
    const unsigned ma = __ballot_sync(kFull, in_a), mb = __ballot_sync(kFull, in_b);
    if (lane == 0) {
      c_mask[c] = ma;
      c_mask[cap + c] = mb;
    }
  }
  __syncthreads();
  // phase C: prefix sums of the masks' populations per half (warps 0 and 1), then reserve
  // I's tiles: the self tile and one tile per 16 entries of the longer half
  if (w < 2) {
    const uint32_t* mk = c_mask + (size_t)w * cap;
    int* pre = c_pre + (size_t)w * (cap + 1);
    int carry = 0;
    for (int base = 0; base < n_cand; base += 32) {
      const int c = base + lane;
      const int v = c < n_cand ? __popc(mk[c]) : 0;
      int incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
      }
      if (c < n_cand) pre[c] = carry + incl - v;
      carry += __shfl_sync(kFull, incl, 31);
    }
    if (lane == 0) pre[n_cand] = carry;
  }
  __syncthreads();
  if (w == 0) {
    if (lane == 0) {
      const int tot_a = c_pre[n_cand], tot_b = c_pre[(cap + 1) + n_cand];
      const int nt = 1 + (max(tot_a, tot_b) + 15) / 16;
      int t0 = atomicAdd(a.n_tiles, nt);
      if (t0 + nt > a.tile_capacity) {
        report_status(a.status, kStatusTileOverflow);
        t0 = -1;
      }
      s_tile0 = t0;
      s_ntiles = nt;
      if (a.block_tiles) {
        a.block_tiles[2 * I] = t0;
        a.block_tiles[2 * I + 1] = t0 < 0 ? 0 : nt;
      }
    }
  }
  __syncthreads();
  if (s_tile0 < 0) return;
  const int half = lane >> 4;
  const uint32_t* my_mask = c_mask + (size_t)half * cap;
  const int* my_pre = c_pre + (size_t)half * (cap + 1);
  const int total = my_pre[n_cand];
  const int ai = a.sorted_atom[32 * I + lane];
  const Partners partners = load_partners(a, ai);
  // phase D: whole tiles per warp; tile 0 is I's self tile
  for (int k = w; k < s_ntiles; k += kCtaWarps) {
    int slot = -1, flag = 0;
    double sh[3] = {0.0, 0.0, 0.0};
    if (k == 0) {
      slot = ai < 0 ? -1 : 32 * I + lane;
      flag = kTileSelf | ((a.min_width < reach + 2.0 * ri) ? kTilePairImage : 0);
    } else {
      const int e = 16 * (k - 1) + (lane & 15);  // this half's entry
      if (e < total) {
        int lo = 0, hi_c = n_cand - 1;  // last candidate with pre <= e
        while (lo < hi_c) {
          const int mid = (lo + hi_c + 1) >> 1;
          if (my_pre[mid] <= e) lo = mid;
          else hi_c = mid - 1;
        }
        const int bit = nth_set_bit(my_mask[lo], e - my_pre[lo]);
        slot = 32 * c_J[lo] + bit;
        flag = c_un[lo] ? kTilePairImage : 0;
        sh[0] = c_d[lo];
        sh[1] = c_d[cap + lo];
        sh[2] = c_d[2 * cap + lo];
      }
      flag = __reduce_or_sync(kFull, flag) | kTileHalves;
    }
    s_slots[w][lane] = slot;
    __syncwarp();
    const uint32_t m = k == 0 ? entry_mask(a, ai, partners, s_slots[w])
                              : entry_mask_half(a, ai, partners, s_slots[w], lane & 16);
    const int t = s_tile0 + k;
    int mslot = -1;
    int flags = flag;
    if (__any_sync(kFull, m != 0)) {
      if (lane == 0) mslot = atomicAdd(a.n_masks, 1);
      mslot = __shfl_sync(kFull, mslot, 0);
      if (mslot < a.mask_capacity) {
        a.masks[32 * mslot + lane] = m;
        flags |= kTileHasMask;
      } else {
        if (lane == 0) report_status(a.status, kStatusTileOverflow);
        mslot = -1;
      }
    }
    if (lane == 0) a.tiles[t] = make_int4(I, flags, mslot, 0);
    if (k > 0) write_entry<kDouble>(a, t, lane, slot, sh);
    __syncwarp();
  }
}

__global__ void nl_finish(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = i; k < a.n_cols; k += gridDim.x * blockDim.x) {
    a.col_count[k] = 0;
    a.col_cursor[k] = 0;
  }
}

// Inside a captured step: the rebuild kernels sit in the body of a conditional graph node
// that runs only when the integrator raised the flag.
__global__ void nl_set_condition(const int* rebuild, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, *rebuild != 0 ? 1u : 0u);
}

__global__ void nl_clear_flag(NlistArgs a) {
  if (*a.rebuild == 0) return;
  *a.rebuild = 0;
  *a.rebuild_count += 1;
  if (a.prune) *a.prune = 1;  // the pruned list derives from the tiles just built
}

// ---- pruned list ---------------------------------------------------------------------------
// The rebuild keeps every particle within cutoff + skin of a half block's box; between rebuilds
// the pair kernel needs only those within cutoff of a particle of the half.  The prune keeps an
// entry while it lies within cutoff + margin of some particle of its half at the current
// positions and packs each half's kept entries, in their rebuild order, 16 to an inner tile; the
// integrator asks for a new prune once a particle has moved more than margin / 2 since the last
// one, so every pair within the cutoff until then stays listed (a pair approaches by less than
// the margin, and it is among the rebuild's tiles while no particle moved skin / 2).
// Two kernels.  The keep pass gives every rebuild tile one warp over the whole list (two rounds
// of loads: the tile, then its particles) and stores the kept bits of its 32 entries.  The
// placement pass gives each block I one CTA: a prefix over I's tiles gives each kept entry its
// place, the kept entries move with their exclusion columns (the bits of the i-slots that
// exclude them), then each inner tile gets its masks (exclusions, padding) and header.  Block
// I's self tile is copied.  A block with more tiles than the shared arrays hold keeps all its
// entries (still a valid list).  The last placement CTA to finish closes the prune.
constexpr int kPruneMaxTiles = 256;
constexpr int kPruneSharedCols = 64;  // inner tiles whose exclusion columns stay in shared memory
constexpr int kPruneKeepWarps = 8;
constexpr int kPruneUnroll = 4;       // rebuild tiles a placement warp loads in one round
constexpr int kPlaceWarps = 4;        // placement CTA: 128 threads, all blocks resident at once

template <bool kDouble>
__global__ void __launch_bounds__(32 * kPruneKeepWarps) nl_prune_keep(const NlistArgs a,
                                                                     const PruneArgs p) {
  if (*p.prune == 0) return;
  using T4 = typename std::conditional<kDouble, double4, float4>::type;
  using R = typename std::conditional<kDouble, double, float>::type;
  __shared__ T4 s_i[kPruneKeepWarps][32];
  __shared__ int s_ok[kPruneKeepWarps][32];
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // the placement pass allocates from zero
    *p.n_tiles = 0;
    *p.done = 0u;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, hb = lane & 16;
  const int n_t = min(*a.n_tiles, a.tile_capacity);
  const T4* posq = reinterpret_cast<const T4*>(p.posq);
  const T4* ent = reinterpret_cast<const T4*>(a.entries);
  const R reach2 = (R)p.reach2;
  Box<R> b;
  b.ax = (R)a.box.ax; b.bx = (R)a.box.bx; b.by = (R)a.box.by;
  b.cx = (R)a.box.cx; b.cy = (R)a.box.cy; b.cz = (R)a.box.cz;
  b.inv_ax = (R)a.box.inv_ax; b.inv_by = (R)a.box.inv_by; b.inv_cz = (R)a.box.inv_cz;
  for (int t = blockIdx.x * kPruneKeepWarps + w; t < n_t; t += gridDim.x * kPruneKeepWarps) {
    const int4 hdr = a.tiles[t];
    const T4 e = ent[32 * (size_t)t + lane];
    const int ai = a.sorted_atom[32 * hdr.x + lane];
    const T4 pi = posq[32 * hdr.x + lane];
    int slot;
    if constexpr (kDouble) slot = (int)e.w;
    else slot = __float_as_int(e.w);
    T4 pj = pi;
    if (slot >= 0) pj = posq[slot];
    __syncwarp();
    s_i[w][lane] = pi;
    s_ok[w][lane] = ai >= 0;
    __syncwarp();
    bool keep = false;
    if (slot >= 0) {
      const R x = pj.x + e.x, y = pj.y + e.y, z = pj.z + e.z;
      const bool image = (hdr.y & kTilePairImage) != 0;
#pragma unroll 4
      for (int q = 0; q < 16; ++q) {
        const T4 c = s_i[w][hb + q];
        R dx = x - c.x, dy = y - c.y, dz = z - c.z;
        if (image) min_image_fast(dx, dy, dz, b);
        keep = keep || (s_ok[w][hb + q] && dx * dx + dy * dy + dz * dz < reach2);
      }
    }
    const unsigned kb = __ballot_sync(kFull, keep);
    if (lane == 0) p.keep[t] = kb;
  }
}

template <bool kDouble>
__global__ void __launch_bounds__(32 * kPlaceWarps) nl_prune_place(const NlistArgs a,
                                                                const PruneArgs p) {
  if (*p.prune == 0) return;
  using T4 = typename std::conditional<kDouble, double4, float4>::type;
  using R = typename std::conditional<kDouble, double, float>::type;
  __shared__ int s_iatom[32];
  __shared__ unsigned s_keep[kPruneMaxTiles];
  __shared__ int s_pre[2][kPruneMaxTiles + 1];
  __shared__ uint32_t s_cols[kPruneSharedCols][32];
  __shared__ int s_t0, s_nt, s_img;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int I = blockIdx.x;
  int t_out = -1, n_out = 0;
  if (I < *a.n_blocks) {
    t_out = a.block_tiles[2 * I];
    n_out = a.block_tiles[2 * I + 1];
  }
  // (a block of an overflowed build places nothing; the rebuild reported it)
  if (t_out >= 0 && n_out >= 1 && t_out + n_out <= a.tile_capacity) {
    const T4* ent = reinterpret_cast<const T4*>(a.entries);
    T4* ent_in = reinterpret_cast<T4*>(p.entries);
    const int n_nbr = n_out - 1;  // tile t_out is I's self tile
    const bool all = n_nbr > kPruneMaxTiles;
    const int n_scan = all ? 0 : n_nbr;
    if (w == 0) {
      const int ai = a.sorted_atom[32 * I + lane];
      s_iatom[lane] = ai;
      if (ai >= 0)
        for (int c = 0; c < 3; ++c) p.pos_prune[3 * ai + c] = a.pos[3 * ai + c];
      if (lane == 0) s_img = 0;
    }
    for (int k = threadIdx.x; k < n_scan; k += blockDim.x) s_keep[k] = p.keep[t_out + 1 + k];
    __syncthreads();
    // prefix of the kept entries per half over I's tiles (warp h for half h)
    if (w < 2) {
      int carry = 0;
      for (int base = 0; base < n_scan; base += 32) {
        const int k = base + lane;
        const int v = k < n_scan ? __popc((s_keep[k] >> (16 * w)) & 0xffffu) : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += y;
        }
        if (k < n_scan) s_pre[w][k] = carry + incl - v;
        carry += __shfl_sync(kFull, incl, 31);
      }
      if (lane == 0) s_pre[w][n_scan] = carry;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int longest = all ? 16 * n_nbr : max(s_pre[0][n_nbr], s_pre[1][n_nbr]);
      const int nt = 1 + (longest + 15) / 16;
      int t0 = atomicAdd(p.n_tiles, nt);
      if (t0 + nt > p.capacity) {
        report_status(a.status, kStatusTileOverflow);
        t0 = -1;
      }
      s_t0 = t0;
      s_nt = nt;
    }
    __syncthreads();
    if (s_t0 >= 0) {
      // exclusion columns of the inner neighbour tiles: shared memory, or the global scratch
      // for a block with more tiles than that holds
      const bool shared_cols = s_nt - 1 <= kPruneSharedCols;
      uint32_t* cols = shared_cols ? &s_cols[0][0] : p.cols + 32 * (size_t)(s_t0 + 1);
      // block I's self tile, unchanged (its mask slot becomes its tile index)
      if (w == 0) {
        int4 hdr = a.tiles[t_out];
        const bool masked = (hdr.y & kTileHasMask) != 0 && hdr.z >= 0;
        p.masks[32 * s_t0 + lane] = masked ? a.masks[32 * hdr.z + lane] : 0u;
        hdr.z = s_t0;
        if (!masked) hdr.y &= ~kTileHasMask;
        if (lane == 0) p.tiles[s_t0] = hdr;
      }
      // the kept entries to their inner places, with their exclusion columns; a warp loads
      // kPruneUnroll tiles (headers, entries, then mask rows) before it moves them
      for (int k0 = w; k0 < n_nbr; k0 += kPruneUnroll * kPlaceWarps) {
        int4 hdr[kPruneUnroll];
        T4 e[kPruneUnroll];
        uint32_t row[kPruneUnroll];
#pragma unroll
        for (int u = 0; u < kPruneUnroll; ++u) {
          const int k = k0 + u * kPlaceWarps;
          hdr[u] = make_int4(0, 0, -1, 0);
          if (k < n_nbr) {
            hdr[u] = a.tiles[t_out + 1 + k];
            e[u] = ent[32 * (size_t)(t_out + 1 + k) + lane];
          }
        }
#pragma unroll
        for (int u = 0; u < kPruneUnroll; ++u)
          row[u] = ((hdr[u].y & kTileHasMask) && hdr[u].z >= 0) ? a.masks[32 * hdr[u].z + lane]
                                                                 : 0u;
#pragma unroll
        for (int u = 0; u < kPruneUnroll; ++u) {
          const int k = k0 + u * kPlaceWarps;
          if (k >= n_nbr) break;
          if (lane == 0 && (hdr[u].y & kTilePairImage)) atomicOr(&s_img, kTilePairImage);
          const unsigned kb = all ? kFull : s_keep[k];  // all: the tile as it is, padding too
          uint32_t col = 0u;  // i-slots of this entry's half that exclude it
          if ((hdr[u].y & kTileHasMask) && hdr[u].z >= 0) {
            for (int q = 0; q < 32; ++q) {
              const unsigned c = __ballot_sync(kFull, (row[u] >> q) & 1u);
              if (lane == q) col = c;
            }
          }
          if ((kb >> lane) & 1u) {
            const int half = lane >> 4;
            const unsigned before = kb & ((1u << lane) - 1u) & (half ? 0xffff0000u : 0xffffu);
            const int r = (all ? 16 * k : s_pre[half][k]) + __popc(before);
            const int j = r / 16, q = 16 * half + (r & 15);
            ent_in[32 * (size_t)(s_t0 + 1 + j) + q] = e[u];
            cols[32 * j + q] = col;
          }
        }
      }
      // padding places of each half's last tile
      const int tot_a = all ? 16 * n_nbr : s_pre[0][n_nbr];
      const int tot_b = all ? 16 * n_nbr : s_pre[1][n_nbr];
      for (int idx = threadIdx.x; idx < (s_nt - 1) * 32; idx += blockDim.x) {
        const int j = idx >> 5, q = idx & 31, r = 16 * j + (q & 15);
        if (r >= ((q & 16) ? tot_b : tot_a)) {
          T4 pad;
          pad.x = pad.y = pad.z = R(0);
          if constexpr (kDouble) pad.w = -1.0;
          else pad.w = __int_as_float(-1);
          ent_in[32 * (size_t)(s_t0 + 1 + j) + q] = pad;
          cols[32 * j + q] = 0u;
        }
      }
      __syncthreads();
      // masks (exclusions of the lane's i-slot among its half's entries, padding) and headers
      const int ai = s_iatom[lane];
      const int hb = lane & 16, tot = hb ? tot_b : tot_a;
      for (int j = w; j < s_nt - 1; j += kPlaceWarps) {
        const int ti = s_t0 + 1 + j;
        uint32_t m = 0u;
        if (ai < 0) {
          m = kFull;
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const bool pad = 16 * j + q >= tot;
            const bool excl = (cols[32 * j + hb + q] >> lane) & 1u;
            if (pad || excl) m |= 1u << (hb + q);
          }
        }
        p.masks[32 * (size_t)ti + lane] = m;
        const bool any = __any_sync(kFull, m != 0u);
        if (lane == 0)
          p.tiles[ti] = make_int4(I, kTileHalves | s_img | (any ? kTileHasMask : 0), ti, 0);
      }
    }
  }
  // the last CTA to finish: tile count within capacity, prune done
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(p.done, 1u) == gridDim.x - 1) {
      __threadfence();
      const int used = atomicAdd(p.n_tiles, 0);
      if (used > p.capacity) *p.n_tiles = p.capacity;
      *p.prune = 0;
      *p.prune_count += 1;
    }
  }
}

__global__ void nl_prune_condition(const int* prune, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, *prune != 0 ? 1u : 0u);
}

}  // namespace

void launch_nlist_condition(const NlistArgs& a, cudaGraphConditionalHandle handle,
                            cudaStream_t s) {
  nl_set_condition<<<1, 1, 0, s>>>(a.rebuild, handle);
}

void launch_prune_condition(const PruneArgs& p, cudaGraphConditionalHandle handle, cudaStream_t s) {
  nl_prune_condition<<<1, 1, 0, s>>>(p.prune, handle);
}

void launch_nlist_prune(const NlistArgs& a, const PruneArgs& p, bool double_entries,
                        cudaStream_t s) {
  const int block_cap = a.slot_capacity / 32;
  // the keep pass: as many CTAs as fit on the device at once, striding over the tiles
  static int resident[2] = {0, 0};
  int& r = resident[double_entries ? 1 : 0];
  if (r == 0) {
    if (double_entries)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, nl_prune_keep<true>, 32 * kPruneKeepWarps, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, nl_prune_keep<false>, 32 * kPruneKeepWarps, 0);
    r = std::max(r, 1);
  }
  const int keep_grid =
      std::max(1, std::min(ceil_div(a.tile_capacity, kPruneKeepWarps), r * p.sm_count));
  if (double_entries) {
    nl_prune_keep<true><<<keep_grid, 32 * kPruneKeepWarps, 0, s>>>(a, p);
    nl_prune_place<true><<<block_cap, 32 * kPlaceWarps, 0, s>>>(a, p);
  } else {
    nl_prune_keep<false><<<keep_grid, 32 * kPruneKeepWarps, 0, s>>>(a, p);
    nl_prune_place<false><<<block_cap, 32 * kPlaceWarps, 0, s>>>(a, p);
  }
}

void launch_nlist_rebuild(const NlistArgs& a, bool double_entries, cudaStream_t s,
                          const std::function<void(cudaStream_t)>& with_list) {
  const int tb = 256;
  const int ga = ceil_div(a.n_atoms, tb);
  const int block_cap = a.slot_capacity / 32;
  nl_columns<<<ga, tb, 0, s>>>(a);
  nl_col_scan<<<1, 1024, 0, s>>>(a);
  nl_col_scatter<<<ga, tb, 0, s>>>(a);
  int m = 1;
  while (m < a.col_max) m <<= 1;
  nl_col_sort<<<a.n_cols, 256, sizeof(unsigned long long) * m, s>>>(a);
  nl_bounds<<<ceil_div((long long)block_cap * 32, tb), tb, 0, s>>>(a);
  const bool rectangular = a.periodic && a.box.bx == 0.0 && a.box.cx == 0.0 && a.box.cy == 0.0;
  if (rectangular && a.max_cand > 0 && a.halves) {
    const size_t bytes = (size_t)a.max_cand * (3 * 8 + 4 + 4 + 2 * 4 + 2 * 4) + 8;
    if (double_entries) {
      cudaFuncSetAttribute(nl_lists_cta<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      nl_lists_cta<true><<<block_cap, 32 * kCtaWarps, bytes, s>>>(a);
    } else {
      cudaFuncSetAttribute(nl_lists_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      nl_lists_cta<false><<<block_cap, 32 * kCtaWarps, bytes, s>>>(a);
    }
  } else {
    const int gl = ceil_div(block_cap, kListWarps);
    if (double_entries)
      nl_lists<true><<<gl, 32 * kListWarps, 0, s>>>(a);
    else
      nl_lists<false><<<gl, 32 * kListWarps, 0, s>>>(a);
  }
  if (with_list) with_list(s);
  nl_finish<<<std::max(1, std::min(ceil_div(a.n_cols, tb), 148 * 4)), tb, 0, s>>>(a);
  nl_clear_flag<<<1, 1, 0, s>>>(a);
}

}  // namespace ommb200
