// Neighbour tiles for periodic cutoff methods.
//
// The reference enumerates candidate pairs from a linked-list cell grid rebuilt at every
// evaluation (forces/neighbors.rs:96-181) and tests each pair against r^2 < rc^2
// (forces/nonbonded.rs:862).  Here particles are sorted into 32-slot blocks along a Morton
// curve of small voxels, block bounding boxes are computed, and every block pair whose boxes
// come within cutoff + skin becomes a tile.  The list is rebuilt only when some particle has
// moved more than skin/2 since the last rebuild (the integrator raises `rebuild`), so every
// pair inside the cutoff at any step in between is covered by a tile; the pair kernel applies
// the reference's exact cutoff test, which makes the interacting pair set the reference's.
//
// Every kernel returns at once unless `rebuild` is set, so the sequence can sit in a CUDA
// graph that is replayed every step.  The sort is a stable counting sort (ties broken by
// particle index), so the slot order, and with it every force sum, is deterministic.
#include "kernels.h"

namespace ommb200 {
namespace {

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void nl_keys(NlistArgs a) {
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
  const int vx = min(max((int)(x * b.inv_ax * a.n_vox[0]), 0), a.n_vox[0] - 1);
  const int vy = min(max((int)(y * b.inv_by * a.n_vox[1]), 0), a.n_vox[1] - 1);
  const int vz = min(max((int)(z * b.inv_cz * a.n_vox[2]), 0), a.n_vox[2] - 1);
  const int key = (int)(spread_bits(vx) | (spread_bits(vy) << 1) | (spread_bits(vz) << 2));
  a.key[i] = key;
  atomicAdd(&a.key_count[key], 1);
}

// Single-CTA exclusive scan of the voxel counts.
__global__ void __launch_bounds__(1024) nl_scan(NlistArgs a) {
  if (*a.rebuild == 0) return;
  __shared__ int partial[1024];
  const int t = threadIdx.x;
  const int chunk = (a.n_keys + 1023) / 1024;
  const int lo = min(t * chunk, a.n_keys), hi = min(lo + chunk, a.n_keys);
  int sum = 0;
  for (int k = lo; k < hi; ++k) sum += a.key_count[k];
  partial[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int v = t >= off ? partial[t - off] : 0;
    __syncthreads();
    partial[t] += v;
    __syncthreads();
  }
  int run = partial[t] - sum;
  for (int k = lo; k < hi; ++k) {
    a.key_start[k] = run;
    run += a.key_count[k];
  }
  if (t == 1023) a.key_start[a.n_keys] = partial[1023];
}

__global__ void nl_scatter(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms) return;
  const int key = a.key[i];
  const int slot = a.key_start[key] + atomicAdd(&a.key_cursor[key], 1);
  a.scratch_atoms[slot] = i;
}

// Stable order inside each voxel: rank = number of voxel members with a smaller index.
__global__ void nl_order(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms) return;
  const int key = a.key[i];
  const int s0 = a.key_start[key], c = a.key_count[key];
  int rank = 0;
  for (int k = 0; k < c; ++k) rank += a.scratch_atoms[s0 + k] < i;
  a.sorted_atom[s0 + rank] = i;
  a.atom_slot[i] = s0 + rank;
}

// One warp per block: bounding box of the wrapped rebuild positions.
__global__ void nl_bounds(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int lane = threadIdx.x & 31;
  const int blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (blk >= a.n_blocks) return;
  const int atom = a.sorted_atom[32 * blk + lane];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (atom >= 0) {
    const Box<double>& b = a.box;
    const double n0 = a.image[3 * atom], n1 = a.image[3 * atom + 1], n2 = a.image[3 * atom + 2];
    const double w[3] = {a.pos_ref[3 * atom] - (n0 * b.ax + n1 * b.bx + n2 * b.cx),
                         a.pos_ref[3 * atom + 1] - (n1 * b.by + n2 * b.cy),
                         a.pos_ref[3 * atom + 2] - n2 * b.cz};
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = w[d];
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
    }
  if (lane == 0)
    for (int d = 0; d < 3; ++d) {
      a.block_center[3 * blk + d] = 0.5 * (lo[d] + hi[d]);
      a.block_half[3 * blk + d] = 0.5 * (hi[d] - lo[d]);
    }
}

__device__ __forceinline__ double box_gap2(const double d[3], const double* hi, const double* hj) {
  double s = 0.0;
  for (int k = 0; k < 3; ++k) {
    double g = fabs(d[k]) - hi[k] - hj[k];
    g = g > 0.0 ? g : 0.0;
    s += g * g;
  }
  return s;
}

// One thread per block pair (I <= J).
template <bool kDoubleShift>
__global__ void nl_tiles(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const long long nb = a.n_blocks;
  const long long total = nb * (nb + 1) / 2;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total;
       p += (long long)gridDim.x * blockDim.x) {
    // row I holds pairs (I, I..nb-1); rows start at I*nb - I(I-1)/2
    long long I = (long long)((2.0 * nb + 1.0 - sqrt((2.0 * nb + 1.0) * (2.0 * nb + 1.0) - 8.0 * p)) * 0.5);
    if (I < 0) I = 0;
    if (I >= nb) I = nb - 1;
    while (I > 0 && I * nb - I * (I - 1) / 2 > p) --I;
    while (I + 1 < nb && (I + 1) * nb - (I + 1) * I / 2 <= p) ++I;
    const long long J = I + (p - (I * nb - I * (I - 1) / 2));
    const double* ci = a.block_center + 3 * I;
    const double* cj = a.block_center + 3 * J;
    const double* hi = a.block_half + 3 * I;
    const double* hj = a.block_half + 3 * J;
    double d[3] = {cj[0] - ci[0], cj[1] - ci[1], cj[2] - ci[2]};
    const Box<double>& b = a.box;
    if (a.periodic) min_image_fast(d[0], d[1], d[2], b);
    const double reach = a.cutoff + a.skin;
    const double ri = sqrt(hi[0] * hi[0] + hi[1] * hi[1] + hi[2] * hi[2]);
    const double rj = sqrt(hj[0] * hj[0] + hj[1] * hj[1] + hj[2] * hj[2]);
    bool safe = true;
    double best = box_gap2(d, hi, hj);
    if (a.periodic) {
      const double need = reach + ri + rj;
      for (int m0 = -1; m0 <= 1; ++m0)
        for (int m1 = -1; m1 <= 1; ++m1)
          for (int m2 = -1; m2 <= 1; ++m2) {
            if (m0 == 0 && m1 == 0 && m2 == 0) continue;
            const double e[3] = {d[0] + m0 * b.ax + m1 * b.bx + m2 * b.cx,
                                 d[1] + m1 * b.by + m2 * b.cy, d[2] + m2 * b.cz};
            if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] < need * need) safe = false;
            best = fmin(best, box_gap2(e, hi, hj));
          }
    }
    const double gap2 = safe ? box_gap2(d, hi, hj) : best;
    if (I != J && gap2 >= reach * reach) continue;
    const int t = atomicAdd(a.n_tiles, 1);
    if (t >= a.tile_capacity) {
      report_status(a.status, kStatusTileOverflow);
      continue;
    }
    a.tiles[t] = make_int4((int)I, (int)J, safe ? 0 : kTilePairImage, -1);
    if (kDoubleShift)
      reinterpret_cast<double4*>(a.tile_shift)[t] = make_double4(d[0], d[1], d[2], 0.0);
    else
      reinterpret_cast<float4*>(a.tile_shift)[t] =
          make_float4((float)d[0], (float)d[1], (float)d[2], 0.0f);
  }
}

// One warp per tile: exclusion and padding masks (bit m of lane l: skip pair (l, m)).
__global__ void nl_masks(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int lane = threadIdx.x & 31;
  const int nt = min(*a.n_tiles, a.tile_capacity);
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nt;
       t += (gridDim.x * blockDim.x) >> 5) {
    const int4 tile = a.tiles[t];
    const int ai = a.sorted_atom[32 * tile.x + lane];
    const int aj = a.sorted_atom[32 * tile.y + lane];
    uint32_t mask = __ballot_sync(0xffffffffu, aj < 0);
    if (ai < 0) {
      mask = 0xffffffffu;
    } else {
      for (int k = a.excl_start[ai]; k < a.excl_start[ai + 1]; ++k) {
        const int s = a.atom_slot[a.excl_list[k]];
        if ((s >> 5) == tile.y) mask |= 1u << (s & 31);
      }
    }
    if (__any_sync(0xffffffffu, mask != 0)) {
      int slot = 0;
      if (lane == 0) slot = atomicAdd(a.n_masks, 1);
      slot = __shfl_sync(0xffffffffu, slot, 0);
      if (slot < a.mask_capacity) {
        a.masks[32 * slot + lane] = mask;
        if (lane == 0) a.tiles[t] = make_int4(tile.x, tile.y, tile.z | kTileHasMask, slot);
      } else if (lane == 0) {
        report_status(a.status, kStatusTileOverflow);
      }
    }
  }
}

__global__ void nl_finish(NlistArgs a) {
  if (*a.rebuild == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = i; k < a.n_keys; k += gridDim.x * blockDim.x) {
    a.key_count[k] = 0;
    a.key_cursor[k] = 0;
  }
}

__global__ void nl_clear_flag(int* rebuild) { *rebuild = 0; }

}  // namespace

void launch_nlist_rebuild(const NlistArgs& a, bool double_shift, cudaStream_t s) {
  const int tb = 256;
  const int ga = ceil_div(a.n_atoms, tb);
  nl_keys<<<ga, tb, 0, s>>>(a);
  nl_scan<<<1, 1024, 0, s>>>(a);
  nl_scatter<<<ga, tb, 0, s>>>(a);
  nl_order<<<ga, tb, 0, s>>>(a);
  nl_bounds<<<ceil_div((long long)a.n_blocks * 32, tb), tb, 0, s>>>(a);
  const long long pairs = (long long)a.n_blocks * (a.n_blocks + 1) / 2;
  const int gt = (int)std::min<long long>((pairs + tb - 1) / tb, 148LL * 64);
  if (double_shift)
    nl_tiles<true><<<gt, tb, 0, s>>>(a);
  else
    nl_tiles<false><<<gt, tb, 0, s>>>(a);
  nl_masks<<<148 * 8, tb, 0, s>>>(a);
  nl_finish<<<std::min(ceil_div(a.n_keys, tb), 148 * 4), tb, 0, s>>>(a);
  nl_clear_flag<<<1, 1, 0, s>>>(a.rebuild);
}

}  // namespace ommb200
