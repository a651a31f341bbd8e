// Learned Born radii for GBSAOBCForce (no reference counterpart; the OBC terms follow
// forces/gbsa_obc.rs:184-309).  The HCT integral of particle i is split as
//   I_i = I_short_i + tail_i,   I_short_i = sum_j H(r_ij; rho_i, s_j) S(r_ij)
// with S the quintic switch from rs to rc (1.8 -> 2.0 nm), and tail_i predicted by the radii
// network (radii_mlp.cu) from 32 radial symmetry functions (Behler & Parrinello, Phys. Rev.
// Lett. 98, 146401 (2007)) G_if = sum_j exp(-eta (r_ij - mu_f)^2) fc(r_ij) over r_ij < rf =
// 1.2 nm, fc(r) = (cos(pi r / rf) + 1) / 2.
// Everything here is short-ranged: per 32-slot block a list of the blocks of its segment whose
// boxes come within rc, then one CTA per block gathers features and I_short (front), visiting
// each ordered pair from the i side only, so each particle's sums belong to one lane per warp
// and meet in a fixed order; or the forces -dE/dx through I_short and the network (back), once
// per pair with the j side's share committed in fixed point.
//
// The exact pass still runs every `judge_interval` MD steps as the judge: it supplies that
// step's radii, the network is compared with it (largest per-particle radius relative error),
// the particles' features and exact tails become the training snapshot, and a few Adam steps
// follow unless the network's error is already within half the tolerance.  Until the next
// judge the network's radii are used only if it passed (error below `tolerance`); otherwise
// the exact passes run.
#include "gb_math.cuh"
#include "kernels.h"
#include "pair_math.cuh"

namespace ommb200 {
namespace {

using namespace gb;

constexpr int kNF = kRadiiFeatures;
constexpr int kWarps = 4;
constexpr float kMu0 = 0.1f;               // first Gaussian centre (nm)
constexpr float kDmu = 1.1f / 31.0f;       // centre spacing: 0.1 .. 1.2 nm
constexpr float kEta = 1.0f / (2.0f * 0.07f * 0.07f);  // Gaussian width 0.07 nm
constexpr float kPiF = 3.14159265358979f;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float switch_value(float r, float rs, float rc, float* deriv) {
  if (r <= rs) {
    *deriv = 0.f;
    return 1.f;
  }
  const float inv_w = rcp_r(rc - rs), t = (r - rs) * inv_w;
  *deriv = -30.f * t * t * (1.f - t) * (1.f - t) * inv_w;
  return 1.f + t * t * t * (-10.f + t * (15.f - 6.f * t));
}

// gbsa_obc.rs:278-309 with SFU reciprocals and logarithm: the descreening integral H and the
// derivative factor G (dH/dr = -2 r G) of one ordered pair.
__device__ __forceinline__ float3 position(const double* pos, int atom) {
  return make_float3((float)pos[3 * atom], (float)pos[3 * atom + 1], (float)pos[3 * atom + 2]);
}

__global__ void lr_control(LearnedGbArgs a, int judge_allowed, int step_offset) {
  LearnedState* st = a.state;
  const unsigned long long step = *a.step + (unsigned long long)step_offset;
  const int judge = judge_allowed && (step % (unsigned long long)a.judge_interval == 0ull);
  const int use = st->active && !judge;
  st->judge = judge;
  st->use_learned = use;
  st->need = use | judge;
  if (judge_allowed) {
    if (use)
      st->learned_evals += 1;
    else
      st->exact_evals += 1;
  }
  if (judge) {
    st->judges += 1;
    st->max_err_bits = 0u;
  }
}

// One warp per block: bounding box of its particles.
__global__ void lr_boxes(LearnedGbArgs a, GbArgs g) {
  if (!a.state->need) return;
  const int lane = threadIdx.x & 31;
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (b >= a.n_blocks) return;
  const int atom = g.slot_atom[32 * b + lane];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (atom >= 0) {
    const float3 p = position(g.pos, atom);
    lo[0] = hi[0] = p.x;
    lo[1] = hi[1] = p.y;
    lo[2] = hi[2] = p.z;
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(kFull, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(kFull, hi[d], o));
    }
  if (lane == 0) {
    a.block_box[2 * b] = make_float4(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]),
                                     0.5f * (lo[2] + hi[2]), 0.f);
    a.block_box[2 * b + 1] = make_float4(0.5f * (hi[0] - lo[0]), 0.5f * (hi[1] - lo[1]),
                                         0.5f * (hi[2] - lo[2]), 0.f);
  }
}

// One warp per block I: the blocks of I's segment whose boxes come within rf of I's box ("near":
// features and integral; stored from the front of I's row, I itself included) and those
// within rc but not rf ("far": integral only; stored from the back), in block order.
__global__ void lr_neighbors(LearnedGbArgs a) {
  if (!a.state->need) return;
  const int lane = threadIdx.x & 31;
  const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (I >= a.n_blocks) return;
  const float4 ci = a.block_box[2 * I], hi = a.block_box[2 * I + 1];
  const int first = a.block_first[I], count = a.block_count[I];
  const float rc2 = a.rc * a.rc, rf2 = a.rf * a.rf;
  int* row = a.nbr + (size_t)I * a.max_nbr;
  int n_near = 0, n_far = 0;
  for (int base = 0; base < count; base += 32) {
    const int J = first + base + lane;
    float gap2 = INFINITY;
    if (base + lane < count) {
      const float4 cj = a.block_box[2 * J], hj = a.block_box[2 * J + 1];
      const float gx = fmaxf(fabsf(cj.x - ci.x) - hi.x - hj.x, 0.f);
      const float gy = fmaxf(fabsf(cj.y - ci.y) - hi.y - hj.y, 0.f);
      const float gz = fmaxf(fabsf(cj.z - ci.z) - hi.z - hj.z, 0.f);
      gap2 = gx * gx + gy * gy + gz * gz;
    }
    const bool near = gap2 < rf2, far = !near && gap2 < rc2;
    const unsigned mn = __ballot_sync(kFull, near), mf = __ballot_sync(kFull, far);
    const unsigned below = (1u << lane) - 1u;
    // a segment has at most max_nbr blocks, so the two ends never meet
    if (near) row[n_near + __popc(mn & below)] = J;
    if (far) row[a.max_nbr - 1 - (n_far + __popc(mf & below))] = J;
    n_near += __popc(mn);
    n_far += __popc(mf);
  }
  if (lane == 0) {
    a.nbr_count[2 * I] = n_near;
    a.nbr_count[2 * I + 1] = n_far;
  }
}

// Block J and whether it is near, for entry q of I's lists (near entries first).
__device__ __forceinline__ int list_block(const LearnedGbArgs& a, int I, int q, int n_near,
                                          bool* near) {
  *near = q < n_near;
  const int* row = a.nbr + (size_t)I * a.max_nbr;
  return *near ? row[q] : row[a.max_nbr - 1 - (q - n_near)];
}

// e_f = exp(-eta (r - mu_f)^2) for all f from three exponentials: the centre f = 15 and the
// first ratios of neighbouring Gaussians, which then change by q = exp(-2 eta dmu^2) per step.
// Every e_f is at most 1 and, for r < 1.2 nm, e_15 stays far above the FP32 range limit.
__device__ __forceinline__ void gaussians(float r, float q, float* e) {
  constexpr int c = 15;
  const float x = r - (kMu0 + c * kDmu);
  const float a = 2.f * kEta * kDmu * x, b = kEta * kDmu * kDmu;
  e[c] = __expf(-kEta * x * x);
  float up = __expf(a - b), down = __expf(-a - b);
#pragma unroll
  for (int f = c + 1; f < kNF; ++f) {
    e[f] = e[f - 1] * up;
    up *= q;
  }
#pragma unroll
  for (int f = c - 1; f >= 0; --f) {
    e[f] = e[f + 1] * down;
    down *= q;
  }
}

// One CTA per block I, lane = particle i; the CTA's warps share I's near / far list and their
// partial sums meet in shared memory in a fixed order.  Radial features (near blocks, r < rf)
// and the switched short-range integral (r < rc) over every particle j != i.
__global__ void __launch_bounds__(32 * kWarps) lr_features(LearnedGbArgs a, GbArgs g) {
  if (!a.state->need) return;
  __shared__ float4 s_pos[kWarps][32];  // xyz, 1 for a particle / 0 for padding
  __shared__ float s_scaled[kWarps][32];
  __shared__ float s_red[kWarps][32][kNF + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const float rc2 = a.rc * a.rc, rf2 = a.rf * a.rf;
  const float q = __expf(-2.f * kEta * kDmu * kDmu);
  const float fc_k = kPiF / a.rf;
  for (int I = blockIdx.x; I < a.n_blocks; I += gridDim.x) {
    const int ai = g.slot_atom[32 * I + lane];
    float3 pi = make_float3(0.f, 0.f, 0.f);
    float off_i = 1.f;
    if (ai >= 0) {
      pi = position(g.pos, ai);
      off_i = (float)(g.radius[ai] - kDielectricOffset);
    }
    float G[kNF];
#pragma unroll
    for (int f = 0; f < kNF; ++f) G[f] = 0.f;
    float ishort = 0.f;
    const int n_near = a.nbr_count[2 * I], nn = n_near + a.nbr_count[2 * I + 1];
    for (int it = w; it < nn; it += kWarps) {
      bool near;
      const int J = list_block(a, I, it, n_near, &near);
      const int aj = g.slot_atom[32 * J + lane];
      if (aj >= 0) {
        const float3 p = position(g.pos, aj);
        s_pos[w][lane] = make_float4(p.x, p.y, p.z, 1.f);
        s_scaled[w][lane] = (float)((g.radius[aj] - kDielectricOffset) * g.scale[aj]);
      } else {
        s_pos[w][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        s_scaled[w][lane] = 0.f;
      }
      __syncwarp();
      if (ai >= 0) {
        for (int k = 0; k < 32; ++k) {
          const int jl = (lane + k) & 31;
          const float4 pj = s_pos[w][jl];
          if (pj.w == 0.f || (J == I && jl == lane)) continue;
          const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
          const float r2 = dx * dx + dy * dy + dz * dz;
          if (r2 >= rc2) continue;
          const float inv_r = rsqrt_r(r2), r = r2 * inv_r;
          float ds, h, gr;
          const float sw = switch_value(r, a.rs, a.rc, &ds);
          descreening_fast(off_i, s_scaled[w][jl], r, inv_r, &h, &gr);
          ishort = fmaf(h, sw, ishort);
          if (!near || r2 >= rf2) continue;
          const float fc = 0.5f * (__cosf(fc_k * r) + 1.f);  // SFU cosine
          float e[kNF];
          gaussians(r, q, e);
#pragma unroll
          for (int f = 0; f < kNF; ++f) G[f] = fmaf(e[f], fc, G[f]);
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int f = 0; f < kNF; ++f) s_red[w][lane][f] = G[f];
    s_red[w][lane][kNF] = ishort;
    __syncthreads();
    if (w == 0 && ai >= 0) {
      float4* out = reinterpret_cast<float4*>(a.features + (size_t)ai * kNF);
      float v[kNF + 1];
#pragma unroll
      for (int f = 0; f <= kNF; ++f) {
        float t = s_red[0][lane][f];
        for (int u = 1; u < kWarps; ++u) t += s_red[u][lane][f];
        v[f] = t;
      }
#pragma unroll
      for (int f = 0; f < kNF / 4; ++f)
        out[f] = make_float4(v[4 * f], v[4 * f + 1], v[4 * f + 2], v[4 * f + 3]);
      a.short_sum[ai] = to_fixed((double)v[kNF], kBornScale);
    }
    __syncthreads();
  }
}

// One CTA per block I as above: F_i = sum_j (D_i Phi'_ij + D_j Phi'_ji) / r d_ij,
// Phi_ij = H(r; i, j) S(r) + sum_f (d tail_i / d G_if) g_f(r), D = dE/dI (half the chain
// value the GB chain kernel leaves per slot).  The pair term is symmetric in i and j, so each
// pair of blocks is done once, from the lower block (J >= I in I's list): the force on each
// entry of J travels with it one lane per warp shuffle and is committed in fixed point after
// the 32 steps; the self block visits each pair from both sides and keeps i-forces only.
template <class Real>
__global__ void __launch_bounds__(32 * kWarps) lr_forces(LearnedGbArgs a, GbArgs g) {
  if (!a.state->use_learned) return;
  __shared__ float4 s_pos[kWarps][32];
  __shared__ float4 s_par[kWarps][32];        // offset radius, scaled radius, D, valid
  __shared__ float s_w[kWarps][32][kNF + 1];  // D_j d tail_j / d G_j (padded rows)
  __shared__ float s_red[kWarps][32][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const float rc2 = a.rc * a.rc, rf2 = a.rf * a.rf;
  const Real* chain = reinterpret_cast<const Real*>(g.dedr_slot);
  const float fc_k = kPiF / a.rf;
  const float q = __expf(-2.f * kEta * kDmu * kDmu);
  const float fscale = (float)kForceScale;
  for (int I = blockIdx.x; I < a.n_blocks; I += gridDim.x) {
    const int si = 32 * I + lane;
    const int ai = g.slot_atom[si];
    float3 pi = make_float3(0.f, 0.f, 0.f);
    float off_i = 1.f, sc_i = 0.f, d_i = 0.f;
    float wi[kNF];
#pragma unroll
    for (int f = 0; f < kNF; ++f) wi[f] = 0.f;
    if (ai >= 0) {
      pi = position(g.pos, ai);
      off_i = (float)(g.radius[ai] - kDielectricOffset);
      sc_i = (float)((g.radius[ai] - kDielectricOffset) * g.scale[ai]);
      d_i = 0.5f * (float)chain[si];
      const float4* dt = reinterpret_cast<const float4*>(a.dtail + (size_t)ai * kNF);
#pragma unroll
      for (int qq = 0; qq < kNF / 4; ++qq) {
        const float4 v = dt[qq];
        wi[4 * qq] = d_i * v.x;
        wi[4 * qq + 1] = d_i * v.y;
        wi[4 * qq + 2] = d_i * v.z;
        wi[4 * qq + 3] = d_i * v.w;
      }
    }
    float fx = 0.f, fy = 0.f, fz = 0.f;
    const int n_near = a.nbr_count[2 * I], nn = n_near + a.nbr_count[2 * I + 1];
    for (int it = w; it < nn; it += kWarps) {
      bool near;
      const int J = list_block(a, I, it, n_near, &near);
      if (J < I) continue;  // done from block J's side
      const bool self = J == I;
      const int sj = 32 * J + lane;
      const int aj = g.slot_atom[sj];
      if (aj >= 0) {
        const float3 p = position(g.pos, aj);
        const float off = (float)(g.radius[aj] - kDielectricOffset);
        const float dj = 0.5f * (float)chain[sj];
        s_pos[w][lane] = make_float4(p.x, p.y, p.z, 1.f);
        s_par[w][lane] = make_float4(off, (float)((g.radius[aj] - kDielectricOffset) * g.scale[aj]),
                                     dj, 1.f);
        if (near) {
          const float4* dt = reinterpret_cast<const float4*>(a.dtail + (size_t)aj * kNF);
#pragma unroll
          for (int qq = 0; qq < kNF / 4; ++qq) {
            const float4 v = dt[qq];
            s_w[w][lane][4 * qq] = dj * v.x;
            s_w[w][lane][4 * qq + 1] = dj * v.y;
            s_w[w][lane][4 * qq + 2] = dj * v.z;
            s_w[w][lane][4 * qq + 3] = dj * v.w;
          }
        }
      } else {
        s_pos[w][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        s_par[w][lane] = make_float4(1.f, 0.f, 0.f, 0.f);
      }
      __syncwarp();
      float gx = 0.f, gy = 0.f, gz = 0.f;  // force on the entry now in this lane's rotation
      const int src = (lane + 1) & 31;
      for (int k = self ? 1 : 0; k < 32; ++k) {
        const int jl = (lane + k) & 31;
        const float4 pj = s_pos[w][jl];
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        float radial = 0.f;
        if (ai >= 0 && pj.w != 0.f && r2 < rc2) {
          const float inv_r = rsqrt_r(r2), r = r2 * inv_r;
          const float4 pr = s_par[w][jl];
          float ds, hij, hji, gij, gji;
          const float sw = switch_value(r, a.rs, a.rc, &ds);
          // dH/dr = -2 r descreening_gradient (gbsa_obc.rs:297-309)
          descreening_fast(off_i, pr.y, r, inv_r, &hij, &gij);
          descreening_fast(pr.x, sc_i, r, inv_r, &hji, &gji);
          float phi = d_i * (-2.f * r * gij * sw + hij * ds) + pr.z * (-2.f * r * gji * sw + hji * ds);
          if (near && r2 < rf2) {
            float sn, cs;
            __sincosf(fc_k * r, &sn, &cs);  // SFU sine and cosine
            const float fc = 0.5f * (cs + 1.f), dfc = -0.5f * fc_k * sn;
            float e[kNF];
            gaussians(r, q, e);
            // sum_f W_f g_f'(r),  g_f' = e_f (-2 eta (r - mu_f) fc + dfc)
            float s0 = 0.f, s1 = 0.f;
#pragma unroll
            for (int f = 0; f < kNF; ++f) {
              const float we = (wi[f] + s_w[w][jl][f]) * e[f];
              s0 += we;
              s1 = fmaf(we, r - (kMu0 + f * kDmu), s1);
            }
            phi += dfc * s0 - 2.f * kEta * fc * s1;
          }
          radial = phi * inv_r;
        }
        fx = fmaf(radial, dx, fx);
        fy = fmaf(radial, dy, fy);
        fz = fmaf(radial, dz, fz);
        if (!self) {
          gx = fmaf(-radial, dx, gx);
          gy = fmaf(-radial, dy, gy);
          gz = fmaf(-radial, dz, gz);
          gx = __shfl_sync(kFull, gx, src);
          gy = __shfl_sync(kFull, gy, src);
          gz = __shfl_sync(kFull, gz, src);
        }
      }
      if (!self && aj >= 0) {
        add_fixed(g.force + aj, to_fixed(gx, fscale));
        add_fixed(g.force + g.n_atoms + aj, to_fixed(gy, fscale));
        add_fixed(g.force + 2 * g.n_atoms + aj, to_fixed(gz, fscale));
      }
      __syncwarp();
    }
    s_red[w][lane][0] = fx;
    s_red[w][lane][1] = fy;
    s_red[w][lane][2] = fz;
    __syncthreads();
    if (w == 0 && ai >= 0) {
      float f3[3];
      for (int c = 0; c < 3; ++c) {
        float t = s_red[0][lane][c];
        for (int u = 1; u < kWarps; ++u) t += s_red[u][lane][c];
        f3[c] = t;
      }
      add_fixed(g.force + ai, to_fixed(f3[0], fscale));
      add_fixed(g.force + g.n_atoms + ai, to_fixed(f3[1], fscale));
      add_fixed(g.force + 2 * g.n_atoms + ai, to_fixed(f3[2], fscale));
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double obc_radius(double integral, double rho) {
  const double offset = rho - kDielectricOffset;
  const double psi = 0.5 * offset * integral;
  const double t = tanh(psi - 0.8 * psi * psi + 4.85 * psi * psi * psi);
  return 1.0 / (1.0 / offset - t / rho);
}

// Judge: radius error of the network against the exact integral, and the training snapshot.
__global__ void lr_judge(LearnedGbArgs a, GbArgs g) {
  if (!a.state->judge) return;
  const int atom = blockIdx.x * blockDim.x + threadIdx.x;
  if (atom >= a.n_atoms) return;
  const double rho = g.radius[atom];
  const double exact = (double)g.born_sum[atom] * kBornScaleInv;
  const double shrt = (double)a.short_sum[atom] * kBornScaleInv;
  const double re = obc_radius(exact, rho);
  const double rl =
      obc_radius(shrt + (double)a.tail[atom] + (double)a.seg_offset[g.atom_segment[atom]], rho);
  float err = (float)fabs((rl - re) / re);
  if (!(err <= 1e30f)) err = 1e30f;
  atomicMax(&a.state->max_err_bits, __float_as_uint(err));
  const float4* src = reinterpret_cast<const float4*>(a.features + (size_t)atom * kNF);
  float4* dst = reinterpret_cast<float4*>(a.snap_features + (size_t)atom * kNF);
#pragma unroll
  for (int q = 0; q < kNF / 4; ++q) dst[q] = src[q];
  a.snap_target[atom] = (float)(exact - shrt);
}

// After training, one block per system: the constant tail offset that makes the first-order
// GB energy error of the retrained network vanish at the main configuration,
//   offset = sum_i D_i (exact_i - tail_i) / sum_i D_i,  D_i = dE/dI_i,
// (the plain mean difference when the D_i nearly cancel).  The offset is fixed until the next
// judge, so it shifts the energy and radii but not the forces' consistency.
__global__ void __launch_bounds__(256) lr_offsets(LearnedGbArgs a, GbArgs g) {
  if (!a.state->judge) return;
  __shared__ double s_v[3][256];
  const int seg = blockIdx.x, t = threadIdx.x;
  const int first = a.seg_first[seg], count = a.seg_count[seg];
  double num = 0.0, den = 0.0, mag = 0.0, diff = 0.0;
  for (int i = first + t; i < first + count; i += 256) {
    const double R = g.born_radius[i];
    const double d = 0.5 * (g.dedr_self[i] + (double)g.dedr_sum[i] * kForceScaleInv) * R * R *
                     g.chain[i];
    const double e = (double)a.snap_target[i] - (double)a.tail[i];
    num += d * e;
    den += d;
    mag += fabs(d);
    diff += e;
  }
  double v[4] = {num, den, mag, diff};
  for (int k = 0; k < 4; ++k) {
    __syncthreads();
    s_v[0][t] = v[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (t < o) s_v[0][t] += s_v[0][t + o];
      __syncthreads();
    }
    v[k] = s_v[0][0];
  }
  if (t == 0)
    a.seg_offset[seg] = (float)(fabs(v[1]) > 1e-3 * v[2] ? v[0] / v[1] : v[3] / count);
}

__global__ void lr_judge_finish(LearnedGbArgs a) {
  LearnedState* st = a.state;
  if (!st->judge) return;
  const float err = __uint_as_float(st->max_err_bits);
  st->last_error = err;
  st->active = st->initialized && err <= a.tolerance;
  // a network within half the tolerance keeps its weights (the offsets are still refitted)
  st->train = !st->initialized || !(err <= 0.5f * a.tolerance);
}

// First judge only: feature and target normalisation from the snapshot (fixed afterwards),
// by a fixed-order block reduction.
__global__ void __launch_bounds__(256) lr_normalize(LearnedGbArgs a) {
  LearnedState* st = a.state;
  if (!st->judge || st->initialized) return;
  __shared__ double s_sum[256], s_sq[256];
  const int t = threadIdx.x;
  for (int q = 0; q <= kNF; ++q) {  // q == kNF: the target
    double sum = 0.0, sq = 0.0;
    for (int i = t; i < a.n_atoms; i += 256) {
      const double v = q < kNF ? (double)a.snap_features[(size_t)i * kNF + q] : (double)a.snap_target[i];
      sum += v;
      sq += v * v;
    }
    s_sum[t] = sum;
    s_sq[t] = sq;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (t < o) {
        s_sum[t] += s_sum[t + o];
        s_sq[t] += s_sq[t + o];
      }
      __syncthreads();
    }
    if (t == 0) {
      const double mean = s_sum[0] / a.n_atoms;
      const double var = fmax(s_sq[0] / a.n_atoms - mean * mean, 0.0);
      const double sd = sqrt(var);
      if (q < kNF) {
        a.params[kRadiiMlpOffMean + q] = (float)mean;
        a.params[kRadiiMlpOffInvStd + q] = (float)(1.0 / fmax(sd, 1e-3));
      } else {
        a.params[kRadiiMlpOffTMean] = (float)mean;
        a.params[kRadiiMlpOffTScale] = (float)fmax(sd, 1e-6);
        st->initialized = 1;
      }
    }
    __syncthreads();
  }
}

}  // namespace

void launch_learned_control(const LearnedGbArgs& a, bool judge_allowed, int step_offset,
                            cudaStream_t s) {
  lr_control<<<1, 1, 0, s>>>(a, judge_allowed ? 1 : 0, step_offset);
}

template <class Real>
void launch_learned_phase(const LearnedGbArgs& a, const GbArgs& g, int phase, int sm_count,
                          cudaStream_t s) {
  const int wb = ceil_div(a.n_blocks * 32, 128);
  const int ctas = std::max(1, a.n_blocks);  // one CTA per block: the scheduler balances uneven lists
  switch (phase) {
    case kLrLists:
      lr_boxes<<<wb, 128, 0, s>>>(a, g);
      lr_neighbors<<<wb, 128, 0, s>>>(a);
      break;
    case kLrFeatures:
      lr_features<<<ctas, 32 * kWarps, 0, s>>>(a, g);
      break;
    case kLrInfer:
      launch_mlp_infer(a.n_atoms, a.features, a.params, a.tail, a.dtail, a.status, sm_count, s,
                       &a.state->need);
      break;
    case kLrForces:
      lr_forces<Real><<<ctas, 32 * kWarps, 0, s>>>(a, g);
      break;
    case kLrJudge:
      lr_judge<<<ceil_div(a.n_atoms, 256), 256, 0, s>>>(a, g);
      lr_judge_finish<<<1, 1, 0, s>>>(a);
      lr_normalize<<<1, 256, 0, s>>>(a);
      break;
    case kLrTrain:
      launch_mlp_train(a.n_atoms, a.snap_features, a.snap_target, a.params, a.moments,
                       a.moments + kRadiiMlpTrainable, a.adam_t, a.train_steps, a.batch,
                       a.learning_rate, a.seed, nullptr, a.loss, a.status, s, &a.state->train);
      break;
    case kLrOffsets:
      // the retrained network on the main configuration, then the per-system offsets
      launch_mlp_infer(a.n_atoms, a.snap_features, a.params, a.tail, nullptr, a.status, sm_count,
                       s, &a.state->judge);
      lr_offsets<<<a.n_segments, 256, 0, s>>>(a, g);
      break;
  }
}

template void launch_learned_phase<float>(const LearnedGbArgs&, const GbArgs&, int, int,
                                          cudaStream_t);
template void launch_learned_phase<double>(const LearnedGbArgs&, const GbArgs&, int, int,
                                           cudaStream_t);

}  // namespace ommb200
