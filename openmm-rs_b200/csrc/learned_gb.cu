// Learned Born radii for GBSAOBCForce (no reference counterpart; the OBC terms follow
// forces/gbsa_obc.rs:184-309).  The HCT integral of particle i is split as
//   I_i = I_short_i + tail_i,   I_short_i = sum_j H(r_ij; rho_i, s_j) S(r_ij)
// with S the quintic switch from rs to rc (1.8 -> 2.0 nm), and tail_i predicted by the radii
// network (radii_mlp.cu) from 32 radial symmetry functions (Behler & Parrinello, Phys. Rev.
// Lett. 98, 146401 (2007)) G_if = sum_j exp(-eta (r_ij - mu_f)^2) fc(r_ij) over r_ij < rf =
// 1.2 nm, fc(r) = (cos(pi r / rf) + 1) / 2.
// Everything here is short-ranged: per 32-slot block a list of the blocks of its segment whose
// boxes come within rc; one CTA per block sorts those blocks' particles into lists per half of
// the block (within rf or rc of the half's box) and gathers features and I_short (front),
// visiting each ordered pair from the i side only, so each particle's sums belong to one lane per warp
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

// e_f = exp(-eta (r - mu_f)^2) around the centre feature c = 15, x = r - mu_c:
//   e_{c +- k} = e_c U_+-^k Q_k,  U_+- = exp(+-2 eta dmu x - eta dmu^2),  Q_k = exp(-eta dmu^2 k (k-1)),
// so one running product per side (three exponentials per pair) and the constants Q_k give all
// 32.  Every e_f is at most 1, and for r < 1.2 nm the running products stay far inside the FP32
// range (e_c >= 1e-18, U^k <= 1e30).
constexpr int kCentre = 15;
constexpr float kMuC = kMu0 + kCentre * kDmu;

// exp(x), x <= 0, as a constant expression: the Taylor series of exp(x / 2^20), squared 20 times
// (relative error about 1e-10 for |x| < 50).
constexpr double const_exp(double x) {
  const double y = x / 1048576.0;
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 12; ++n) {
    term *= y / n;
    sum += term;
  }
  for (int k = 0; k < 20; ++k) sum *= sum;
  return sum;
}
constexpr float gauss_q(int k) {
  return (float)const_exp(-(double)kEta * (double)kDmu * (double)kDmu * k * (k - 1));
}
// Q_{|f - c|} per feature f
__constant__ float c_gauss_q[kNF] = {
    gauss_q(15), gauss_q(14), gauss_q(13), gauss_q(12), gauss_q(11), gauss_q(10), gauss_q(9),
    gauss_q(8),  gauss_q(7),  gauss_q(6),  gauss_q(5),  gauss_q(4),  gauss_q(3),  gauss_q(2),
    gauss_q(1),  gauss_q(0),  gauss_q(1),  gauss_q(2),  gauss_q(3),  gauss_q(4),  gauss_q(5),
    gauss_q(6),  gauss_q(7),  gauss_q(8),  gauss_q(9),  gauss_q(10), gauss_q(11), gauss_q(12),
    gauss_q(13), gauss_q(14), gauss_q(15), gauss_q(16)};

// e_c and the two ratios U_+ (up) and U_- (down) of a pair at distance r.
__device__ __forceinline__ void gauss_seeds(float r, float* ec, float* up, float* down) {
  const float x = r - kMuC;
  const float a = 2.f * kEta * kDmu * x, b = kEta * kDmu * kDmu;
  *ec = __expf(-kEta * x * x);
  *up = __expf(a - b);
  *down = __expf(-a - b);
}

// G_f += scale e_f for all f.  Each side runs two products (odd and even steps, ratio U^2), which
// halves the dependent chain.
__device__ __forceinline__ void add_gaussians(float r, float scale, float* G) {
  float ec, up, down;
  gauss_seeds(r, &ec, &up, &down);
  const float v0 = ec * scale;
  G[kCentre] += v0;
  const float up2 = up * up, down2 = down * down;
  float va = v0 * up, vb = v0 * up2;
#pragma unroll
  for (int k = 1; kCentre + k < kNF; k += 2) {
    G[kCentre + k] = fmaf(va, c_gauss_q[kCentre + k], G[kCentre + k]);
    if (kCentre + k + 1 < kNF)
      G[kCentre + k + 1] = fmaf(vb, c_gauss_q[kCentre + k + 1], G[kCentre + k + 1]);
    va *= up2;
    vb *= up2;
  }
  va = v0 * down;
  vb = v0 * down2;
#pragma unroll
  for (int k = 1; kCentre - k >= 0; k += 2) {
    G[kCentre - k] = fmaf(va, c_gauss_q[kCentre - k], G[kCentre - k]);
    if (kCentre - k - 1 >= 0)
      G[kCentre - k - 1] = fmaf(vb, c_gauss_q[kCentre - k - 1], G[kCentre - k - 1]);
    va *= down2;
    vb *= down2;
  }
}

__device__ __forceinline__ float component(const float4& v, int c) {
  return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}

// s0 = sum_f W_f e_f and t = sum_f W_f e_f mu_f for the pair weights W_f = W_if + W_jf, given
// premultiplied as A_f = W_f Q_{|f - c|} (own part wq in registers, the partner's sq as 16-byte
// aligned shared rows).  With e_{c +- k} = e_c U_+-^k Q_k, U = U_+, D = U_-:
//   s0 = e_c S,  S = A_c + U P_+(U) + D P_-(D),  P_+(U) = sum_{k>=1} A_{c+k} U^(k-1)  (likewise P_-),
//   t  = e_c (mu_c S + dmu (U (P_+ + U P_+') - D (P_- + D P_-'))),
// the polynomials and their derivatives by Horner's rule: three operations per feature.
__device__ __forceinline__ void weighted_gaussians(float r, const float* wq, const float4* sq,
                                                   float* s0, float* t) {
  float ec, up, down;
  gauss_seeds(r, &ec, &up, &down);
  float pu = wq[kNF - 1] + component(sq[(kNF - 1) >> 2], (kNF - 1) & 3), du = 0.f;
#pragma unroll
  for (int f = kNF - 2; f > kCentre; --f) {
    du = fmaf(du, up, pu);
    pu = fmaf(pu, up, wq[f] + component(sq[f >> 2], f & 3));
  }
  float pd = wq[0] + component(sq[0], 0), dd = 0.f;
#pragma unroll
  for (int f = 1; f < kCentre; ++f) {
    dd = fmaf(dd, down, pd);
    pd = fmaf(pd, down, wq[f] + component(sq[f >> 2], f & 3));
  }
  const float sum = wq[kCentre] + component(sq[kCentre >> 2], kCentre & 3) + up * pu + down * pd;
  const float moment = up * fmaf(up, du, pu) - down * fmaf(down, dd, pd);
  *s0 = ec * sum;
  *t = ec * fmaf(kMuC, sum, kDmu * moment);
}

template <class Real>
__device__ __forceinline__ float4 slot_pos(const void* posq, int s) {
  const typename V4<Real>::T4 p = reinterpret_cast<const typename V4<Real>::T4*>(posq)[s];
  return make_float4((float)p.x, (float)p.y, (float)p.z, 0.f);
}
template <class Real>
__device__ __forceinline__ float2 slot_par(const void* params, int s) {
  const typename V4<Real>::T2 p = reinterpret_cast<const typename V4<Real>::T2*>(params)[s];
  return make_float2((float)p.x, (float)p.y);
}

// Particle-level entry lists of a block I, built a chunk of I's block list at a time in shared
// memory: every particle j of the chunk's blocks goes to the list of each half of I (slots 0-15,
// 16-31) whose bounding box it comes within rf of ("near": features and integral) or within rc
// of ("far": integral only).  A tile then pairs 16 entries of each half's list with that half's
// 16 particles, so a lane meets only particles near its own half of the block.  The lists are
// filled in block order by a prefix over the chunk, so every run visits the same pairs in the
// same order.
constexpr int kChunk = 16;             // blocks of I's list per chunk
constexpr int kListCap = 32 * kChunk;  // entries per list per chunk
enum : int { kNearA, kNearB, kFarA, kFarB };
constexpr float kListMargin = 1e-4f;   // nm added to both cutoffs for the box tests

// Centre and half extents of the two halves of block I (negative half extent: empty half).
struct HalfBoxes {
  float3 c[2], h[2];
};

struct EntryLists {
  HalfBoxes box;  // the two halves of I
  int slot[4][kListCap];
  unsigned bits[kChunk][4];
  int pre[4][kChunk + 1];
  int block[kChunk];
};

__device__ __forceinline__ HalfBoxes half_boxes(float3 p, bool valid) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (valid) {
    lo[0] = hi[0] = p.x;
    lo[1] = hi[1] = p.y;
    lo[2] = hi[2] = p.z;
  }
  for (int o = 8; o > 0; o >>= 1)
    for (int d = 0; d < 3; ++d) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(kFull, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(kFull, hi[d], o));
    }
  HalfBoxes b;
  for (int h = 0; h < 2; ++h) {
    float l[3], u[3];
    for (int d = 0; d < 3; ++d) {
      l[d] = __shfl_sync(kFull, lo[d], 16 * h);
      u[d] = __shfl_sync(kFull, hi[d], 16 * h);
    }
    const bool empty = l[0] > u[0];
    b.c[h] = make_float3(0.5f * (l[0] + u[0]), 0.5f * (l[1] + u[1]), 0.5f * (l[2] + u[2]));
    b.h[h] = empty ? make_float3(-1.f, -1.f, -1.f)
                   : make_float3(0.5f * (u[0] - l[0]), 0.5f * (u[1] - l[1]), 0.5f * (u[2] - l[2]));
  }
  return b;
}

__device__ __forceinline__ float box_gap2(float3 p, float3 c, float3 h) {
  const float gx = fmaxf(fabsf(p.x - c.x) - h.x, 0.f);
  const float gy = fmaxf(fabsf(p.y - c.y) - h.y, 0.f);
  const float gz = fmaxf(fabsf(p.z - c.z) - h.z, 0.f);
  return gx * gx + gy * gy + gz * gz;
}

// Fills L with the entries of blocks q0 .. q0 + kChunk - 1 of I's list (blocks below I skipped
// when `upper`) and returns the number of blocks taken.  Ends with the CTA synchronised.
template <class Real>
__device__ int build_entry_lists(const LearnedGbArgs& a, const GbArgs& g, int I, int q0, int nn,
                                 int n_near, bool upper, EntryLists& L) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nq = min(kChunk, nn - q0);
  const float rc_m = a.rc + kListMargin, rf_m = a.rf + kListMargin;
  const float rc2 = rc_m * rc_m, rf2 = rf_m * rf_m;
  for (int qq = w; qq < nq; qq += kWarps) {
    bool unused;
    const int J = list_block(a, I, q0 + qq, n_near, &unused);
    bool in[4] = {false, false, false, false};
    if (!(upper && J < I)) {
      const int aj = g.slot_atom[32 * J + lane];
      const float4 p4 = slot_pos<Real>(g.posq, 32 * J + lane);
      if (aj >= 0) {
        const float3 p = make_float3(p4.x, p4.y, p4.z);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float3 hh = L.box.h[h];
          if (hh.x < 0.f) continue;
          const float gap2 = box_gap2(p, L.box.c[h], hh);
          in[kNearA + h] = gap2 < rf2;
          in[kFarA + h] = gap2 >= rf2 && gap2 < rc2;
        }
      }
    }
    const unsigned b0 = __ballot_sync(kFull, in[0]), b1 = __ballot_sync(kFull, in[1]);
    const unsigned b2 = __ballot_sync(kFull, in[2]), b3 = __ballot_sync(kFull, in[3]);
    if (lane == 0) {
      L.bits[qq][0] = b0;
      L.bits[qq][1] = b1;
      L.bits[qq][2] = b2;
      L.bits[qq][3] = b3;
      L.block[qq] = J;
    }
  }
  __syncthreads();
  if (w == 0) {  // exclusive prefix of the four lists' counts over the chunk's blocks (nq <= 32)
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int c = lane < nq ? __popc(L.bits[lane][l]) : 0;
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < nq) L.pre[l][lane] = incl - c;
      if (lane == nq - 1) L.pre[l][nq] = incl;
    }
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  for (int qq = w; qq < nq; qq += kWarps) {
    const int slot = 32 * L.block[qq] + lane;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const unsigned b = L.bits[qq][l];
      if ((b >> lane) & 1u) L.slot[l][L.pre[l][qq] + __popc(b & below)] = slot;
    }
  }
  __syncthreads();
  return nq;
}

// One CTA per block I, lane = particle i; the CTA's warps share I's entry lists (one tile of 16
// entries per half at a time) and their partial sums meet in shared memory in a fixed order.
// Radial features (near entries, r < rf) and the switched short-range integral (r < rc) over
// every particle j != i.
template <class Real>
__global__ void __launch_bounds__(32 * kWarps) lr_features(LearnedGbArgs a, GbArgs g) {
  if (!a.state->need) return;
  __shared__ EntryLists s_lists;
  __shared__ float4 s_pos[kWarps][32];  // xyz, slot as int bits (-1: no entry)
  __shared__ float s_scaled[kWarps][32];
  __shared__ float s_red[kWarps][32][kNF + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int hbase = lane & 16;
  const float rc2 = a.rc * a.rc, rf2 = a.rf * a.rf;
  const float fc_k = kPiF / a.rf;
  for (int I = blockIdx.x; I < a.n_blocks; I += gridDim.x) {
    const int si = 32 * I + lane;
    const int ai = g.slot_atom[si];
    const float4 p4 = slot_pos<Real>(g.posq, si);
    const float3 pi = make_float3(p4.x, p4.y, p4.z);
    const float off_i = ai >= 0 ? slot_par<Real>(g.params, si).x : 1.f;
    {
      const HalfBoxes boxes = half_boxes(pi, ai >= 0);
      if (threadIdx.x == 0) s_lists.box = boxes;
    }
    __syncthreads();
    float G[kNF];
#pragma unroll
    for (int f = 0; f < kNF; ++f) G[f] = 0.f;
    float ishort = 0.f;
    const int n_near = a.nbr_count[2 * I], nn = n_near + a.nbr_count[2 * I + 1];
    for (int q0 = 0; q0 < nn; q0 += kChunk) {
      const int nq = build_entry_lists<Real>(a, g, I, q0, nn, n_near, false, s_lists);
      const int n_na = s_lists.pre[kNearA][nq], n_nb = s_lists.pre[kNearB][nq];
      const int n_fa = s_lists.pre[kFarA][nq], n_fb = s_lists.pre[kFarB][nq];
      const int t_near = (max(n_na, n_nb) + 15) >> 4, t_far = (max(n_fa, n_fb) + 15) >> 4;
      for (int t = w; t < t_near + t_far; t += kWarps) {
        const bool near = t < t_near;  // uniform over the warp
        const int list = (near ? kNearA : kFarA) + (lane >> 4);
        const int e = 16 * (near ? t : t - t_near) + (lane & 15);
        const int slot = e < s_lists.pre[list][nq] ? s_lists.slot[list][e] : -1;
        if (slot >= 0) {
          const float4 p = slot_pos<Real>(g.posq, slot);
          s_pos[w][lane] = make_float4(p.x, p.y, p.z, __int_as_float(slot));
          s_scaled[w][lane] = slot_par<Real>(g.params, slot).y;
        } else {
          s_pos[w][lane] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
          s_scaled[w][lane] = 0.f;
        }
        __syncwarp();
        if (ai >= 0) {
#pragma unroll 2
          for (int k = 0; k < 16; ++k) {
            const int jl = hbase | ((lane + k) & 15);
            const float4 pj = s_pos[w][jl];
            const int sj = __float_as_int(pj.w);
            if (sj < 0 || sj == si) continue;
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
            add_gaussians(r, fc, G);
          }
        }
        __syncwarp();
      }
      __syncthreads();  // the next chunk refills the lists
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
// pair is done once, from the lower block (entries of blocks J >= I only): the force on each
// entry travels with it one lane per warp shuffle within its half and is committed in fixed
// point after the 16 steps; pairs inside block I are visited from both sides and keep their
// i-forces only.
template <class Real>
__global__ void __launch_bounds__(32 * kWarps, 5) lr_forces(LearnedGbArgs a, GbArgs g) {
  if (!a.state->use_learned) return;
  __shared__ EntryLists s_lists;
  __shared__ float4 s_pos[kWarps][32];        // xyz, slot as int bits (-1: no entry)
  __shared__ float4 s_par[kWarps][32];        // offset radius, scaled radius, D
  // D_j d tail_j / d G_jf times Q_{|f - c|}; rows of kNF + 4 floats stay 16-byte aligned for
  // vector access, and the rows of 8 consecutive entries fall in distinct banks
  __shared__ __align__(16) float s_w[kWarps][32][kNF + 4];
  __shared__ float s_red[kWarps][32][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int hbase = lane & 16;
  const float rc2 = a.rc * a.rc, rf2 = a.rf * a.rf;
  const Real* chain = reinterpret_cast<const Real*>(g.dedr_slot);
  const float fc_k = kPiF / a.rf;
  const float fscale = (float)kForceScale;
  for (int I = blockIdx.x; I < a.n_blocks; I += gridDim.x) {
    const int si = 32 * I + lane;
    const int ai = g.slot_atom[si];
    const float4 p4 = slot_pos<Real>(g.posq, si);
    const float3 pi = make_float3(p4.x, p4.y, p4.z);
    float off_i = 1.f, sc_i = 0.f, d_i = 0.f;
    float wi[kNF];  // D_i d tail_i / d G_if, times Q_{|f - c|}
#pragma unroll
    for (int f = 0; f < kNF; ++f) wi[f] = 0.f;
    if (ai >= 0) {
      const float2 par = slot_par<Real>(g.params, si);
      off_i = par.x;
      sc_i = par.y;
      d_i = 0.5f * (float)chain[si];
      const float4* dt = reinterpret_cast<const float4*>(a.dtail + (size_t)ai * kNF);
#pragma unroll
      for (int qq = 0; qq < kNF / 4; ++qq) {
        const float4 v = dt[qq];
        wi[4 * qq] = d_i * v.x * c_gauss_q[4 * qq];
        wi[4 * qq + 1] = d_i * v.y * c_gauss_q[4 * qq + 1];
        wi[4 * qq + 2] = d_i * v.z * c_gauss_q[4 * qq + 2];
        wi[4 * qq + 3] = d_i * v.w * c_gauss_q[4 * qq + 3];
      }
    }
    {
      const HalfBoxes boxes = half_boxes(pi, ai >= 0);
      if (threadIdx.x == 0) s_lists.box = boxes;
    }
    __syncthreads();
    float fx = 0.f, fy = 0.f, fz = 0.f;
    const int n_near = a.nbr_count[2 * I], nn = n_near + a.nbr_count[2 * I + 1];
    for (int q0 = 0; q0 < nn; q0 += kChunk) {
      const int nq = build_entry_lists<Real>(a, g, I, q0, nn, n_near, true, s_lists);
      const int n_na = s_lists.pre[kNearA][nq], n_nb = s_lists.pre[kNearB][nq];
      const int n_fa = s_lists.pre[kFarA][nq], n_fb = s_lists.pre[kFarB][nq];
      const int t_near = (max(n_na, n_nb) + 15) >> 4, t_far = (max(n_fa, n_fb) + 15) >> 4;
      for (int t = w; t < t_near + t_far; t += kWarps) {
        const bool near = t < t_near;  // uniform over the warp
        const int list = (near ? kNearA : kFarA) + (lane >> 4);
        const int e = 16 * (near ? t : t - t_near) + (lane & 15);
        const int slot = e < s_lists.pre[list][nq] ? s_lists.slot[list][e] : -1;
        int aj = -1;
        if (slot >= 0) {
          aj = g.slot_atom[slot];
          const float4 p = slot_pos<Real>(g.posq, slot);
          const float2 par = slot_par<Real>(g.params, slot);
          const float dj = 0.5f * (float)chain[slot];
          s_pos[w][lane] = make_float4(p.x, p.y, p.z, __int_as_float(slot));
          s_par[w][lane] = make_float4(par.x, par.y, dj, 0.f);
          if (near) {
            const float4* dt = reinterpret_cast<const float4*>(a.dtail + (size_t)aj * kNF);
            float4* row = reinterpret_cast<float4*>(s_w[w][lane]);
#pragma unroll
            for (int qq = 0; qq < kNF / 4; ++qq) {
              const float4 v = dt[qq];
              row[qq] = make_float4(dj * v.x * c_gauss_q[4 * qq], dj * v.y * c_gauss_q[4 * qq + 1],
                                    dj * v.z * c_gauss_q[4 * qq + 2], dj * v.w * c_gauss_q[4 * qq + 3]);
            }
          }
        } else {
          s_pos[w][lane] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
          s_par[w][lane] = make_float4(1.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
        float gx = 0.f, gy = 0.f, gz = 0.f;  // force on the entry now in this lane's rotation
        const int src = hbase | ((lane + 1) & 15);
        for (int k = 0; k < 16; ++k) {
          const int jl = hbase | ((lane + k) & 15);
          const float4 pj = s_pos[w][jl];
          const int sj = __float_as_int(pj.w);
          const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
          const float r2 = dx * dx + dy * dy + dz * dz;
          float radial = 0.f;
          if (ai >= 0 && sj >= 0 && sj != si && r2 < rc2) {
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
              // sum_f W_f g_f'(r),  g_f' = e_f (-2 eta (r - mu_f) fc + dfc),
              // with sum_f W_f e_f (r - mu_f) = r s0 - t
              float s0, t;
              weighted_gaussians(r, wi, reinterpret_cast<const float4*>(s_w[w][jl]), &s0, &t);
              phi += dfc * s0 - 2.f * kEta * fc * (r * s0 - t);
            }
            radial = phi * inv_r;
          }
          fx = fmaf(radial, dx, fx);
          fy = fmaf(radial, dy, fy);
          fz = fmaf(radial, dz, fz);
          gx = fmaf(-radial, dx, gx);
          gy = fmaf(-radial, dy, gy);
          gz = fmaf(-radial, dz, gz);
          gx = __shfl_sync(kFull, gx, src);
          gy = __shfl_sync(kFull, gy, src);
          gz = __shfl_sync(kFull, gz, src);
        }
        if (aj >= 0 && (slot >> 5) != I) {
          add_fixed(g.force + aj, to_fixed(gx, fscale));
          add_fixed(g.force + g.n_atoms + aj, to_fixed(gy, fscale));
          add_fixed(g.force + 2 * g.n_atoms + aj, to_fixed(gz, fscale));
        }
        __syncwarp();
      }
      __syncthreads();  // the next chunk refills the lists
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
      lr_features<Real><<<ctas, 32 * kWarps, 0, s>>>(a, g);
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
