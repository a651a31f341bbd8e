// The learned Born-radii network (no reference counterpart): per particle, 32 radial
// symmetry-function features -> 64 -> 64 -> 1 with tanh, predicting the long-range tail of
// the HCT integral that the O(N^2) OBC descreening pass (gbsa_obc.rs:209-212) would add to
// the short-range part.  Both kernels run on the 5th-generation tensor cores: BF16 operands
// staged in shared memory in the canonical K-major layout, tcgen05.mma with FP32 accumulators
// in tensor memory, tcgen05.ld for the epilogues.  One thread owns one particle (one row of
// the 128-row MMA tile), so activations, output layer and the elementwise parts of the
// backward pass stay in registers.
//
// Inference (every MD step, all particles):
//   D1 = X W1          h1 = tanh(D1 + b1)
//   D2 = h1 W2         h2 = tanh(D2 + b2)      y = h2 . w3 + b3,  tail = y t_scale + t_mean
//   D3 = d2 W2^T       d2 = w3 (1 - h2^2)
//   D4 = d1 W1^T       d1 = D3 (1 - h1^2)      d tail / d G = D4 inv_std t_scale
// Training (one CTA, Adam (Kingma & Ba 2015) on mean-squared error of the normalised tail over
// batches of particles): the weight gradients h1^T d2 and d1^T X of each 128-particle chunk
// are one M = 128, N = 96, K = 128 MMA chain accumulated in tensor memory across the batch;
// bias gradients are fixed-order block reductions, so a training step is deterministic.
#include <atomic>

#include "kernels.h"
#include "tcgen05.cuh"

namespace ommb200 {
namespace {

using bf16 = __nv_bfloat16;
using namespace tc;

constexpr int kNF = 32, kH = 64;
// Polls of an mbarrier wait before a kernel gives up (about a millisecond).  The waits for a
// round of MMAs take their limit from the launch (ommb200_set_tensor_core_wait_limit lowers it
// to exercise the time-out path); the drain after a time-out always takes the full limit, so
// no MMA still writes tensor memory when it is freed.
constexpr uint32_t kWaitLimit = 1u << 22;
std::atomic<uint32_t> g_wait_limit{kWaitLimit};

// parameter block (floats)
constexpr int kOffW1 = 0, kOffB1 = 2048, kOffW2 = 2112, kOffB2 = 6208, kOffW3 = 6272,
              kOffB3 = 6336, kOffMean = kRadiiMlpOffMean, kOffInvStd = kRadiiMlpOffInvStd,
              kOffTMean = kRadiiMlpOffTMean, kOffTScale = kRadiiMlpOffTScale;
static_assert(kOffTScale + 1 == kRadiiMlpParams, "parameter block layout");

// per-CTA constants next to the operands: b1, b2, w3, mean, inv_std, b3, t_mean, t_scale
struct Consts {
  float b1[kH], b2[kH], w3[kH], mean[kNF], inv_std[kNF], b3, t_mean, t_scale, pad;
};

// Writes the BF16 weight operands (B matrices, K-major) and the FP32 constants.
//   w1f: N = 64 (j) x K = 32 (f), element (j, f) = W1[f][j]      (X W1)
//   w2f: N = 64 (k) x K = 64 (j), element (k, j) = W2[j][k]      (h1 W2)
//   w2b: N = 64 (j) x K = 64 (k), element (j, k) = W2[j][k]      (d2 W2^T)
//   w1b: N = 32 (f) x K = 64 (j), element (f, j) = W1[f][j]      (d1 W1^T), optional
__device__ void stage_weights(const float* __restrict__ P, uint8_t* w1f, uint8_t* w2f,
                              uint8_t* w2b, uint8_t* w1b, Consts* c) {
  for (int idx = threadIdx.x; idx < kNF * kH; idx += blockDim.x) {
    const int f = idx / kH, j = idx % kH;
    const bf16 v = __float2bfloat16_rn(P[kOffW1 + idx]);
    *reinterpret_cast<bf16*>(w1f + kmajor_offset(j, f, kNF)) = v;
    if (w1b) *reinterpret_cast<bf16*>(w1b + kmajor_offset(f, j, kH)) = v;
  }
  for (int idx = threadIdx.x; idx < kH * kH; idx += blockDim.x) {
    const int j = idx / kH, k = idx % kH;
    const bf16 v = __float2bfloat16_rn(P[kOffW2 + idx]);
    *reinterpret_cast<bf16*>(w2f + kmajor_offset(k, j, kH)) = v;
    *reinterpret_cast<bf16*>(w2b + kmajor_offset(j, k, kH)) = v;
  }
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    c->b1[i] = P[kOffB1 + i];
    c->b2[i] = P[kOffB2 + i];
    c->w3[i] = P[kOffW3 + i];
  }
  for (int i = threadIdx.x; i < kNF; i += blockDim.x) {
    c->mean[i] = P[kOffMean + i];
    c->inv_std[i] = P[kOffInvStd + i];
  }
  if (threadIdx.x == 0) {
    c->b3 = P[kOffB3];
    c->t_mean = P[kOffTMean];
    c->t_scale = P[kOffTScale];
  }
}

// Normalised features of one particle as BF16 row `row` of a K = 32 operand; returns them.
__device__ __forceinline__ void stage_features(const float* __restrict__ G, int atom, bool valid,
                                               const Consts* c, uint8_t* xa, int row,
                                               float* x) {
  if (valid) {
    const float4* g4 = reinterpret_cast<const float4*>(G + (size_t)atom * kNF);
#pragma unroll
    for (int q = 0; q < kNF / 4; ++q) {
      const float4 v = g4[q];
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int f = 0; f < kNF; ++f) x[f] = (x[f] - c->mean[f]) * c->inv_std[f];
  } else {
#pragma unroll
    for (int f = 0; f < kNF; ++f) x[f] = 0.f;
  }
#pragma unroll
  for (int q = 0; q < kNF / 8; ++q)
    *reinterpret_cast<uint4*>(xa + kmajor_offset(row, 8 * q, kNF)) = pack8_bf16(x + 8 * q);
}

__device__ __forceinline__ void store_row64(uint8_t* base, int row, int col0, const float* v) {
  *reinterpret_cast<uint4*>(base + kmajor_offset(row, col0, kH)) = pack8_bf16(v);
  *reinterpret_cast<uint4*>(base + kmajor_offset(row, col0 + 8, kH)) = pack8_bf16(v + 8);
}

// ---- inference ---------------------------------------------------------------------------
struct InferSmem {
  static constexpr uint32_t w1f = 0, w2f = 4096, w2b = 12288, w1b = 20480, xa = 24576,
                            ha = 32768, consts = 49152;
  static constexpr uint32_t mbar = consts + ((sizeof(Consts) + 15) / 16) * 16;
  static constexpr uint32_t slot = mbar + 8;
  static constexpr uint32_t bytes = slot + 8;
};
// 100 KiB per CTA caps residency at two CTAs per SM, whose 2 x 256 tensor-memory columns fit
// the SM's 512, so tcgen05.alloc never waits on another CTA.
constexpr uint32_t kInferSmemLaunch = 100 * 1024;
constexpr uint32_t kInferTmemCols = 256;
static_assert(InferSmem::bytes <= kInferSmemLaunch, "inference shared memory");

__global__ void __launch_bounds__(128) mlp_infer_kernel(int n, const float* __restrict__ G,
                                                        const float* __restrict__ P,
                                                        float* __restrict__ tail,
                                                        float* __restrict__ dtail,
                                                        int* status, const int* gate,
                                                        uint32_t wait_limit) {
  if (gate && *gate == 0) return;
  extern __shared__ __align__(1024) uint8_t sm[];
  using L = InferSmem;
  __shared__ int s_ok;
  Consts* c = reinterpret_cast<Consts*>(sm + L::consts);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + L::mbar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + L::slot);
  const int tid = threadIdx.x, warp = tid >> 5;
  stage_weights(P, sm + L::w1f, sm + L::w2f, sm + L::w2b, sm + L::w1b, c);
  if (tid == 0) {
    mbar_init(mbar, 1);
    s_ok = 1;
  }
  if (warp == 0) tmem_alloc(slot, kInferTmemCols);
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *slot;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  const uint32_t a_x = smem_addr(sm + L::xa), a_h = smem_addr(sm + L::ha);
  const uint32_t b_w1f = smem_addr(sm + L::w1f), b_w2f = smem_addr(sm + L::w2f);
  const uint32_t b_w2b = smem_addr(sm + L::w2b), b_w1b = smem_addr(sm + L::w1b);
  uint32_t phase = 0;
  bool ok = true;
  // one MMA round: thread 0 issues the K steps, commits, waits; everyone learns the outcome
  auto round = [&](uint32_t d, uint32_t a, uint32_t b, int ksteps, uint32_t sbo_a,
                   uint32_t sbo_b, uint32_t idesc) {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      for (int k = 0; k < ksteps; ++k)
        mma_bf16(tmem + d, smem_desc(a + 256 * k, 128, sbo_a), smem_desc(b + 256 * k, 128, sbo_b),
                 idesc, k > 0);
      mma_commit(mbar);
      s_ok = mbar_wait(mbar, phase, wait_limit) ? 1 : 0;
    }
    __syncthreads();
    fence_after_sync();
    phase ^= 1;
    return s_ok != 0;
  };
  const int tiles = (n + 127) / 128;
  for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const int atom = t * 128 + tid;
    const bool valid = atom < n;
    float v[16], h[16];
    {
      float x[kNF];
      stage_features(G, atom, valid, c, sm + L::xa, tid, x);
    }
    if (!(ok = round(0, a_x, b_w1f, kNF / 16, kNF * 16, kNF * 16, idesc_bf16(128, 64)))) break;
    for (int q = 0; q < 4; ++q) {  // h1
      tmem_ld16(tmem + lane + 16 * q, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) h[i] = tanhf(v[i] + c->b1[16 * q + i]);
      store_row64(sm + L::ha, tid, 16 * q, h);
    }
    if (!(ok = round(64, a_h, b_w2f, kH / 16, kH * 16, kH * 16, idesc_bf16(128, 64)))) break;
    float y = 0.f;
    for (int q = 0; q < 4; ++q) {  // h2, output, d2
      tmem_ld16(tmem + lane + 64 + 16 * q, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float w = c->w3[16 * q + i];
        const float h2 = tanhf(v[i] + c->b2[16 * q + i]);
        y = fmaf(h2, w, y);
        h[i] = w * (1.f - h2 * h2);
      }
      store_row64(sm + L::ha, tid, 16 * q, h);
    }
    if (valid) tail[atom] = (y + c->b3) * c->t_scale + c->t_mean;
    if (dtail == nullptr) {
      fence_before_sync();
      __syncthreads();
      continue;
    }
    if (!(ok = round(128, a_h, b_w2b, kH / 16, kH * 16, kH * 16, idesc_bf16(128, 64)))) break;
    for (int q = 0; q < 4; ++q) {  // d1
      float z[16];
      tmem_ld16(tmem + lane + 128 + 16 * q, v);
      tmem_ld16(tmem + lane + 16 * q, z);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float h1 = tanhf(z[i] + c->b1[16 * q + i]);
        h[i] = v[i] * (1.f - h1 * h1);
      }
      store_row64(sm + L::ha, tid, 16 * q, h);
    }
    if (!(ok = round(192, a_h, b_w1b, kH / 16, kH * 16, kH * 16, idesc_bf16(128, 32)))) break;
    for (int q = 0; q < 2; ++q) {  // d tail / d G
      tmem_ld16(tmem + lane + 192 + 16 * q, v);
      if (valid) {
        float4* out = reinterpret_cast<float4*>(dtail + (size_t)atom * kNF + 16 * q);
#pragma unroll
        for (int i = 0; i < 4; ++i)
          out[i] = make_float4(v[4 * i] * c->inv_std[16 * q + 4 * i] * c->t_scale,
                               v[4 * i + 1] * c->inv_std[16 * q + 4 * i + 1] * c->t_scale,
                               v[4 * i + 2] * c->inv_std[16 * q + 4 * i + 2] * c->t_scale,
                               v[4 * i + 3] * c->inv_std[16 * q + 4 * i + 3] * c->t_scale);
      }
    }
    fence_before_sync();
    __syncthreads();
  }
  fence_before_sync();
  __syncthreads();
  if (!ok && tid == 0) {
    report_status(status, kStatusTimeout);
    mbar_wait(mbar, phase ^ 1, kWaitLimit);  // let the MMAs in flight drain
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, kInferTmemCols);
  }
}

// ---- training --------------------------------------------------------------------------
struct TrainSmem {
  static constexpr uint32_t w1f = 0, w2f = 4096, w2b = 12288, xa = 20480, ha = 28672,
                            ga = 45056,   // A of the gradient MMA: 128 rows x 128 particles
                            gb = 77824,   // B of the gradient MMA:  96 rows x 128 particles
                            consts = 102400;
  static constexpr uint32_t partial = consts + ((sizeof(Consts) + 15) / 16) * 16;  // [4][196]
  static constexpr uint32_t acc = partial + 4 * 196 * 4;                           // [196]
  static constexpr uint32_t mbar = acc + 196 * 4;
  static constexpr uint32_t slot = mbar + 8;
  static constexpr uint32_t bytes = slot + 8;
};
constexpr uint32_t kTrainTmemCols = 512;
// reduction slots: dW3 [0, 64), db2 [64, 128), db1 [128, 192), db3 192, loss 193
constexpr int kRedW3 = 0, kRedB2 = 64, kRedB1 = 128, kRedB3 = 192, kRedLoss = 193, kRed = 194;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// splitmix64 (Steele, Lea & Flood 2014): the batch draw of particle slot i at Adam step t.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void adam(float* p, float* m, float* v, float g, float lr, float bc1,
                                     float bc2) {
  const float mm = 0.9f * *m + 0.1f * g;
  const float vv = 0.999f * *v + 0.001f * g * g;
  *m = mm;
  *v = vv;
  *p -= lr * (mm / bc1) / (sqrtf(vv / bc2) + 1e-8f);
}

__global__ void __launch_bounds__(128) mlp_train_kernel(int n, const float* __restrict__ G,
                                                        const float* __restrict__ target,
                                                        float* P, float* adam_m, float* adam_v,
                                                        int* adam_t, int steps, int batch,
                                                        float lr, unsigned long long seed,
                                                        float* grad_out, float* loss_out,
                                                        int* status, const int* gate,
                                                        uint32_t wait_limit) {
  if (gate && *gate == 0) return;
  extern __shared__ __align__(1024) uint8_t sm[];
  using L = TrainSmem;
  __shared__ int s_ok;
  Consts* c = reinterpret_cast<Consts*>(sm + L::consts);
  float* partial = reinterpret_cast<float*>(sm + L::partial);
  float* acc = reinterpret_cast<float*>(sm + L::acc);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + L::mbar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + L::slot);
  const int tid = threadIdx.x, warp = tid >> 5, lane_id = tid & 31;
  if (tid == 0) {
    mbar_init(mbar, 1);
    s_ok = 1;
  }
  if (warp == 0) tmem_alloc(slot, kTrainTmemCols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *slot;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  const uint32_t a_x = smem_addr(sm + L::xa), a_h = smem_addr(sm + L::ha);
  const uint32_t a_g = smem_addr(sm + L::ga), b_g = smem_addr(sm + L::gb);
  const uint32_t b_w1f = smem_addr(sm + L::w1f), b_w2f = smem_addr(sm + L::w2f);
  const uint32_t b_w2b = smem_addr(sm + L::w2b);
  uint32_t phase = 0;
  bool ok = true;
  auto round = [&](uint32_t d, uint32_t a, uint32_t b, int ksteps, uint32_t sbo_a,
                   uint32_t sbo_b, uint32_t idesc, bool accumulate) {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      for (int k = 0; k < ksteps; ++k)
        mma_bf16(tmem + d, smem_desc(a + 256 * k, 128, sbo_a), smem_desc(b + 256 * k, 128, sbo_b),
                 idesc, accumulate || k > 0);
      mma_commit(mbar);
      s_ok = mbar_wait(mbar, phase, wait_limit) ? 1 : 0;
    }
    __syncthreads();
    fence_after_sync();
    phase ^= 1;
    return s_ok != 0;
  };
  // block-wide fixed-order sum of one value per thread into acc[slot]
  auto reduce = [&](int idx, float v) {
    v = warp_sum(v);
    if (lane_id == 0) partial[warp * 196 + idx] = v;
  };
  const int t0 = *adam_t;
  const int chunks = batch / 128;
  for (int s = 0; s < steps && ok; ++s) {
    stage_weights(P, sm + L::w1f, sm + L::w2f, sm + L::w2b, nullptr, c);
    for (int i = tid; i < kRed; i += 128) acc[i] = 0.f;
    const int tstep = t0 + s + 1;
    for (int ch = 0; ch < chunks && ok; ++ch) {
      __syncthreads();  // constants staged, previous chunk's reductions consumed
      const int ib = ch * 128 + tid;
      const int idx = batch == n ? ib
                                 : (int)(mix64(seed ^ ((unsigned long long)tstep << 32) ^
                                               (unsigned long long)ib) %
                                         (unsigned long long)n);
      float x[kNF], v[16], h[16];
      stage_features(G, idx, true, c, sm + L::xa, tid, x);
#pragma unroll
      for (int f = 0; f < kNF; ++f)  // X^T as rows 64..95 of the gradient B operand
        *reinterpret_cast<bf16*>(sm + L::gb + kmajor_offset(64 + f, tid, 128)) =
            __float2bfloat16_rn(x[f]);
      const float tn = (target[idx] - c->t_mean) / c->t_scale;
      if (!(ok = round(0, a_x, b_w1f, kNF / 16, kNF * 16, kNF * 16, idesc_bf16(128, 64), false)))
        break;
      for (int q = 0; q < 4; ++q) {  // h1 -> A of layer 2 and rows 0..63 of the gradient A
        tmem_ld16(tmem + lane + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) h[i] = tanhf(v[i] + c->b1[16 * q + i]);
        store_row64(sm + L::ha, tid, 16 * q, h);
#pragma unroll
        for (int i = 0; i < 16; ++i)
          *reinterpret_cast<bf16*>(sm + L::ga + kmajor_offset(16 * q + i, tid, 128)) =
              __float2bfloat16_rn(h[i]);
      }
      if (!(ok = round(64, a_h, b_w2f, kH / 16, kH * 16, kH * 16, idesc_bf16(128, 64), false)))
        break;
      float h2[kH];
      float y = 0.f;
      for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem + lane + 64 + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          h2[16 * q + i] = tanhf(v[i] + c->b2[16 * q + i]);
          y = fmaf(h2[16 * q + i], c->w3[16 * q + i], y);
        }
      }
      y += c->b3;
      const float g = 2.f * (y - tn) / (float)batch;
      for (int q = 0; q < 4; ++q) {  // d2 = g w3 (1 - h2^2) -> A of layer-2 backward, B rows
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int k = 16 * q + i;
          h[i] = g * c->w3[k] * (1.f - h2[k] * h2[k]);
        }
        store_row64(sm + L::ha, tid, 16 * q, h);
#pragma unroll
        for (int i = 0; i < 16; ++i)
          *reinterpret_cast<bf16*>(sm + L::gb + kmajor_offset(16 * q + i, tid, 128)) =
              __float2bfloat16_rn(h[i]);
        for (int i = 0; i < 16; ++i) {
          reduce(kRedW3 + 16 * q + i, g * h2[16 * q + i]);
          reduce(kRedB2 + 16 * q + i, h[i]);
        }
      }
      reduce(kRedB3, g);
      reduce(kRedLoss, (y - tn) * (y - tn));
      if (!(ok = round(128, a_h, b_w2b, kH / 16, kH * 16, kH * 16, idesc_bf16(128, 64), false)))
        break;
      for (int q = 0; q < 4; ++q) {  // d1 = (d2 W2^T)(1 - h1^2) -> rows 64..127 of A
        float z[16];
        tmem_ld16(tmem + lane + 128 + 16 * q, v);
        tmem_ld16(tmem + lane + 16 * q, z);
        for (int i = 0; i < 16; ++i) {
          const float h1 = tanhf(z[i] + c->b1[16 * q + i]);
          const float d1 = v[i] * (1.f - h1 * h1);
          *reinterpret_cast<bf16*>(sm + L::ga + kmajor_offset(64 + 16 * q + i, tid, 128)) =
              __float2bfloat16_rn(d1);
          reduce(kRedB1 + 16 * q + i, d1);
        }
      }
      __syncthreads();
      for (int i = tid; i < kRed; i += 128)
        acc[i] += ((partial[i] + partial[196 + i]) + partial[392 + i]) + partial[588 + i];
      // [h1^T; d1^T] x [d2^T; X^T]^T accumulated over the batch: dW2 and dW1^T blocks
      if (!(ok = round(256, a_g, b_g, 128 / 16, 128 * 16, 128 * 16, idesc_bf16(128, 96), ch > 0)))
        break;
    }
    if (!ok) break;
    // Adam on the gradient of this batch; thread r < 64 owns row r of W2 and b1/b2/w3[r],
    // thread 64 + j owns column j of W1; thread 0 owns b3
    const float bc1 = 1.f - powf(0.9f, (float)tstep), bc2 = 1.f - powf(0.999f, (float)tstep);
    const bool last = s == steps - 1;
    float gr[16];
    if (tid < 64) {
      for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem + lane + 256 + 16 * q, gr);
        for (int i = 0; i < 16; ++i) {
          const int p = kOffW2 + tid * kH + 16 * q + i;
          if (grad_out && last) grad_out[p] = gr[i];
          adam(P + p, adam_m + p, adam_v + p, gr[i], lr, bc1, bc2);
        }
      }
      const int pb[3] = {kOffB1 + tid, kOffB2 + tid, kOffW3 + tid};
      const float gb[3] = {acc[kRedB1 + tid], acc[kRedB2 + tid], acc[kRedW3 + tid]};
      for (int k = 0; k < 3; ++k) {
        if (grad_out && last) grad_out[pb[k]] = gb[k];
        adam(P + pb[k], adam_m + pb[k], adam_v + pb[k], gb[k], lr, bc1, bc2);
      }
      if (tid == 0) {
        if (grad_out && last) grad_out[kOffB3] = acc[kRedB3];
        adam(P + kOffB3, adam_m + kOffB3, adam_v + kOffB3, acc[kRedB3], lr, bc1, bc2);
        if (loss_out) loss_out[s] = acc[kRedLoss] / (float)batch;
      }
    } else {
      const int j = tid - 64;
      for (int q = 0; q < 2; ++q) {
        tmem_ld16(tmem + lane + 256 + 64 + 16 * q, gr);
        for (int i = 0; i < 16; ++i) {
          const int p = kOffW1 + (16 * q + i) * kH + j;
          if (grad_out && last) grad_out[p] = gr[i];
          adam(P + p, adam_m + p, adam_v + p, gr[i], lr, bc1, bc2);
        }
      }
    }
    fence_before_sync();
    __syncthreads();  // parameter writes visible to the next step's staging
  }
  fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    if (ok) {
      *adam_t = t0 + steps;
    } else {
      report_status(status, kStatusTimeout);
      mbar_wait(mbar, phase ^ 1, kWaitLimit);
    }
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, kTrainTmemCols);
  }
}

}  // namespace

void launch_mlp_infer(int n, const float* features, const float* params, float* tail,
                      float* dtail, int* status, int sm_count, cudaStream_t s, const int* gate) {
  if (n <= 0) return;
  cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kInferSmemLaunch);
  const int tiles = (n + 127) / 128;
  const int grid = std::max(1, std::min(tiles, 2 * sm_count));
  mlp_infer_kernel<<<grid, 128, kInferSmemLaunch, s>>>(n, features, params, tail, dtail, status,
                                                       gate, g_wait_limit.load());
}

void launch_mlp_train(int n, const float* features, const float* targets, float* params,
                      float* adam_m, float* adam_v, int* adam_t, int steps, int batch, float lr,
                      unsigned long long seed, float* grad_out, float* loss_out, int* status,
                      cudaStream_t s, const int* gate) {
  if (n <= 0 || steps <= 0) return;
  cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       TrainSmem::bytes);
  mlp_train_kernel<<<1, 128, TrainSmem::bytes, s>>>(n, features, targets, params, adam_m, adam_v,
                                                    adam_t, steps, batch, lr, seed, grad_out,
                                                    loss_out, status, gate, g_wait_limit.load());
}

void set_tensor_wait_limit(long long polls) {
  g_wait_limit.store(polls < 0 ? kWaitLimit : (uint32_t)std::min<long long>(polls, kWaitLimit));
}

}  // namespace ommb200
