// Allocation-free variant of the nonbonded pair kernel, for callers that cannot call
// cudaMalloc: code running inside another framework's memory pool, whose accounting a private
// allocation would bypass, or a plugin that may only use the buffers it is handed.  The
// caller passes device inputs and outputs; the
// kernel's scratch (packed block coordinates and 64-bit fixed-point accumulators) lives in the
// file-scope array below, which every GPU that loads the library holds until the process
// exits.  It serves non-periodic systems of at most kNoAllocMaxAtoms particles without
// exceptions (NoCutoff: bare Coulomb; CutoffNonPeriodic: reaction field, LJ cut plainly at the
// cutoff with no switching function), with the same arithmetic as the Context's
// mixed-precision path.
//
// Every call shares the one array and clears what must start at zero, so calls that overlap
// on the GPU (different streams, or different host threads on the same device) race.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>

#include "../../include/ommb200.h"
#include "kernels.h"
#include "model.h"
#include "pair_math.cuh"

namespace ommb200 {

constexpr int kNoAllocMaxAtoms = 8192;

namespace {

constexpr size_t kPosqBytes = sizeof(float4) * kNoAllocMaxAtoms;
constexpr size_t kLjBytes = sizeof(float2) * kNoAllocMaxAtoms;
constexpr size_t kForceBytes = sizeof(long long) * 3 * kNoAllocMaxAtoms;
constexpr size_t kEnergyBytes = sizeof(long long) * 8;
constexpr size_t kScratchBytes = kPosqBytes + kLjBytes + kForceBytes + kEnergyBytes;  // 384 KiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct ScratchView {
  float4* posq;
  float2* ljp;
  long long* force;   // [3][n]
  long long* energy;  // [1]
};

ScratchView view(void* base) {
  unsigned char* p = static_cast<unsigned char*>(base);
  ScratchView v;
  v.posq = reinterpret_cast<float4*>(p);
  v.ljp = reinterpret_cast<float2*>(p + kPosqBytes);
  v.force = reinterpret_cast<long long*>(p + kPosqBytes + kLjBytes);
  v.energy = reinterpret_cast<long long*>(p + kPosqBytes + kLjBytes + kForceBytes);
  return v;
}

// Device address of the array and the SM count, looked up once per CUDA context (the module,
// and with it the array, is loaded per context) with that context current.  The context comes
// from the driver's cuCtxGetCurrent, reached through the runtime's entry-point query so that
// the library needs no link against the driver library.
struct ScratchInfo {
  void* addr;
  int sm_count;
};

ScratchInfo scratch_info() {
  using GetCurrent = CUresult (*)(CUcontext*);
  static std::mutex mu;
  static GetCurrent get_current = nullptr;
  static std::map<CUcontext, ScratchInfo> known;
  std::lock_guard<std::mutex> lock(mu);
  auto fail = [](const char* what, cudaError_t e) {
    throw Error(OMMB200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  if (!get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      fail("cudaGetDriverEntryPoint(cuCtxGetCurrent)", e);
    get_current = reinterpret_cast<GetCurrent>(fn);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) == CUDA_SUCCESS && ctx) {
    auto it = known.find(ctx);
    if (it != known.end()) return it->second;
  }
  // first use in this context: the symbol lookup also initialises the runtime's context on
  // this thread when none was current
  ScratchInfo info{nullptr, 0};
  cudaError_t e = cudaGetSymbolAddress(&info.addr, g_noalloc_scratch);
  if (e != cudaSuccess || !info.addr) fail("cudaGetSymbolAddress", e);
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx)
    throw Error(OMMB200_ERR_CUDA, "no current CUDA context");
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) fail("cudaGetDevice", e);
  e = cudaDeviceGetAttribute(&info.sm_count, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) fail("cudaDeviceGetAttribute", e);
  known.emplace(ctx, info);
  return info;
}

__global__ void na_prepare(int n, int slots, const double* pos, const double* q, const double* sigma,
                           const double* eps, ScratchView s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *s.energy = 0;
  if (i >= slots) return;
  if (i < n) {
    const double sk = sqrt(kOne4PiEps0);
    s.posq[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2],
                            (float)(q[i] * sk));
    s.ljp[i] = make_float2((float)(0.5 * sigma[i]), (float)(2.0 * sqrt(eps[i])));
    s.force[i] = 0;
    s.force[n + i] = 0;
    s.force[2 * n + i] = 0;
  } else {
    s.posq[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.ljp[i] = make_float2(0.f, 0.f);
  }
}

// One warp per block pair (I <= J), as the Context's tile kernel evaluates a static tile.
template <int kElec>
__global__ void __launch_bounds__(128) na_pairs(PairArgs<float> a, int n, int n_blocks, ScratchView s) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ float4 s_pos[4][32];
  __shared__ float2 s_lj[4][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long total = (long long)n_blocks * (n_blocks + 1) / 2;
  long long e_fixed = 0;
  for (long long p = (long long)blockIdx.x * 4 + w; p < total; p += (long long)gridDim.x * 4) {
    long long I = (long long)((2.0 * n_blocks + 1.0 -
                               sqrt((2.0 * n_blocks + 1.0) * (2.0 * n_blocks + 1.0) - 8.0 * p)) * 0.5);
    if (I < 0) I = 0;
    if (I >= n_blocks) I = n_blocks - 1;
    while (I > 0 && I * n_blocks - I * (I - 1) / 2 > p) --I;
    while (I + 1 < n_blocks && (I + 1) * n_blocks - (I + 1) * I / 2 <= p) ++I;
    const long long J = I + (p - (I * n_blocks - I * (I - 1) / 2));
    const bool self = I == J;
    const int i = 32 * (int)I + lane, j = 32 * (int)J + lane;
    const float4 pi = s.posq[i];
    const float2 li = s.ljp[i];
    s_pos[w][lane] = s.posq[j];
    s_lj[w][lane] = s.ljp[j];
    __syncwarp();
    float fix = 0.f, fiy = 0.f, fiz = 0.f, fjx = 0.f, fjy = 0.f, fjz = 0.f;
    double e_tile = 0.0;
    for (int k = self ? 1 : 0; k < 32; ++k) {
      const int jl = (lane + k) & 31;
      const int jj = 32 * (int)J + jl;
      const float4 pj = s_pos[w][jl];
      const float2 lj = s_lj[w][jl];
      const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
      const float r2 = dx * dx + dy * dy + dz * dz;
      bool use = i < n && jj < n;
      if (a.use_cutoff && use) {
        bool inside = r2 < a.cutoff2;
        if (fabsf(r2 - a.cutoff2) < a.band)
          inside = exact_inside(a.pos, i, jj, 0, a.box_exact, a.cutoff2_exact);
        use = inside;
      }
      float fo, en;
      pair_terms<float, kElec, true, false>(a, use ? r2 : 1.f, pi.w * pj.w, li.x + lj.x, li.y * lj.y,
                                            fo, en);
      fo = use ? fo : 0.f;
      fix = fmaf(fo, dx, fix);
      fiy = fmaf(fo, dy, fiy);
      fiz = fmaf(fo, dz, fiz);
      if (use) e_tile += (self ? 0.5 : 1.0) * (double)en;
      if (!self) {
        fjx = fmaf(-fo, dx, fjx);
        fjy = fmaf(-fo, dy, fjy);
        fjz = fmaf(-fo, dz, fjz);
        const int src = (lane + 1) & 31;
        fjx = __shfl_sync(FULL, fjx, src);
        fjy = __shfl_sync(FULL, fjy, src);
        fjz = __shfl_sync(FULL, fjz, src);
      }
    }
    const float fs = (float)kForceScale;
    if (i < n) {
      add_fixed(s.force + i, to_fixed(fix, fs));
      add_fixed(s.force + n + i, to_fixed(fiy, fs));
      add_fixed(s.force + 2 * n + i, to_fixed(fiz, fs));
    }
    if (!self && j < n) {
      add_fixed(s.force + j, to_fixed(fjx, fs));
      add_fixed(s.force + n + j, to_fixed(fjy, fs));
      add_fixed(s.force + 2 * n + j, to_fixed(fjz, fs));
    }
    for (int off = 16; off > 0; off >>= 1) e_tile += __shfl_xor_sync(FULL, e_tile, off);
    e_fixed += to_fixed(e_tile, kEnergyScale);
    __syncwarp();
  }
  if (lane == 0 && e_fixed) add_fixed(s.energy, e_fixed);
}

__global__ void na_finish(int n, ScratchView s, double* forces, double* energy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *energy = (double)*s.energy * kEnergyScaleInv;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c) forces[3 * i + c] = (double)s.force[(long long)c * n + i] * kForceScaleInv;
}

}  // namespace

void nonbonded_forces_noalloc(int n, const double* pos, const double* q, const double* sigma,
                              const double* eps, int method, double cutoff, double rf_dielectric,
                              double* forces, double* energy, cudaStream_t stream) {
  if (n < 1 || n > kNoAllocMaxAtoms)
    throw Error(OMMB200_ERR_INVALID_ARG,
                "ommb200_nonbonded_forces_noalloc accepts 1 to 8192 particles (its static "
                "scratch holds 8192); use a Context for larger systems");
  if (method != OMMB200_NO_CUTOFF && method != OMMB200_CUTOFF_NON_PERIODIC)
    throw Error(OMMB200_ERR_INVALID_ARG, "the allocation-free path supports NoCutoff and CutoffNonPeriodic");
  if (!pos || !q || !sigma || !eps || !forces || !energy)
    throw Error(OMMB200_ERR_INVALID_ARG, "null device pointer");
  const bool cut = method == OMMB200_CUTOFF_NON_PERIODIC;
  if (cut && !(std::isfinite(cutoff) && cutoff > 0.0))
    throw Error(OMMB200_ERR_INVALID_ARG, "cutoff must be positive and finite");
  const ScratchInfo info = scratch_info();
  const ScratchView s = view(info.addr);
  const int blocks = (n + 31) / 32, slots = 32 * blocks;
  PairArgs<float> a{};
  a.pos = pos;
  a.use_cutoff = cut;
  a.cutoff2 = (float)(cutoff * cutoff);
  a.cutoff2_exact = cutoff * cutoff;
  a.band = (float)(cutoff * cutoff * 1e-4);
  if (cut) {
    const double rc3 = cutoff * cutoff * cutoff;
    const double krf = std::isinf(rf_dielectric) ? 0.5 / rc3
                                                 : (rf_dielectric - 1.0) / (2.0 * rf_dielectric + 1.0) / rc3;
    const double crf = std::isinf(rf_dielectric) ? 1.5 / cutoff
                                                 : (3.0 * rf_dielectric) / (2.0 * rf_dielectric + 1.0) / cutoff;
    a.krf = (float)krf;
    a.crf = (float)crf;
  }
  na_prepare<<<(slots + 255) / 256, 256, 0, stream>>>(n, slots, pos, q, sigma, eps, s);
  const long long tiles = (long long)blocks * (blocks + 1) / 2;
  const int grid = (int)std::min<long long>((tiles + 3) / 4, (long long)info.sm_count * 8);
  if (cut)
    na_pairs<kElecReactionField><<<grid, 128, 0, stream>>>(a, n, blocks, s);
  else
    na_pairs<kElecCoulomb><<<grid, 128, 0, stream>>>(a, n, blocks, s);
  na_finish<<<(n + 255) / 256, 256, 0, stream>>>(n, s, forces, energy);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(OMMB200_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
}

}  // namespace ommb200
