// Diagnostics with no reference counterpart: FP32 FMA throughput of the device, used as the
// roofline denominator of the FP32 pair kernel.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/ommb200.h"
#include "model.h"

namespace ommb200 {
namespace {

// Eight independent FMA chains per thread keep every FP32 pipe busy.
__global__ void __launch_bounds__(256) fma_probe(float* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

}  // namespace

double measure_fp32_peak(int device) {
  if (cudaSetDevice(device) != cudaSuccess) throw Error(OMMB200_ERR_CUDA, "cudaSetDevice failed");
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) throw Error(OMMB200_ERR_CUDA, "cudaMalloc failed");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  fma_probe<<<blocks, threads>>>(out, 64, 0.999f, 1e-4f);
  double best = 0.0;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(t0);
    fma_probe<<<blocks, threads>>>(out, iters, 0.999f, 1e-4f);
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    if (ms > 0.f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) throw Error(OMMB200_ERR_CUDA, cudaGetErrorString(err));
  return best;
}

}  // namespace ommb200
