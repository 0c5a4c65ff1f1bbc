// FP32 FMA throughput probe used as the roofline denominator of the force
// kernel (no measured FP32 figure is provided for the device otherwise).
#include <cuda_runtime.h>

#include "../../include/pb/pb.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_ffma(float *out, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
  }
  float s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int pb_peak_fp32(double *tflops) {
  if (!tflops) return PB_ERR_ARG;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PB_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess) return PB_ERR_OOM;
  const int blocks = sms * 8;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_ffma<<<blocks, 256>>>(out, 0.999999f, 1e-7f);  // warm-up
  cudaEventRecord(a);
  const int reps = 10;
  for (int r = 0; r < reps; ++r) k_ffma<<<blocks, 256>>>(out, 0.999999f, 1e-7f);
  cudaEventRecord(b);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0) return PB_ERR_CUDA;
  const double flops = 2.0 * kChains * kIters * 256.0 * blocks * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return PB_OK;
}
