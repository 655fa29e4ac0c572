// Measured issue-rate peaks of this GPU for the e-map's roofline: SFU
// reciprocal square roots per second and FP32 FMAs per second, each from a
// kernel of independent dependency chains that keeps every SM's pipe busy.
#include <cuda_runtime.h>

#include "../../include/fastgrid_b200.h"
#include "ag_device.cuh"

namespace {

constexpr int kChains = 8;

__global__ void rsqrt_peak_kernel(float* out, int iters, float seed) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) v[c] = seed + 0.25f * c + threadIdx.x * 1e-6f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = agd::rsqrt_approx(v[c]);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += v[c];
  if (s == -1.f) out[blockIdx.x] = s;  // never true; keeps the chains live
}

__global__ void ffma_peak_kernel(float* out, int iters, float seed) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) v[c] = seed + 0.25f * c + threadIdx.x * 1e-6f;
  const float a = 0.999999f, b = 1e-7f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = fmaf(v[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += v[c];
  if (s == -1.f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" int ag_measure_peaks(int device, double* rsqrt_per_s, double* ffma_per_s) {
  if (cudaSetDevice(device) != cudaSuccess) return AG_E_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * 65536) != cudaSuccess) return AG_E_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  double res[2] = {0, 0};
  for (int which = 0; which < 2; which++) {
    const int iters = which == 0 ? 4096 : 16384;
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
      cudaEventRecord(e0);
      if (which == 0) rsqrt_peak_kernel<<<blocks, threads>>>(out, iters, 1.5f);
      else ffma_peak_kernel<<<blocks, threads>>>(out, iters, 1.5f);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;
    }
    res[which] = (double)blocks * threads * iters * kChains / (best * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return AG_E_CUDA;
  if (rsqrt_per_s) *rsqrt_per_s = res[0];
  if (ffma_per_s) *ffma_per_s = res[1];
  return AG_OK;
}
