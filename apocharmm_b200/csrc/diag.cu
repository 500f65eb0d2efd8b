// FP32 peak probe: dependent-free FMA chains, 8 independent accumulators per
// thread, one resident wave per SM pair; reports FLOP/s of the device.
#include <cuda_runtime.h>

#include "capi_internal.h"

namespace {
__global__ void fma_probe_kernel(float *out, int iters, float a, float b) {
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
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains alive
}
}  // namespace

extern "C" apo_status apo_diag_fp32_peak_tflops(double *tflops) {
  const char *fn = "apo_diag_fp32_peak_tflops";
  return apocapi::guard([&]() -> apo_status {
    APO_RETURN_IF(apocapi::require_ptr(tflops, fn, "tflops"));
    int dev, nsm;
    APO_CUDA(cudaGetDevice(&dev));
    APO_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    float *out;
    APO_CUDA(cudaMalloc(&out, 1024 * sizeof(float)));
    const int threads = 1024, blocks = nsm * 2, iters = 20000;
    cudaEvent_t e0, e1;
    APO_CUDA(cudaEventCreate(&e0));
    APO_CUDA(cudaEventCreate(&e1));
    fma_probe_kernel<<<blocks, threads>>>(out, 100, 0.999f, 1e-4f);
    APO_CUDA(cudaEventRecord(e0));
    fma_probe_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-4f);
    APO_CUDA(cudaEventRecord(e1));
    APO_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    APO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
    return APO_STATUS_OK;
  }, fn);
}
