// probe.cu -- nv_measure_fp64_peak: FP64 FMA throughput of this device, the denominator of
// the FP64 CUDA-core roofline (the driver's measured peaks cover HBM and tensor cores only).
#include "handle.cuh"

namespace {

// 8 independent FMA chains per thread, 2 flops each; enough warps to fill every pipe.
__global__ void __launch_bounds__(256) k_fma_probe(double *out, int iters, double a, double b) {
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-9 + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fma(r[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) k_fma_probe32(float *out, int iters, float a, float b) {
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-6f + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], a, b);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 12345.678f) out[0] = s;
}

}  // namespace

extern "C" int nv_measure_fp32_peak(int32_t device, double *tflops) {
  if (!tflops) return set_error(NV_ERR_ARG, "nv_measure_fp32_peak: null output");
  NV_CUDA(cudaSetDevice(device));
  int sms = 0;
  NV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *out = nullptr;
  NV_CUDA(cudaMalloc(&out, sizeof(float)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 8192;
  k_fma_probe32<<<blocks, threads>>>(out, 64, 0.999999f, 1e-7f);
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    k_fma_probe32<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  NV_CUDA(cudaGetLastError());
  *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
  return NV_OK;
}

extern "C" int nv_measure_fp64_peak(int32_t device, double *tflops) {
  if (!tflops) return set_error(NV_ERR_ARG, "nv_measure_fp64_peak: null output");
  NV_CUDA(cudaSetDevice(device));
  int sms = 0;
  NV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  double *out = nullptr;
  NV_CUDA(cudaMalloc(&out, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  k_fma_probe<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    k_fma_probe<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  NV_CUDA(cudaGetLastError());
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return NV_OK;
}
