// peak_probe.cuh -- FP64 FMA throughput probe (roofline denominator).
// Every thread runs 8 independent FMA chains; the grid covers every SM with
// 8 CTAs of 256 threads.  FLOPs = 2 * threads * chains * iterations.
#pragma once
#include <cuda_runtime.h>

namespace pgb {

__global__ void __launch_bounds__(256) k_fp64_fma(int iters, double a, double b, double *sink) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == 123.456) sink[0] = s;  // never true; keeps the chains live
}

inline int fp64_peak_probe(double *tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return -3;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  k_fp64_fma<<<blocks, threads>>>(1024, 0.9999999, 1e-7, sink);  // warm-up
  double best = 0.0;
  for (int rep = 0; rep < 5; rep++) {
    cudaEventRecord(e0);
    k_fp64_fma<<<blocks, threads>>>(iters, 0.9999999, 1e-7, sink);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double fl = 2.0 * blocks * threads * 8.0 * iters;
    if (ms > 0) best = fl / (ms * 1e-3) / 1e12 > best ? fl / (ms * 1e-3) / 1e12 : best;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return -2;
  *tflops = best;
  return 0;
}

}  // namespace pgb
