// FP64 FMA throughput probe: the FP64 roofline denominator for the hydro
// kernels (which do no tensor-core work).  Every thread runs 8 independent
// DFMA chains so the pipe, not latency, bounds the loop.
#include <cuda_runtime.h>

#include "camr_b200.h"
#include "camr_common.cuh"

namespace {

constexpr int kIters = 4096;
constexpr int kChains = 8;

__global__ void k_dfma(double* out, double b, double c) {
  double a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) a[i] = threadIdx.x * 1e-9 + i;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += a[i];
  if (s == 1.2345) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" camr_status camr_measure_fp64_peak(double* tflops, void* stream) {
  if (!tflops) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return CAMR_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = nsm * 8, threads = 256;
  k_dfma<<<blocks, threads, 0, st>>>(out, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0, st);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) k_dfma<<<blocks, threads, 0, st>>>(out, 0.999999, 1e-7);
  cudaEventRecord(e1, st);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  camr::count_launch(reps + 1);
  const double flops = 2.0 * double(kIters) * kChains * double(blocks) * threads * reps;
  *tflops = flops / (double(ms) * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return e == cudaSuccess ? CAMR_OK : CAMR_ERR_CUDA;
}
