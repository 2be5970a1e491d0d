// FP64 FMA throughput probe: the FP64 roofline denominator for the hydro
// kernels (which do no tensor-core work).  Every thread runs 8 independent
// DFMA chains so the pipe, not latency, bounds the loop.
#include <cuda_runtime.h>

#include "camr_b200.h"
#include "camr_common.cuh"
#include "rndiv.h"

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

// ---------------------------------------------------------------------------
// Device check of rn_div (rndiv.h) against the IEEE division: random
// operands over +-60 binades, quotients next to rounding midpoints and
// their neighbours, integer ratios, and special operands, from a
// splitmix64 stream per thread.
namespace {

__device__ __forceinline__ uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double unit12(uint64_t r) {  // in [1, 2)
  return __longlong_as_double(static_cast<long long>((r >> 12) | 0x3FF0000000000000ull));
}

__device__ __forceinline__ void rd_check(double a, double b, unsigned long long* bad) {
  const double y = 1.0 / b;
  const double q = camr::rn_div(a, b, y);
  const double w = a / b;
  if (__double_as_longlong(q) != __double_as_longlong(w) && !(isnan(q) && isnan(w)))
    atomicAdd(bad, 1ull);
}

__global__ void k_rn_div_check(int64_t n, uint64_t seed, unsigned long long* bad) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint64_t s = seed ^ (uint64_t(t) * 0xD1B54A32D192ED03ull);
  const uint64_t r1 = splitmix(s), r2 = splitmix(s), r3 = splitmix(s), r4 = splitmix(s);
  const double a = ((r3 & 1) ? 1.0 : -1.0) * scalbn(unit12(r1), int(r3 >> 1 & 127) % 121 - 60);
  const double b = ((r4 & 1) ? 1.0 : -1.0) * scalbn(unit12(r2), int(r4 >> 1 & 127) % 121 - 60);
  rd_check(a, b, bad);
  // next to the midpoint m between q and its successor: a = b * m with b an
  // odd integer of at most 13 bits times a power of two
  const uint64_t r5 = splitmix(s), r6 = splitmix(s);
  const double q = scalbn(unit12(r5), int(r6 & 63) % 41 - 20);
  const double m = q + 0.5 * (nextafter(q, 1e300) - q);
  const double bm = scalbn(double((r6 >> 8) % 4096 * 2 + 1), int(r6 >> 24 & 31) % 21 - 10);
  const double am = bm * m;
  rd_check(am, bm, bad);
  rd_check(nextafter(am, 1e300), bm, bad);
  rd_check(nextafter(am, -1e300), bm, bad);
  const uint64_t r7 = splitmix(s);
  rd_check(double(int64_t(r7 % 2000001) - 1000000), double(int64_t((r7 >> 32) % 2001) - 1000),
           bad);
  if (t == 0) {
    const double sp[] = {0.0, -0.0, 1.0, -1.0, 3.0, 0.1, 1e-7, 1e-200, -1e-300, 1e300,
                         scalbn(1.0, -500), scalbn(1.0, 499), scalbn(1.0, 500),
                         scalbn(1.0, -501), 5e-324, INFINITY, -INFINITY, NAN};
    for (double x : sp)
      for (double z : sp) rd_check(x, z, bad);
  }
}

}  // namespace

extern "C" camr_status camr_check_rn_div(int64_t n, uint64_t seed, int64_t* mismatches,
                                         void* stream) {
  if (n < 1 || !mismatches) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&bad, sizeof(*bad)) != cudaSuccess) return CAMR_ERR_NOMEM;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(*bad), st);
  if (e == cudaSuccess) {
    k_rn_div_check<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, seed, bad);
    e = cudaGetLastError();
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(bad);
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  *mismatches = int64_t(h);
  return CAMR_OK;
}
