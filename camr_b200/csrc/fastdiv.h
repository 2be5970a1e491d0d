// Flat-index decoding without 64-bit division, shared by host and device
// code (the host side builds the divisors; a host compiler can include this
// header on its own).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define CAMR_HD __host__ __device__ __forceinline__
#else
#define CAMR_HD inline
#endif

// 0: every decode divides in 64 bits (the comparison build).
#ifndef CAMR_FASTDIV
#define CAMR_FASTDIV 1
#endif

namespace camr {

// Quotient of a non-negative index below 2^31 by an invariant divisor with
// one multiply-high and a shift instead of a 64-bit division (Granlund &
// Montgomery, "Division by Invariant Integers using Multiplication", PLDI
// 1994): m = ceil(2^p / d) with p = 31 + ceil(log2 d) gives
// floor(n / d) = floor(n m / 2^p) for all n < 2^31, since m - 2^p/d < 1 makes
// the error n (m - 2^p/d) / 2^p < 2^-ceil(log2 d) <= 1/d.  m == 0: d == 1.
struct FastDiv {
  unsigned m;
  int s;  // p - 32
};

inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f{0u, 0};
  if (d <= 1) return f;
  int l = 0;
  while ((1ull << l) < d) ++l;
  const int p = 31 + l;
  f.m = unsigned(((1ull << p) + d - 1) / d);
  f.s = p - 32;
  return f;
}

CAMR_HD unsigned fastdiv(unsigned n, FastDiv f) {
#ifdef __CUDA_ARCH__
  return f.m ? (__umulhi(n, f.m) >> f.s) : n;
#else
  return f.m ? unsigned((static_cast<unsigned long long>(n) * f.m) >> 32) >> f.s : n;
#endif
}

// Flat index t < n0*n1*n2 -> (i, j, k) offsets, i fastest; the fast path
// when the extent is below 2^31 (fast != 0).
struct Decode3 {
  int n0, n01;
  int fast;
  FastDiv d0, d01;
};

inline Decode3 make_decode3(int n0, int n1, int n2) {
  Decode3 c;
  c.n0 = n0;
  c.n01 = n0 * n1;
  c.fast = CAMR_FASTDIV && int64_t(n0) * n1 * n2 < (int64_t(1) << 31) && n0 > 0 && n1 > 0;
  c.d0 = make_fastdiv(c.fast ? unsigned(n0) : 1u);
  c.d01 = make_fastdiv(c.fast ? unsigned(c.n01) : 1u);
  return c;
}

CAMR_HD void decode3(const Decode3& c, int64_t t, int& i, int& j,
                                                 int& k) {
  if (c.fast) {
    const unsigned u = unsigned(t);
    const unsigned kk = fastdiv(u, c.d01);
    const unsigned r = u - kk * unsigned(c.n01);
    const unsigned jj = fastdiv(r, c.d0);
    i = int(r - jj * unsigned(c.n0));
    j = int(jj);
    k = int(kk);
  } else {
    const int64_t nxy = int64_t(c.n01);
    k = int(t / nxy);
    const int64_t r = t - int64_t(k) * nxy;
    j = int(r / c.n0);
    i = int(r - int64_t(j) * c.n0);
  }
}

}  // namespace camr
