// Correctly rounded quotients that share a divisor.  A quotient a / b is
// formed from y = RN(1/b), computed once by an IEEE division and shared by
// every quotient with the same divisor, with the fused multiply-add
// corrections of P. Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990 (see also
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, the chapter
// on division with an FMA):
//
//   q0 = RN(a y)                      relative error below 2u + u^2
//   q1 = RN(q0 + RN(a - b q0) y)      error O(u^2) before its rounding, so
//                                     q1 is within one ulp of a/b
//   q  = RN(q1 + RN(a - b q1) y)      with y = RN(1/b) and q1 faithful, the
//                                     remainder a - b q1 is exact and q is
//                                     RN(a/b) (Markstein's theorem)
//
// (u = 2^-53).  The theorem needs no overflow or underflow in the
// intermediates: operands whose magnitudes lie in [2^-500, 2^500) keep q,
// both remainders and y far inside the normal range; any other operand
// (zero, subnormal, huge, infinite, NaN) takes the IEEE division, so the
// result always equals `a / b` in round-to-nearest-even, bit for bit.
// The kernels are compiled without FMA contraction, and these are the only
// fused operations: each replaces a full division by one multiply and four
// fused multiply-adds.  A host compiler can include this header on its own.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define CAMR_RD __host__ __device__ __forceinline__
#else
#include <cmath>
#define CAMR_RD inline
#endif

namespace camr {

CAMR_RD int rd_biased_exponent(double x) {
#if defined(__CUDA_ARCH__)
  return (__double2hiint(x) >> 20) & 0x7ff;
#else
  uint64_t u;
  memcpy(&u, &x, sizeof(u));
  return int((u >> 52) & 0x7ff);
#endif
}

CAMR_RD double rd_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

// |x| in [2^-500, 2^500): the operand range of rn_div_unchecked.
CAMR_RD bool rd_in_range(double x) { return unsigned(rd_biased_exponent(x) - 523) < 1000u; }

// a / b from y = RN(1/b) when the caller has checked rd_in_range(a) and
// rd_in_range(b) (for a group of quotients at once, so that the group's
// quotients form one branch-free block).
CAMR_RD double rn_div_unchecked(double a, double b, double y) {
  const double q0 = a * y;
  const double q1 = rd_fma(rd_fma(-b, q0, a), y, q0);
  return rd_fma(rd_fma(-b, q1, a), y, q1);
}

// q[m] = n[m] / b for m < M, rounded to nearest even: with b and every
// n[m] in range, from one reciprocal in a branch-free block; otherwise by
// the divisions.
template <int M>
CAMR_RD void rn_div_group(const double* n, double b, double* q) {
  bool ok = rd_in_range(b);
#pragma unroll
  for (int m = 0; m < M; ++m) ok = ok & rd_in_range(n[m]);
  if (ok) {
    const double y = 1.0 / b;
#pragma unroll
    for (int m = 0; m < M; ++m) q[m] = rn_div_unchecked(n[m], b, y);
  } else {
#pragma unroll
    for (int m = 0; m < M; ++m) q[m] = n[m] / b;
  }
}

// a / b given y = 1.0 / b (an IEEE division), rounded to nearest even.
CAMR_RD double rn_div(double a, double b, double y) {
  // biased exponents 523..1522: magnitudes in [2^-500, 2^500)
  if (unsigned(rd_biased_exponent(a) - 523) < 1000u &&
      unsigned(rd_biased_exponent(b) - 523) < 1000u) {
    const double q0 = a * y;
    const double q1 = rd_fma(rd_fma(-b, q0, a), y, q0);
    return rd_fma(rd_fma(-b, q1, a), y, q1);
  }
  return a / b;
}

}  // namespace camr
