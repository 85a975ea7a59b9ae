// tb_fastmath.cuh -- branch-free FP64 reciprocal, reciprocal square root and
// logarithm for the ring-pair loops.
//
// The library functions behind 1.0/x, sqrt(x) and log(x) carry special-case
// branches (zero, infinity, NaN, subnormals) that split the hot loops into
// divergence regions and keep the compiler from interleaving consecutive
// pairs.  The ring-pair arguments are always positive normal numbers, so
// these versions drop the special cases:
//
//  * rcp_nr / rsqrt_nr: the PTX hardware approximations rcp.approx.ftz.f64 /
//    rsqrt.approx.ftz.f64 (about 2^-22 relative) refined by Newton-Raphson
//    iterations written out below (for 1/x: y <- y + y e, e = 1 - x y; for
//    1/sqrt(x): y <- y + y e (1/2 + 3/8 e), e = 1 - x y^2), which square
//    (resp. cube) the relative error per step.
//  * log_bf: Cody & Waite argument reduction t = 2^k m, m in [sqrt(1/2),
//    sqrt(2)), then log m = 2 atanh(s), s = (m - 1)/(m + 1), summed as the
//    odd series 2 (s + s^3/3 + s^5/5 + ...) through s^21 (|s| <= 0.1716, so
//    the next term is below 2^-55 of the sum), and k log 2 added in two parts
//    (log 2 split into a 32-bit head and its remainder).
// All three are accurate to about 1 ulp (checked against the library
// functions by tests/test_gpu_kernels.py through tb_probe_math).
#pragma once

#include <cstdint>

namespace tb {

__device__ __forceinline__ double rcp_approx(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

__device__ __forceinline__ double rsqrt_approx(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

// 1/x for positive normal x.
__device__ __forceinline__ double rcp_nr(double x) {
  double y = rcp_approx(x);
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// 1/sqrt(x) for positive normal x.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y = rsqrt_approx(x);
  double e = fma(-x * y, y, 1.0);
  y = fma(y * e, fma(0.375, e, 0.5), y);
  e = fma(-x * y, y, 1.0);
  return fma(y * e, 0.5, y);
}

// Coefficients 1/(2j+1), j = 1..10, of the atanh series.
__constant__ double C_ATANH[10] = {1.0 / 3,  1.0 / 5,  1.0 / 7,  1.0 / 9,  1.0 / 11,
                                   1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19, 1.0 / 21};

// log(t) for positive normal t.
__device__ __forceinline__ double log_bf(double t) {
  const long long bits = __double_as_longlong(t);
  int k = int((bits >> 52) & 0x7ff) - 1023;
  double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);  // [1, 2)
  const bool big = m > 1.4142135623730951;
  m = big ? 0.5 * m : m;
  k += big ? 1 : 0;
  const double f = m - 1.0;            // exact (Sterbenz)
  const double s = f * rcp_nr(2.0 + f);
  const double s2 = s * s;
  double p = C_ATANH[9];
#pragma unroll
  for (int j = 8; j >= 0; j--) p = fma(p, s2, C_ATANH[j]);
  // log m = 2 s + 2 s^3 P(s^2)
  const double logm = fma(2.0 * s * s2, p, 2.0 * s);
  const double kd = double(k);
  const double LN2_HI = 0.6931471803691238;     // log 2 with its significand cut to 32 bits
  const double LN2_LO = 1.9082149292705877e-10;  // log 2 - LN2_HI, rounded
  return fma(kd, LN2_HI, fma(kd, LN2_LO, logm));
}

}  // namespace tb
