// tb_fill.cuh -- matrix entries of the radial BEM fill: the off-diagonal
// 16-point Gauss sums and the singular self terms, shared by the single-
// geometry kernels and the batched persistent solve.
#pragma once

#include "tb_common.cuh"
#include "tb_internal.cuh"

namespace tb {

// Entry (i, j) of the matrix (radial.c:249-310): the collocation point of
// element i against the 16 Gauss rings of element j (staged in r[], z[], w[]),
// by the row's excitation type.
__device__ __forceinline__ double fill_entry(const double* __restrict__ vertices, const uint8_t* __restrict__ types,
                                             const double* __restrict__ values, int64_t i, const double* r,
                                             const double* z, const double* w) {
  Cubic cu;
  cu.load(vertices + i * 12);
  double tr, tz, tj;
  cu.point(0.0, false, tr, tz, tj);
  const int ty_ = types[i];
  double acc = 0.0;
  if (ty_ == VOLTAGE_FIXED || ty_ == VOLTAGE_FUN || ty_ == MAGNETOSTATIC_POT) {
#pragma unroll 4
    for (int k = 0; k < NQ; k++) acc += w[k] * (ring_pot_nopi(tr, tz, r[k], z[k]) * INV_PI);
  } else if (ty_ == DIELECTRIC || ty_ == MAGNETIZABLE) {
    double nr, nz;
    cu.normal(0.0, nr, nz);
    double f = flux_factor(values[i]);
#pragma unroll 4
    for (int k = 0; k < NQ; k++) acc += w[k] * field_dot_normal_ring(tr, tz, r[k] - tr, z[k] - tz, nr, nz, f);
  } else {
    acc = __longlong_as_double(0x7ff8000000000000LL);  // unknown type: NaN
  }
  return acc;
}

// ---------------------------------------------------------------- self terms
// Composite 16-point Gauss-Legendre on [-1, 0] and [0, 1], each split into
// the dyadic intervals [2^-(m+1), 2^-m], m < SELF_LEVELS, plus [0, 2^-L].
// The self integrand is smooth + smooth * log|alpha|, so each dyadic piece
// is integrated to ~1e-17 relative and the innermost piece contributes
// ~2^-L L log 2 of the total.
constexpr int SELF_LEVELS = 52;
constexpr int SELF_POINTS = 2 * (SELF_LEVELS + 1) * NQ;

__device__ __forceinline__ double self_integrand(const Cubic& c, double tr, double tz, double nr, double nz,
                                                 bool flux, double factor, double alpha) {
  double dr, dz, j;
  c.point(alpha, true, dr, dz, j);
  if (!flux) return j * potential_radial_ring(tr, tz, dr, dz);
  return j * field_dot_normal_ring(tr, tz, dr, dz, nr, nz, factor);
}

// Self term of element i by one warp (all lanes call it; every lane gets the value).
__device__ inline double self_term_warp(const double* __restrict__ vertices, const uint8_t* __restrict__ types,
                                        const double* __restrict__ values, int64_t i, int lane) {
  Cubic c;
  c.load(vertices + i * 12);
  double tr, tz, tj, nr, nz;
  c.point(0.0, false, tr, tz, tj);
  c.normal(0.0, nr, nz);
  int ty = types[i];
  bool flux = ty == DIELECTRIC || ty == MAGNETIZABLE;
  bool pot = ty == VOLTAGE_FIXED || ty == VOLTAGE_FUN || ty == MAGNETOSTATIC_POT;
  double factor = flux ? flux_factor(values[i]) : 0.0;
  double acc = 0.0;
  for (int p = lane; p < SELF_POINTS; p += 32) {
    int k = p % NQ;
    int lvl = (p / NQ) % (SELF_LEVELS + 1);
    double sgn = (p / (NQ * (SELF_LEVELS + 1))) ? 1.0 : -1.0;
    double hi = ldexp(1.0, -lvl);
    double lo = lvl == SELF_LEVELS ? 0.0 : 0.5 * hi;
    double half = 0.5 * (hi - lo), mid = 0.5 * (hi + lo);
    double a = sgn * (mid + half * gauss_x(k));
    acc += half * gauss_w(k) * self_integrand(c, tr, tz, nr, nz, flux, factor, a);
  }
  acc = warp_sum(acc);
  double v = flux ? acc - 1.0 : acc;
  if (!flux && !pot) v = __longlong_as_double(0x7ff8000000000000LL);  // unknown type: NaN
  return v;
}

}  // namespace tb
