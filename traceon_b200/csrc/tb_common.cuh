// tb_common.cuh -- constants and the per-pair arithmetic of the radial BEM path.
//
// All functions here are FP64 and are shared by every kernel of the library.
// The algorithms are those of the reference C backend (Traceon v0.10.0,
// traceon/backend/*.c); each function names the routine it reproduces.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "tb_fastmath.cuh"

#define TB_HD __host__ __device__ __forceinline__

namespace tb {

constexpr int NQ = 16;              // N_QUAD_2D, utilities_2d.c:2
constexpr int NDERIV = 9;           // DERIV_2D_MAX, utilities_2d.c:89
constexpr int NTRI = 12;            // N_TRIANGLE_QUAD, utilities_3d.c
constexpr double MIN_AXIS = 1e-10;  // MIN_DISTANCE_AXIS, three_d.c:2
constexpr double MU0 = 1.25663706212e-06;   // MU_0, definitions.c:31
constexpr double STEP_MAX = 0.01;   // TRACING_STEP_MAX, tracing.c:5
constexpr double PI = 3.14159265358979323846;
constexpr double INV_PI = 0.31830988618379067154;

// Excitation type codes, definitions.c:34-40 / excitation.py:49-58
enum ExcitationType : uint8_t {
  VOLTAGE_FIXED = 1, VOLTAGE_FUN = 2, DIELECTRIC = 3, CURRENT = 4,
  MAGNETOSTATIC_POT = 5, MAGNETIZABLE = 6
};

// 16-point Gauss-Legendre nodes and weights in the reference's order,
// utilities_2d.c:3-4.
__host__ __device__ inline double gauss_x(int k) {
  constexpr double X[NQ] = {
      -0.0950125098376374, 0.0950125098376374, -0.2816035507792589, 0.2816035507792589,
      -0.4580167776572274, 0.4580167776572274, -0.6178762444026438, 0.6178762444026438,
      -0.7554044083550030, 0.7554044083550030, -0.8656312023878318, 0.8656312023878318,
      -0.9445750230732326, 0.9445750230732326, -0.9894009349916499, 0.9894009349916499};
  return X[k];
}
__host__ __device__ inline double gauss_w(int k) {
  constexpr double W[NQ] = {
      0.1894506104550685, 0.1894506104550685, 0.1826034150449236, 0.1826034150449236,
      0.1691565193950025, 0.1691565193950025, 0.1495959888165767, 0.1495959888165767,
      0.1246289712555339, 0.1246289712555339, 0.0951585116824928, 0.0951585116824928,
      0.0622535239386479, 0.0622535239386479, 0.0271524594117541, 0.0271524594117541};
  return W[k];
}

// ---------------------------------------------------------------- elliptic
// Cody (1965) log-polynomial forms K(1-p) = A(p) + log(1/p) B(p) and
// E(1-p) = C(p) + log(1/p) D(p), degree 7 (elliptic.c:9-35, :43-69),
// evaluated here by Horner's rule.
// The device forms read the coefficients from constant memory, which FP64
// FMA instructions take as a direct operand; literal 64-bit constants would
// have to be materialised into registers inside the hot loops.
__constant__ double C_KA[8] = {1.3862943611198906, 9.65736020516771e-2, 3.08909633861795e-2,
                               1.52618320622534e-2, 1.25565693543211e-2, 1.68695685967517e-2,
                               1.09423810688623e-2, 1.40704915496101e-3};
__constant__ double C_KB[8] = {0.5, 1.24999998585309e-1, 7.03114105853296e-2, 4.87379510945218e-2,
                               3.57218443007327e-2, 2.09857677336790e-2, 5.81807961871996e-3,
                               3.42805719229748e-4};
__constant__ double C_EA[8] = {1.0, 4.43147193467733e-1, 5.68115681053803e-2, 2.21862206993846e-2,
                               1.56847700239786e-2, 1.92284389022977e-2, 1.21819481486695e-2,
                               1.55618744745296e-3};
__constant__ double C_EB[8] = {0.0, 2.49999998448655e-1, 9.37488062098189e-2, 5.84950297066166e-2,
                               4.09074821593164e-2, 2.35091602564984e-2, 6.45682247315060e-3,
                               3.78886487349367e-4};

__device__ __forceinline__ double horner_c(const double* c, double p) {
  double s = c[7];
#pragma unroll
  for (int i = 6; i >= 0; i--) s = fma(s, p, c[i]);
  return s;
}

TB_HD double poly_ka(double p) {
#ifdef __CUDA_ARCH__
  return horner_c(C_KA, p);
#else
  return ((((((1.40704915496101e-3 * p + 1.09423810688623e-2) * p + 1.68695685967517e-2) * p +
             1.25565693543211e-2) * p + 1.52618320622534e-2) * p + 3.08909633861795e-2) * p +
          9.65736020516771e-2) * p + 1.3862943611198906;
#endif
}
TB_HD double poly_kb(double p) {
#ifdef __CUDA_ARCH__
  return horner_c(C_KB, p);
#else
  return ((((((3.42805719229748e-4 * p + 5.81807961871996e-3) * p + 2.09857677336790e-2) * p +
             3.57218443007327e-2) * p + 4.87379510945218e-2) * p + 7.03114105853296e-2) * p +
          1.24999998585309e-1) * p + 0.5;
#endif
}
TB_HD double poly_ea(double p) {
#ifdef __CUDA_ARCH__
  return horner_c(C_EA, p);
#else
  return ((((((1.55618744745296e-3 * p + 1.21819481486695e-2) * p + 1.92284389022977e-2) * p +
             1.56847700239786e-2) * p + 2.21862206993846e-2) * p + 5.68115681053803e-2) * p +
          4.43147193467733e-1) * p + 1.0;
#endif
}
TB_HD double poly_eb(double p) {
#ifdef __CUDA_ARCH__
  return horner_c(C_EB, p);
#else
  return ((((((3.78886487349367e-4 * p + 6.45682247315060e-3) * p + 2.35091602564984e-2) * p +
             4.09074821593164e-2) * p + 5.84950297066166e-2) * p + 9.37488062098189e-2) * p +
          2.49999998448655e-1) * p;
#endif
}

TB_HD double ellipkm1(double p) { return poly_ka(p) + log(1.0 / p) * poly_kb(p); }
TB_HD double ellipem1(double p) { return poly_ea(p) + log(1.0 / p) * poly_eb(p); }
// ellipk / ellipe, elliptic.c:37-41, :71-75 (branches as in the reference)
TB_HD double ellipk(double k) {
  if (k > -1) return ellipkm1(1 - k);
  return ellipkm1(1. / (1 - k)) / sqrt(k);
}
TB_HD double ellipe(double k) {
  if (0 <= k && k <= 1) return ellipem1(1 - k);
  return ellipem1(-1 / (k - 1.)) * sqrt(1 - k);
}

// ------------------------------------------------------- line elements
// A line4 element: vertex rows v[0] = start, v[1] = end, v[2] = 1/3-point,
// v[3] = 2/3-point, each (r, y, z) with y == 0.  The cubic Lagrange map
// alpha in [-1, 1] -> (r, z) has its nodes at -1, -1/3, 1/3, 1 in the order
// v[0], v[2], v[3], v[1] (radial.c:128-131, utilities_2d.c:50-87).
struct Cubic {
  double k0[2], k1[2], k2[2], k3[2];  // (r, z) coefficient vectors, times 16

  TB_HD void load(const double* v /* 12 doubles */) {
    for (int d = 0; d < 2; d++) {
      int c = d == 0 ? 0 : 2;
      double x0 = v[0 * 3 + c], x1 = v[2 * 3 + c], x2 = v[3 * 3 + c], x3 = v[1 * 3 + c];
      k3[d] = 9 * x3 - 27 * x2 + 27 * x1 - 9 * x0;
      k2[d] = 9 * x3 - 9 * x2 - 9 * x1 + 9 * x0;
      k1[d] = -x3 + 27 * x2 - 27 * x1 + x0;
      k0[d] = -x3 + 9 * x2 + 9 * x1 - x0;
    }
  }
  // from four (r, y, z) points in parametric order (alpha = -1, -1/3, 1/3, 1)
  TB_HD void load4(const double* p0, const double* p1, const double* p2, const double* p3) {
    double v[12];
    for (int c = 0; c < 3; c++) {
      v[0 * 3 + c] = p0[c];
      v[2 * 3 + c] = p1[c];
      v[3 * 3 + c] = p2[c];
      v[1 * 3 + c] = p3[c];
    }
    load(v);
  }
  // position (delta == false) or position relative to alpha = 0 (delta == true)
  TB_HD void point(double a, bool delta, double& r, double& z, double& jac) const {
    double a2 = a * a, a3 = a2 * a;
    r = (a2 * k2[0] + a3 * k3[0] + a * k1[0] + (delta ? 0.0 : k0[0])) / 16;
    z = (a2 * k2[1] + a3 * k3[1] + a * k1[1] + (delta ? 0.0 : k0[1])) / 16;
    double dr = 2 * a * k2[0] + 3 * a2 * k3[0] + k1[0];
    double dz = 2 * a * k2[1] + 3 * a2 * k3[1] + k1[1];
    jac = sqrt(dr * dr + dz * dz) / 16.;
  }
  // unit normal (dz, -dr)/|.| at alpha, higher_order_normal_radial,
  // utilities_2d.c:31-48 with normal_2d :18-29
  TB_HD void normal(double a, double& nr, double& nz) const {
    double a2 = a * a;
    double tr = (2 * a * k2[0] + 3 * a2 * k3[0] + k1[0]) / 16;
    double tz = (2 * a * k2[1] + 3 * a2 * k3[1] + k1[1]) / 16;
    double l = sqrt(tz * tz + tr * tr);
    nr = tz / l;
    nz = -tr / l;
  }
};

// ------------------------------------------------------- ring kernels
// Geometry of one (observation point, source ring) pair.  (r0, z0) is the
// observation point, (rs, zs) the ring.  With dr = rs - r0, dz = zs - z0:
//   rho2 = dr^2 + dz^2,  D = dz^2 + (rs + r0)^2,  t = rho2 / D = 1 - k^2.
// potential_radial_ring (radial_ring.c:37-43)
//   phi = (1/pi) K(1-t) rs / sqrt(D)
// dr1_potential_radial_ring (radial_ring.c:21-35)
//   d phi/d r0 = -(1/(2 pi r0)) rs (rho2 K + (dr^2 - 2 dr rs - dz^2) E) / (rho2 sqrt(D))
// dz1_potential_radial_ring (radial_ring.c:45-53)
//   d phi/d z0 = (1/pi) dz rs E / (rho2 sqrt(D))
// (the reference's denominators (-2 dr^2 r + dz^2 (2dr - 2r) + 2 dr^3) and
// 4 r^2 - 4 dr r + rho2 reduce to -2 r0 rho2 and D).

// Degree-7 polynomial by Estrin's scheme (depth 3 instead of Horner's 7),
// given t, t^2 and t^4 shared by the four Cody polynomials.
__device__ __forceinline__ double estrin8(const double* c, double t, double t2, double t4) {
  double a = fma(c[1], t, c[0]);
  double b = fma(c[3], t, c[2]);
  double d = fma(c[5], t, c[4]);
  double e = fma(c[7], t, c[6]);
  return fma(t4, fma(t2, e, d), fma(t2, b, a));
}

// Potential of a unit ring, without the 1/pi factor: K(1-t) rs / sqrt(D).
__device__ __forceinline__ double ring_pot_nopi(double r0, double z0, double rs, double zs) {
  double dr = rs - r0, dz = zs - z0;
  double dz2 = dz * dz;
  double rho2 = fma(dr, dr, dz2);
  double s = rs + r0;
  double D = fma(s, s, dz2);
  double rD = rsqrt_nr(D);
  double t = rho2 * rD * rD;
  double t2 = t * t, t4 = t2 * t2;
  double K = fma(-log_bf(t), estrin8(C_KB, t, t2, t4), estrin8(C_KA, t, t2, t4));
  return K * rs * rD;
}

// Accumulates one weighted ring into the partial field sums.  After the
// whole reduction, E_r = Sr / (2 pi r0) (0 on the axis) and E_z = -Sz / pi.
// Optionally accumulates the potential sum Sp (phi = Sp / pi).
template <bool WANT_POT>
__device__ __forceinline__ void ring_field_acc(double r0, double z0, double rs, double zs, double w,
                                               double& Sr, double& Sz, double& Sp) {
  double dr = rs - r0, dz = zs - z0;
  double dz2 = dz * dz;
  double rho2 = fma(dr, dr, dz2);
  double s = rs + r0;
  double D = fma(s, s, dz2);
  double ir = rcp_nr(rho2);        // 1 / rho2
  double rD = rsqrt_nr(D);         // 1 / sqrt(D)
  double t = rho2 * rD * rD;       // rho2 / D
  double t2 = t * t, t4 = t2 * t2;
  double L = -log_bf(t);
  double K = fma(L, estrin8(C_KB, t, t2, t4), estrin8(C_KA, t, t2, t4));
  double E = fma(L, estrin8(C_EB, t, t2, t4), estrin8(C_EA, t, t2, t4));
  double c = w * rs * rD * ir;     // w rs / (rho2 sqrt(D))
  double m = fma(dr, dr - 2.0 * rs, -dz2);   // dr^2 - 2 dr rs - dz^2
  Sr = fma(c, fma(rho2, K, m * E), Sr);
  Sz = fma(c * dz, E, Sz);
  if (WANT_POT) Sp = fma(c * rho2, K, Sp);
}

// Scalar forms with the reference's argument convention (r0, z0, delta_r,
// delta_z), used by the exported scalar helpers and by the matrix fill.
TB_HD double potential_radial_ring(double r0, double z0, double dr, double dz) {
  (void)z0;
  double rho2 = dz * dz + dr * dr;
  double s = dr + 2 * r0;
  double D = dz * dz + s * s;
  double t = rho2 / D;
  return INV_PI * ellipkm1(t) * (dr + r0) / sqrt(D);
}
TB_HD double dr1_potential_radial_ring(double r0, double z0, double dr, double dz) {
  (void)z0;
  if (r0 < MIN_AXIS) return 0.0;
  double rs = r0 + dr;
  double rho2 = dz * dz + dr * dr;
  double s = rs + r0;
  double D = dz * dz + s * s;
  double t = rho2 / D;
  double L = log(1.0 / t);
  double K = poly_ka(t) + L * poly_kb(t);
  double E = poly_ea(t) + L * poly_eb(t);
  return -INV_PI * rs * (rho2 * K + (dr * dr - 2 * dr * rs - dz * dz) * E) / (2 * r0 * rho2 * sqrt(D));
}
TB_HD double dz1_potential_radial_ring(double r0, double z0, double dr, double dz) {
  (void)z0;
  double rs = r0 + dr;
  double rho2 = dz * dz + dr * dr;
  double s = rs + r0;
  double D = dz * dz + s * s;
  double t = rho2 / D;
  double E = ellipem1(t);
  return INV_PI * dz * rs * E / (rho2 * sqrt(D));
}

// flux_density_to_charge_factor, utilities_2d.c:91-105
TB_HD double flux_factor(double K) { return 2.0 * (K - 1) / (1 + K); }

// factor * n . E at (r0, z0) of a unit ring (field_dot_normal_radial,
// radial_ring.c:55-71), with both derivatives sharing one log.
TB_HD double field_dot_normal_ring(double r0, double z0, double dr, double dz, double nr, double nz,
                                   double factor) {
  (void)z0;
  double rs = r0 + dr;
  double rho2 = dz * dz + dr * dr;
  double s = rs + r0;
  double D = dz * dz + s * s;
  double t = rho2 / D;
  double L = log(1.0 / t);
  double K = poly_ka(t) + L * poly_kb(t);
  double E = poly_ea(t) + L * poly_eb(t);
  double inv = 1.0 / (rho2 * sqrt(D));
  double Er = 0.0;
  if (r0 >= MIN_AXIS) Er = INV_PI * rs * (rho2 * K + (dr * dr - 2 * dr * rs - dz * dz) * E) * inv / (2 * r0);
  double Ez = -INV_PI * dz * rs * E * inv;
  return factor * (nr * Er + nz * Ez);
}

// current_field_radial_ring, radial_ring.c:78-107: (H_r, H_z) at (x0, y0)
// of a unit current loop of radius x at height y.
TB_HD void current_field_ring(double x0, double y0, double x, double y, double& hr, double& hz) {
  double a = x, r = x0, z = y0 - y;
  double A = z * z + (a + r) * (a + r);
  double B = z * z + (r - a) * (r - a);
  double k = 4 * r * a / A;
  if (x < MIN_AXIS) {
    hr = 0.;
    hz = 0.;
    return;
  }
  double Ek = ellipe(k), Kk = ellipk(k);
  if (x0 < MIN_AXIS)
    hr = 0.;
  else
    hr = INV_PI * z / (2 * r * sqrt(A)) * ((z * z + r * r + a * a) / B * Ek - Kk);
  hz = INV_PI / (2 * sqrt(A)) * ((a * a - z * z - r * r) / B * Ek + Kk);
}

// axial_derivatives_radial_ring, radial_ring.c:109-122: the 9 derivatives
// d^n/dz0^n of r/(2 |(z0 - z, r)|) by the three-term recurrence.
TB_HD void axial_ring(double z0, double r, double z, double w, double* acc /* 9 */) {
  double dz = z0 - z;
  double R2 = dz * dz + r * r;
  double invR2 = 1.0 / R2;
  double R = sqrt(R2);
  double d0 = 1.0 / R;
  double d1 = -dz * d0 * invR2;
  double ws = w * r * 0.5;
  acc[0] = fma(ws, d0, acc[0]);
  acc[1] = fma(ws, d1, acc[1]);
  double pm = d0, pc = d1;
#pragma unroll
  for (int n = 1; n + 1 < NDERIV; n++) {
    double nx = -invR2 * ((2 * n + 1) * dz * pc + double(n * n) * pm);
    acc[n + 1] = fma(ws, nx, acc[n + 1]);
    pm = pc;
    pc = nx;
  }
}

// current_axial_derivatives_radial_ring, radial_ring.c:124-136
TB_HD void current_axial_ring(double z0, double r, double z, double w, double* acc) {
  double dz = z0 - z;
  double R2 = dz * dz + r * r, R = sqrt(R2), mu = dz / R;
  double dm = -dz / (2 * R);
  double dc = -r * r / (2 * R2 * R);
  acc[0] = fma(w, dm, acc[0]);
  acc[1] = fma(w, dc, acc[1]);
#pragma unroll
  for (int n = 2; n < NDERIV; n++) {
    double nx = -(2 * n - 1) * mu / R * dc - double(n * n - 2 * n) / R2 * dm;
    acc[n] = fma(w, nx, acc[n]);
    dm = dc;
    dc = nx;
  }
}

// Status codes returned by every entry point of the C ABI.
enum Status : int {
  OK = 0,
  BAD_ARG = 1,
  CUDA_ERR = 2,
  NONFINITE = 3,
  UNSUPPORTED = 4,
  SINGULAR = 5,
  TIMEOUT = 6,  // a bounded wait inside a kernel ran out
};

// Per-particle tracer status.
enum TraceStatus : int {
  TRACE_EXITED = 0,        // left the bounds (normal end)
  TRACE_MAX_ATTEMPTS = 1,  // step-attempt cap reached
  TRACE_ROWS_FULL = 2,     // trajectory buffer full; resume from the last row
  TRACE_NONFINITE = 3,     // state became non-finite
  TRACE_ENGINE_TIMEOUT = 4,  // the tensor-core engine's bounded MMA wait ran out; particle abandoned
};

}  // namespace tb
