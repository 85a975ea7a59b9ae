/*
 * traceon_oracle.c -- CPU restatement of Traceon's radial-symmetric BEM path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the test oracle of the CUDA library in
 * traceon_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product path never calls it.
 *
 * Every function restates an algorithm of the reference C backend
 * (traceon/backend/*.c, Traceon v0.10.0) in plain FP64 C; the citation is in
 * the comment above each function.  Parity of this restatement is pinned in
 * tests/test_oracle.py against (a) the reference backend compiled from its own
 * sources into oracle/_ref/ and (b) the golden vectors in tests/golden/ that
 * the reference Python package produced (tests/golden/make_golden.py).
 *
 * Differences that are deliberate and do not change results beyond FP64
 * rounding: polynomials are evaluated by Horner's rule instead of sum of
 * pow(p, i) terms; no -ffast-math.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define OR_PI 3.14159265358979323846
#define OR_NQ 16            /* N_QUAD_2D, utilities_2d.c:2 */
#define OR_NDERIV 9         /* DERIV_2D_MAX, utilities_2d.c:89 */
#define OR_NTRI 12          /* N_TRIANGLE_QUAD, utilities_3d.c */
#define OR_MIN_AXIS 1e-10   /* MIN_DISTANCE_AXIS, three_d.c:2 */
#define OR_MU0 1.25663706212e-06 /* MU_0, definitions.c:31 */
#define OR_STEP_MAX 0.01    /* TRACING_STEP_MAX, tracing.c:5 */

/* 16-point Gauss-Legendre rule on [-1, 1] in the reference's node order
 * (utilities_2d.c:3-4). */
static const double OR_GW[OR_NQ] = {
    0.1894506104550685, 0.1894506104550685, 0.1826034150449236, 0.1826034150449236,
    0.1691565193950025, 0.1691565193950025, 0.1495959888165767, 0.1495959888165767,
    0.1246289712555339, 0.1246289712555339, 0.0951585116824928, 0.0951585116824928,
    0.0622535239386479, 0.0622535239386479, 0.0271524594117541, 0.0271524594117541};
static const double OR_GX[OR_NQ] = {
    -0.0950125098376374, 0.0950125098376374, -0.2816035507792589, 0.2816035507792589,
    -0.4580167776572274, 0.4580167776572274, -0.6178762444026438, 0.6178762444026438,
    -0.7554044083550030, 0.7554044083550030, -0.8656312023878318, 0.8656312023878318,
    -0.9445750230732326, 0.9445750230732326, -0.9894009349916499, 0.9894009349916499};

/* ---------------------------------------------------------------- elliptic */

/* Cody (1965) coefficients of K(1-p) = sum_i (a_i + L b_i) p^i, L = log(1/p)
 * (elliptic.c:9-35).  Index 0 of the a-row is log(4). */
static const double OR_KA[8] = {1.3862943611198906, 9.65736020516771e-2, 3.08909633861795e-2,
    1.52618320622534e-2, 1.25565693543211e-2, 1.68695685967517e-2, 1.09423810688623e-2,
    1.40704915496101e-3};
static const double OR_KB[8] = {0.5, 1.24999998585309e-1, 7.03114105853296e-2,
    4.87379510945218e-2, 3.57218443007327e-2, 2.09857677336790e-2, 5.81807961871996e-3,
    3.42805719229748e-4};
/* Same form for E(1-p) (elliptic.c:43-69). */
static const double OR_EA[8] = {1.0, 4.43147193467733e-1, 5.68115681053803e-2,
    2.21862206993846e-2, 1.56847700239786e-2, 1.92284389022977e-2, 1.21819481486695e-2,
    1.55618744745296e-3};
static const double OR_EB[8] = {0.0, 2.49999998448655e-1, 9.37488062098189e-2,
    5.84950297066166e-2, 4.09074821593164e-2, 2.35091602564984e-2, 6.45682247315060e-3,
    3.78886487349367e-4};

static double horner8(const double *c, double p) {
    double s = c[7];
    for (int i = 6; i >= 0; i--) s = s * p + c[i];
    return s;
}

/* elliptic.c:9-35 */
double or_ellipkm1(double p) {
    double L = log(1.0 / p);
    return horner8(OR_KA, p) + L * horner8(OR_KB, p);
}
/* elliptic.c:43-69 */
double or_ellipem1(double p) {
    double L = log(1.0 / p);
    return horner8(OR_EA, p) + L * horner8(OR_EB, p);
}
/* elliptic.c:37-41 (the k <= -1 branch is kept as the reference has it) */
double or_ellipk(double k) {
    if (k > -1) return or_ellipkm1(1 - k);
    return or_ellipkm1(1. / (1 - k)) / sqrt(k);
}
/* elliptic.c:71-75 */
double or_ellipe(double k) {
    if (0 <= k && k <= 1) return or_ellipem1(1 - k);
    return or_ellipem1(-1 / (k - 1.)) * sqrt(1 - k);
}

/* ------------------------------------------------------- line elements */

/* Cubic Lagrange element through (r,z) nodes at alpha = -1, -1/3, 1/3, 1.
 * The reference stores the nodes of a line4 element as vertex rows
 * [0], [2], [3], [1] (radial.c:128-131), i.e. row 0 = start, row 1 = end,
 * row 2 = 1/3-point, row 3 = 2/3-point.  position_and_jacobian_radial,
 * utilities_2d.c:50-66.  `delta` != 0 gives the position relative to
 * alpha = 0 (delta_position_and_jacobian_radial, utilities_2d.c:68-87). */
static void or_element_point(double alpha, const double v[4][3], int delta,
                             double pos[2], double *jac) {
    /* nodes in parametric order */
    const double *n0 = v[0], *n1 = v[2], *n2 = v[3], *n3 = v[1];
    double a2 = alpha * alpha, a3 = a2 * alpha;
    double c[2], d[2];
    for (int d_ = 0; d_ < 2; d_++) {
        int col = d_ == 0 ? 0 : 2;
        double x0 = n0[col], x1 = n1[col], x2 = n2[col], x3 = n3[col];
        double k3 = 9 * x3 - 27 * x2 + 27 * x1 - 9 * x0;
        double k2 = 9 * x3 - 9 * x2 - 9 * x1 + 9 * x0;
        double k1 = -x3 + 27 * x2 - 27 * x1 + x0;
        double k0 = -x3 + 9 * x2 + 9 * x1 - x0;
        c[d_] = (a2 * k2 + a3 * k3 + alpha * k1 + (delta ? 0.0 : k0)) / 16;
        d[d_] = 2 * alpha * k2 + 3 * a2 * k3 + k1;
    }
    pos[0] = c[0];
    pos[1] = c[1];
    *jac = sqrt(d[0] * d[0] + d[1] * d[1]) / 16.;
}

void or_position_and_jacobian_radial(double alpha, const double v[4][3], double pos[2], double *jac) {
    or_element_point(alpha, v, 0, pos, jac);
}
void or_delta_position_and_jacobian_radial(double alpha, const double v[4][3], double pos[2], double *jac) {
    or_element_point(alpha, v, 1, pos, jac);
}

/* Unit normal (dz/dalpha, -dr/dalpha)/|.| of the cubic element
 * (higher_order_normal_radial, utilities_2d.c:31-48 + normal_2d :18-29). */
void or_higher_order_normal_radial(double alpha, const double v[4][3], double normal[2]) {
    const double *n0 = v[0], *n1 = v[2], *n2 = v[3], *n3 = v[1];
    double a2 = alpha * alpha, t[2];
    for (int d_ = 0; d_ < 2; d_++) {
        int col = d_ == 0 ? 0 : 2;
        double x0 = n0[col], x1 = n1[col], x2 = n2[col], x3 = n3[col];
        t[d_] = (2 * alpha * (9 * x3 - 9 * x2 - 9 * x1 + 9 * x0) +
                 3 * a2 * (9 * x3 - 27 * x2 + 27 * x1 - 9 * x0) - x3 + 27 * x2 - 27 * x1 + x0) / 16;
    }
    double nx = t[1], ny = -t[0];
    double l = sqrt(nx * nx + ny * ny);
    normal[0] = nx / l;
    normal[1] = ny / l;
}

/* fill_jacobian_buffer_radial, radial.c:224-246: jac[i][k] = w_k * |dx/dalpha|,
 * pos[i][k] = (r, z) at Gauss node k. */
void or_fill_jacobian_buffer_radial(double *jac, double *pos, const double *vertices, size_t N) {
    const double (*v)[4][3] = (const double (*)[4][3])vertices;
    for (size_t i = 0; i < N; i++)
        for (int k = 0; k < OR_NQ; k++) {
            double p[2], j;
            or_element_point(OR_GX[k], v[i], 0, p, &j);
            jac[i * OR_NQ + k] = OR_GW[k] * j;
            pos[(i * OR_NQ + k) * 2 + 0] = p[0];
            pos[(i * OR_NQ + k) * 2 + 1] = p[1];
        }
}

/* charge_radial, radial.c:123-148: sum_k 2 pi r_k w_k jac_k * charge */
double or_charge_radial(const double *vertices, double charge) {
    const double (*v)[3] = (const double (*)[3])vertices;
    double s = 0;
    for (int k = 0; k < OR_NQ; k++) {
        double p[2], j;
        or_element_point(OR_GX[k], v, 0, p, &j);
        s += 2 * OR_PI * p[0] * OR_GW[k] * j * charge;
    }
    return s;
}

/* ------------------------------------------------------- ring kernels */

/* potential_radial_ring, radial_ring.c:37-43.  Potential at (r0, z0) of a
 * unit ring charge at (r0 + dr, z0 + dz), in units where charge = sigma/eps0. */
double or_potential_radial_ring(double r0, double z0, double dr, double dz) {
    (void)z0;
    double rho2 = dz * dz + dr * dr;
    double s = dr + 2 * r0;
    double D = dz * dz + s * s;
    double t = rho2 / D;
    return (1. / OR_PI) * or_ellipkm1(t) * (dr + r0) / sqrt(D);
}

/* dr1_potential_radial_ring, radial_ring.c:21-35: d/dr0 of the ring potential */
double or_dr1_potential_radial_ring(double r0, double z0, double dr, double dz) {
    (void)z0;
    if (r0 < OR_MIN_AXIS) return 0.0;
    double r = r0 + dr;
    double rho2 = dz * dz + dr * dr;
    double D = 4 * r * r - 4 * dr * r + rho2;
    double t = rho2 / D;
    double den = (-2 * dr * dr * r + dz * dz * (2 * dr - 2 * r) + 2 * dr * dr * dr) * sqrt(D);
    double kt = rho2 * r * or_ellipkm1(t);
    double et = (-2 * dr * r * r - dz * dz * r + dr * dr * r) * or_ellipem1(t);
    return (1. / OR_PI) * (kt + et) / den;
}

/* dz1_potential_radial_ring, radial_ring.c:45-53: d/dz0 of the ring potential */
double or_dz1_potential_radial_ring(double r0, double z0, double dr, double dz) {
    (void)z0;
    double rho2 = dz * dz + dr * dr;
    double D = 4 * r0 * r0 + 4 * dr * r0 + rho2;
    double t = rho2 / D;
    double den = rho2 * sqrt(D);
    double et = -dz * (r0 + dr) * or_ellipem1(t);
    return (1. / OR_PI) * -et / den;
}

/* flux_density_to_charge_factor, utilities_2d.c:91-105 */
double or_flux_density_to_charge_factor(double K) { return 2.0 * (K - 1) / (1 + K); }

/* field_dot_normal_radial, radial_ring.c:55-71 */
static double or_field_dot_normal(double r0, double z0, double dr, double dz, const double n[2], double K) {
    double Er = -or_dr1_potential_radial_ring(r0, z0, dr, dz);
    double Ez = -or_dz1_potential_radial_ring(r0, z0, dr, dz);
    return or_flux_density_to_charge_factor(K) * (n[0] * Er + n[1] * Ez);
}

/* ------------------------------------------------------- matrix fill */

/* fill_matrix_radial, radial.c:249-310.  Rows [start, end] inclusive; the
 * matrix must be zeroed by the caller (entries are accumulated).  Returns -1
 * for an unknown excitation type instead of exit(1). */
int or_fill_matrix_radial(double *matrix, const double *vertices, const uint8_t *types,
                          const double *values, const double *jac, const double *pos,
                          size_t N, size_t N_matrix, int start, int end) {
    const double (*v)[4][3] = (const double (*)[4][3])vertices;
    for (int i = start; i <= end; i++) {
        double tgt[2], tj;
        or_element_point(0.0, v[i], 0, tgt, &tj);
        int ty = types[i];
        if (ty == 1 || ty == 2 || ty == 5) {
            for (size_t j = 0; j < N; j++)
                for (int k = 0; k < OR_NQ; k++) {
                    const double *p = &pos[(j * OR_NQ + k) * 2];
                    matrix[i * N_matrix + j] += jac[j * OR_NQ + k] *
                        or_potential_radial_ring(tgt[0], tgt[1], p[0] - tgt[0], p[1] - tgt[1]);
                }
        } else if (ty == 3 || ty == 6) {
            double n[2];
            or_higher_order_normal_radial(0.0, v[i], n);
            for (size_t j = 0; j < N; j++)
                for (int k = 0; k < OR_NQ; k++) {
                    const double *p = &pos[(j * OR_NQ + k) * 2];
                    matrix[i * N_matrix + j] += jac[j * OR_NQ + k] *
                        or_field_dot_normal(tgt[0], tgt[1], p[0] - tgt[0], p[1] - tgt[1], n, values[i]);
                }
        } else {
            return -1;
        }
    }
    return 0;
}

/* Integrand of the singular self term of a voltage row, self_potential_radial,
 * radial.c:182-196.  `user` points at the (4,3) vertices of the element.
 * Signature is scipy.LowLevelCallable-compatible: double f(double, void*). */
double or_self_potential_radial(double alpha, void *user) {
    const double (*v)[3] = (const double (*)[3])user;
    double d[2], j, tgt[2], j0;
    or_element_point(alpha, v, 1, d, &j);
    or_element_point(0.0, v, 0, tgt, &j0);
    return j * or_potential_radial_ring(tgt[0], tgt[1], d[0], d[1]);
}

/* Arguments of or_self_field_dot_normal_radial: mirrors
 * struct self_field_dot_normal_radial_args, radial.c:198-201. */
struct or_self_flux_args {
    const double *line_points; /* (4,3) */
    double K;
};

/* self_field_dot_normal_radial, radial.c:203-222 */
double or_self_field_dot_normal_radial(double alpha, void *user) {
    const struct or_self_flux_args *a = (const struct or_self_flux_args *)user;
    const double (*v)[3] = (const double (*)[3])a->line_points;
    double d[2], j, tgt[2], j0, n[2];
    or_element_point(alpha, v, 1, d, &j);
    or_element_point(0.0, v, 0, tgt, &j0);
    or_higher_order_normal_radial(0.0, v, n);
    return j * or_field_dot_normal(tgt[0], tgt[1], d[0], d[1], n, a->K);
}

/* ------------------------------------------------------- field sums */

/* potential_radial, radial.c:105-121 */
double or_potential_radial(const double point[3], const double *q, const double *jac,
                           const double *pos, size_t N) {
    double s = 0, r0 = sqrt(point[0] * point[0] + point[1] * point[1]), z0 = point[2];
    for (size_t i = 0; i < N; i++)
        for (int k = 0; k < OR_NQ; k++) {
            const double *p = &pos[(i * OR_NQ + k) * 2];
            s += q[i] * jac[i * OR_NQ + k] * or_potential_radial_ring(r0, z0, p[0] - r0, p[1] - z0);
        }
    return s;
}

/* field_radial, radial.c:150-173 */
void or_field_radial(const double point[3], double out[3], const double *q, const double *jac,
                     const double *pos, size_t N) {
    double Er = 0, Ez = 0, r = sqrt(point[0] * point[0] + point[1] * point[1]);
    for (size_t i = 0; i < N; i++)
        for (int k = 0; k < OR_NQ; k++) {
            const double *p = &pos[(i * OR_NQ + k) * 2];
            double w = q[i] * jac[i * OR_NQ + k];
            Er -= w * or_dr1_potential_radial_ring(r, point[2], p[0] - r, p[1] - point[2]);
            Ez -= w * or_dz1_potential_radial_ring(r, point[2], p[0] - r, p[1] - point[2]);
        }
    if (r >= OR_MIN_AXIS) {
        out[0] = point[0] / r * Er;
        out[1] = point[1] / r * Er;
    } else {
        out[0] = 0.;
        out[1] = 0.;
    }
    out[2] = Ez;
}

/* axial_derivatives_radial_ring, radial_ring.c:109-122: derivatives
 * d^n/dz0^n of r/(2 R), R = |(z0 - z, r)|, by the three-term recurrence. */
static void or_axial_ring(double z0, double r, double z, double D[OR_NDERIV]) {
    double dz = z0 - z, R2 = dz * dz + r * r, R = sqrt(R2);
    D[0] = 1 / R;
    D[1] = -dz / (R2 * R);
    for (int n = 1; n + 1 < OR_NDERIV; n++)
        D[n + 1] = -1. / R2 * ((2 * n + 1) * dz * D[n] + (double)(n * n) * D[n - 1]);
    for (int n = 0; n < OR_NDERIV; n++) D[n] *= r / 2;
}

/* axial_derivatives_radial, radial.c:18-36 (accumulates into derivs) */
void or_axial_derivatives_radial(double *derivs, const double *q, const double *jac, const double *pos,
                                 size_t N, const double *z, size_t Nz) {
    for (size_t i = 0; i < Nz; i++)
        for (size_t j = 0; j < N; j++)
            for (int k = 0; k < OR_NQ; k++) {
                double D[OR_NDERIV];
                or_axial_ring(z[i], pos[(j * OR_NQ + k) * 2], pos[(j * OR_NQ + k) * 2 + 1], D);
                double w = jac[j * OR_NQ + k] * q[j];
                for (int l = 0; l < OR_NDERIV; l++) derivs[i * OR_NDERIV + l] += w * D[l];
            }
}

/* current_field_radial_ring, radial_ring.c:78-107: (H_r, H_z) at (x0, y0) of a
 * unit current loop of radius x at height y. */
void or_current_field_radial_ring(double x0, double y0, double x, double y, double res[2]) {
    double a = x, r = x0, z = y0 - y;
    double A = z * z + (a + r) * (a + r);
    double B = z * z + (r - a) * (r - a);
    double k = 4 * r * a / A;
    if (x < OR_MIN_AXIS) {
        res[0] = 0.;
        res[1] = 0.;
        return;
    }
    if (x0 < OR_MIN_AXIS)
        res[0] = 0.;
    else
        res[0] = 1. / OR_PI * z / (2 * r * sqrt(A)) * ((z * z + r * r + a * a) / B * or_ellipe(k) - or_ellipk(k));
    res[1] = 1. / OR_PI * 1 / (2 * sqrt(A)) * ((a * a - z * z - r * r) / B * or_ellipe(k) + or_ellipk(k));
}

/* current_field_radial, radial.c:55-83; positions are (N, 12, 3) with y == 0 */
void or_current_field_radial(const double point[3], double out[3], const double *I, const double *jac,
                             const double *pos, size_t N) {
    double Br = 0, Bz = 0, r = sqrt(point[0] * point[0] + point[1] * point[1]);
    for (size_t i = 0; i < N; i++)
        for (int k = 0; k < OR_NTRI; k++) {
            const double *p = &pos[(i * OR_NTRI + k) * 3];
            double f[2];
            or_current_field_radial_ring(r, point[2], p[0], p[2], f);
            Br += I[i] * jac[i * OR_NTRI + k] * f[0];
            Bz += I[i] * jac[i * OR_NTRI + k] * f[1];
        }
    if (r >= OR_MIN_AXIS) {
        out[0] = point[0] / r * Br;
        out[1] = point[1] / r * Br;
    } else {
        out[0] = 0.;
        out[1] = 0.;
    }
    out[2] = Bz;
}

/* current_axial_derivatives_radial_ring, radial_ring.c:124-136 */
static void or_current_axial_ring(double z0, double r, double z, double D[OR_NDERIV]) {
    double dz = z0 - z, R = sqrt(dz * dz + r * r), mu = dz / R;
    D[0] = -dz / (2 * sqrt(dz * dz + r * r));
    D[1] = -r * r / (2 * pow(dz * dz + r * r, 1.5));
    for (int n = 2; n < OR_NDERIV; n++)
        D[n] = -(2 * n - 1) * mu / R * D[n - 1] - (double)(n * n - 2 * n) / (R * R) * D[n - 2];
}

/* current_axial_derivatives_radial, radial.c:85-103 (accumulates) */
void or_current_axial_derivatives_radial(double *derivs, const double *I, const double *jac,
                                         const double *pos, size_t N, const double *z, size_t Nz) {
    for (size_t i = 0; i < Nz; i++)
        for (size_t j = 0; j < N; j++)
            for (int k = 0; k < OR_NTRI; k++) {
                double D[OR_NDERIV];
                const double *p = &pos[(j * OR_NTRI + k) * 3];
                or_current_axial_ring(z[i], p[0], p[2], D);
                for (int l = 0; l < OR_NDERIV; l++) derivs[i * OR_NDERIV + l] += jac[j * OR_NTRI + k] * I[j] * D[l];
            }
}

/* ------------------------------------------------------- axial series */

/* Locate the interval and evaluate the 9 derivative polynomials; shared part
 * of potential_radial_derivs / field_radial_derivs, radial.c:312-384.
 * Returns 0 when z is outside [z_first, z_last]. */
static int or_axial_eval(double z, const double *zi, const double *coeff, size_t Nz, double d[OR_NDERIV]) {
    double z0 = zi[0], zl = zi[Nz - 1];
    if (!(z0 <= z && z <= zl)) return 0;
    double dz = zi[1] - zi[0];
    int idx = (int)((z - z0) / dz);
    if (idx < 0) idx = 0;
    if (idx > (int)Nz - 2) idx = (int)Nz - 2;
    double x = z - zi[idx];
    const double *C = &coeff[(size_t)idx * OR_NDERIV * 6];
    for (int i = 0; i < OR_NDERIV; i++) {
        const double *c = &C[i * 6];
        d[i] = ((((c[0] * x + c[1]) * x + c[2]) * x + c[3]) * x + c[4]) * x + c[5];
    }
    return 1;
}

/* potential_radial_derivs, radial.c:312-344 */
double or_potential_radial_derivs(const double point[3], const double *zi, const double *coeff, size_t Nz) {
    double d[OR_NDERIV];
    if (!or_axial_eval(point[2], zi, coeff, Nz, d)) return 0.0;
    double r2 = point[0] * point[0] + point[1] * point[1];
    return d[0] - r2 / 4 * d[2] + r2 * r2 / 64. * d[4] - r2 * r2 * r2 / 2304. * d[6] +
           r2 * r2 * r2 * r2 / 147456. * d[8];
}

/* field_radial_derivs, radial.c:347-384 */
void or_field_radial_derivs(const double point[3], double f[3], const double *zi, const double *coeff, size_t Nz) {
    double d[OR_NDERIV];
    if (!or_axial_eval(point[2], zi, coeff, Nz, d)) {
        f[0] = f[1] = f[2] = 0.0;
        return;
    }
    double r2 = point[0] * point[0] + point[1] * point[1];
    double fr = 0.5 * (d[2] - r2 / 8 * d[4] + r2 * r2 / 192 * d[6] - r2 * r2 * r2 / 9216 * d[8]);
    double fz = -d[1] + r2 / 4 * d[3] - r2 * r2 / 64 * d[5] + r2 * r2 * r2 / 2304 * d[7];
    f[0] = point[0] * fr;
    f[1] = point[1] * fr;
    f[2] = fz;
}

/* ------------------------------------------------------- tracing */

/* Field providers for the tracer.  Mirrors struct field_evaluation_args
 * (radial.c:175-180) with the charge sets flattened, and struct
 * field_derivs_args (three_d.c:26-31). */
struct or_bem_args {
    const double *eq, *ejac, *epos; size_t eN;   /* electrostatic charges, (N,16), (N,16,2) */
    const double *mq, *mjac, *mpos; size_t mN;   /* magnetostatic charges */
    const double *cI, *cjac, *cpos; size_t cN;   /* current rings, (N,12), (N,12,3) */
    const double *bounds;                        /* (3,2) or NULL */
};
struct or_axial_args {
    const double *z, *ecoeff, *mcoeff; size_t Nz;
};

/* field_radial_traceable, tracing.c:125-165 (strict bounds test) */
static void or_field_bem(const double *p, const double *v, const void *args_, double e[3], double m[3]) {
    (void)v;
    const struct or_bem_args *a = (const struct or_bem_args *)args_;
    const double *b = a->bounds;
    if (b == NULL || (b[0] < p[0] && p[0] < b[1] && b[2] < p[1] && p[1] < b[3] && b[4] < p[2] && p[2] < b[5])) {
        or_field_radial(p, e, a->eq, a->ejac, a->epos, a->eN);
        or_field_radial(p, m, a->mq, a->mjac, a->mpos, a->mN);
        double c[3] = {0, 0, 0};
        or_current_field_radial(p, c, a->cI, a->cjac, a->cpos, a->cN);
        m[0] += c[0];
        m[1] += c[1];
        m[2] += c[2];
    } else {
        e[0] = e[1] = e[2] = 0;
        m[0] = m[1] = m[2] = 0;
    }
}

/* field_radial_derivs_traceable, tracing.c:168-174 */
static void or_field_axial(const double *p, const double *v, const void *args_, double e[3], double m[3]) {
    (void)v;
    const struct or_axial_args *a = (const struct or_axial_args *)args_;
    or_field_radial_derivs(p, e, a->z, a->ecoeff, a->Nz);
    or_field_radial_derivs(p, m, a->z, a->mcoeff, a->Nz);
}

typedef void (*or_field_fn)(const double *, const double *, const void *, double *, double *);

/* Runge-Kutta-Fehlberg 4(5) tableau, tracing.c:9-16 */
static const double RK_B[6][5] = {
    {0, 0, 0, 0, 0},
    {2. / 9., 0, 0, 0, 0},
    {1. / 12., 1. / 4., 0, 0, 0},
    {69. / 128., -243. / 128., 135. / 64., 0, 0},
    {-17. / 12., 27. / 4., -27. / 5., 16. / 15., 0},
    {65. / 432., -5. / 16., 13. / 16., 4. / 27., 5. / 144.}};
static const double RK_CH[6] = {47. / 450., 0., 12. / 25., 32. / 225., 1. / 30., 6. / 25.};
static const double RK_CT[6] = {-1. / 150., 0., 3. / 100., -16. / 75., -1. / 20., 6. / 25.};

/* trace_particle, tracing.c:60-123 (with produce_new_y :20-32 and
 * produce_new_k :34-57).  Row 0 of pos6/times holds the start state.  Stops
 * when the position leaves the inclusive bounds, when max_rows rows are
 * filled, or after max_attempts step attempts (a cap the reference lacks;
 * pass 0 for no cap).  Returns the number of rows written. */
static size_t or_trace(double *times, double *pos6, double qm, or_field_fn ff, const void *args,
                       const double *bounds, double atol, size_t max_rows, long long max_attempts) {
    double y[6];
    for (int i = 0; i < 6; i++) y[i] = pos6[i];
    double V = sqrt(y[3] * y[3] + y[4] * y[4] + y[5] * y[5]);
    double hmax = OR_STEP_MAX / V, h = hmax;
    size_t N = 1;
    long long attempts = 0;
    const double *b = bounds;
    while (b[0] <= y[0] && y[0] <= b[1] && b[2] <= y[1] && y[1] <= b[3] && b[4] <= y[2] && y[2] <= b[5]) {
        if (max_attempts > 0 && attempts >= max_attempts) break;
        attempts++;
        double k[6][6], ys[6];
        for (int s = 0; s < 6; s++) {
            for (int i = 0; i < 6; i++) {
                ys[i] = y[i];
                for (int j = 0; j < s; j++) ys[i] += RK_B[s][j] * k[j][i];
            }
            double e[3] = {0, 0, 0}, m[3] = {0, 0, 0};
            ff(ys, ys + 3, args, e, m);
            /* v x H, cross_product_3d */
            double cx = ys[4] * m[2] - ys[5] * m[1];
            double cy = ys[5] * m[0] - ys[3] * m[2];
            double cz = ys[3] * m[1] - ys[4] * m[0];
            k[s][0] = h * ys[3];
            k[s][1] = h * ys[4];
            k[s][2] = h * ys[5];
            k[s][3] = h * qm * (e[0] + OR_MU0 * cx);
            k[s][4] = h * qm * (e[1] + OR_MU0 * cy);
            k[s][5] = h * qm * (e[2] + OR_MU0 * cz);
        }
        double ep = 0, ev = 0;
        for (int i = 0; i < 3; i++) {
            double a = 0, c = 0;
            for (int j = 0; j < 6; j++) {
                a += RK_CT[j] * k[j][i];
                c += RK_CT[j] * k[j][i + 3];
            }
            if (fabs(a) > ep) ep = fabs(a);
            if (fabs(c) > ev) ev = fabs(c);
        }
        double err = ep + h * ev;
        if (err <= atol) {
            for (int i = 0; i < 6; i++) {
                y[i] += RK_CH[0] * k[0][i] + RK_CH[1] * k[1][i] + RK_CH[2] * k[2][i] + RK_CH[3] * k[3][i] +
                        RK_CH[4] * k[4][i] + RK_CH[5] * k[5][i];
                pos6[N * 6 + i] = y[i];
            }
            times[N] = times[N - 1] + h;
            N += 1;
            if (N == max_rows) return N;
        }
        h = fmin(0.9 * h * pow(atol / err, 0.2), hmax);
    }
    return N;
}

size_t or_trace_particle_bem(double *times, double *pos6, double qm, const struct or_bem_args *args,
                             const double *bounds, double atol, size_t max_rows, long long max_attempts) {
    return or_trace(times, pos6, qm, or_field_bem, args, bounds, atol, max_rows, max_attempts);
}

size_t or_trace_particle_axial(double *times, double *pos6, double qm, const struct or_axial_args *args,
                               const double *bounds, double atol, size_t max_rows, long long max_attempts) {
    return or_trace(times, pos6, qm, or_field_axial, args, bounds, atol, max_rows, max_attempts);
}

/* Field evaluation entry points used by the Python side of the oracle for
 * whole point batches (loops over or_field_radial / or_potential_radial). */
void or_field_radial_batch(const double *points, double *out, size_t M, const double *q, const double *jac,
                           const double *pos, size_t N) {
    for (size_t m = 0; m < M; m++) or_field_radial(points + 3 * m, out + 3 * m, q, jac, pos, N);
}
void or_potential_radial_batch(const double *points, double *out, size_t M, const double *q, const double *jac,
                               const double *pos, size_t N) {
    for (size_t m = 0; m < M; m++) out[m] = or_potential_radial(points + 3 * m, q, jac, pos, N);
}

/* plane_intersection, tracing.c:184-223: linear interpolation of the last
 * crossing of the plane through p0 with the given normal, searched from the
 * end of the trajectory.  Returns 1 when found. */
int or_plane_intersection(const double p0[3], const double n[3], const double *pos6, size_t Np, double res[6]) {
    if (Np < 2) return 0;
    double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
#define KAPPA(row) ((n[2] * p0[2] - pos6[(row) * 6 + 2] * n[2] + n[1] * p0[1] - pos6[(row) * 6 + 1] * n[1] + \
                     n[0] * p0[0] - pos6[(row) * 6 + 0] * n[0]) / nn)
    long i = (long)Np - 1;
    double prev = KAPPA(i);
    for (i = i - 1; i >= 0; i--) {
        double kap = KAPPA(i);
        int s = kap > 0 ? 1 : -1, sp = prev > 0 ? 1 : -1;
        if (s != sp) {
            double diff = kap - prev, f = -prev / diff, pf = kap / diff;
            for (int c = 0; c < 6; c++) res[c] = pf * pos6[(i + 1) * 6 + c] + f * pos6[i * 6 + c];
            return 1;
        }
        prev = kap;
    }
#undef KAPPA
    return 0;
}
