// tb_bem.cu -- BEM assembly and field-sum kernels of the radial path.
//
//   jacobian buffer      radial.c:224-246
//   matrix fill          radial.c:249-310 (off-diagonal 16-point Gauss sums)
//   self integrals       radial.c:182-222 + traceon/backend/__init__.py:688-708
//   potential / field    radial.c:105-173, batched over points
//   axial derivatives    radial.c:18-36
//   axial coefficients   traceon/field.py:914-937
//   axial evaluation     radial.c:312-384, batched over points
//
// Everything is FP64; the kernels are FP64-pipe bound (one log, one sqrt and
// one division per ring pair).
#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "tb_fill.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

// ---------------------------------------------------------------- graded meshes
// Cubic line elements along straight segments, graded toward both ends of
// every segment: segment s from (r0, z0) to (r1, z1) carries off[s + 1] -
// off[s] elements whose nodes are the Chebyshev-Lobatto points
// t_k = (1 - cos(pi k / n)) / 2 (t_0 = 0, t_n = 1) -- the host mesher's rule
// (geometry.graded_nodes), with its operations in the same order and without
// fused multiply-adds.  Rows in the reference's line4 layout [start, end,
// 1/3-point, 2/3-point] of (r, 0, z) (traceon/mesher.py:188-227), every
// coordinate with its low 16 mantissa bits cleared: the truncation the
// reference's Mesh merges points with (traceon/mesher.py:262-290).  One
// thread per element; its segment by binary search of the offsets.
__device__ __forceinline__ double snap16(double x) {
  return __longlong_as_double(__double_as_longlong(x) & (long long)0xFFFFFFFFFFFF0000ULL);
}

__device__ __forceinline__ double cheb_node(int64_t k, int64_t n) {
  if (k <= 0) return 0.0;
  if (k >= n) return 1.0;
  return __dmul_rn(0.5, __dsub_rn(1.0, cos(__ddiv_rn(__dmul_rn(PI, double(k)), double(n)))));
}

__global__ void k_mesh_segments(const double* __restrict__ seg, const int64_t* __restrict__ off, int64_t S,
                                double* __restrict__ out, int64_t N) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  int64_t lo = 0, hi = S - 1;  // the last segment with off[s] <= i
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) / 2;
    if (off[mid] <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  const int64_t n = off[lo + 1] - off[lo], k = i - off[lo];
  const double a = cheb_node(k, n), b = cheb_node(k + 1, n);
  const double d = __dsub_rn(b, a);
  const double t[4] = {a, b, __dadd_rn(a, __ddiv_rn(d, 3.0)), __dadd_rn(a, __ddiv_rn(__dmul_rn(2.0, d), 3.0))};
  const double r0 = seg[4 * lo], z0 = seg[4 * lo + 1], dr = __dsub_rn(seg[4 * lo + 2], r0),
               dz = __dsub_rn(seg[4 * lo + 3], z0);
  double* row = out + i * 12;
  for (int q = 0; q < 4; q++) {
    row[3 * q] = snap16(__dadd_rn(r0, __dmul_rn(dr, t[q])));
    row[3 * q + 1] = 0.0;
    row[3 * q + 2] = snap16(__dadd_rn(z0, __dmul_rn(dz, t[q])));
  }
}

// ---------------------------------------------------------------- jacobian
__global__ void k_jacobian_buffer(const double* __restrict__ vertices, double* __restrict__ jac,
                                  double* __restrict__ pos, int64_t N) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= N * NQ) return;
  int64_t i = g / NQ;
  int k = int(g % NQ);
  Cubic c;
  c.load(vertices + i * 12);
  double r, z, j;
  c.point(gauss_x(k), false, r, z, j);
  jac[g] = gauss_w(k) * j;
  pos[2 * g] = r;
  pos[2 * g + 1] = z;
}

__global__ void k_element_targets(const double* __restrict__ vertices, double* __restrict__ target,
                                  double* __restrict__ normal, int64_t N) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  Cubic c;
  c.load(vertices + i * 12);
  double r, z, j, nr, nz;
  c.point(0.0, false, r, z, j);
  c.normal(0.0, nr, nz);
  if (target) {
    target[2 * i] = r;
    target[2 * i + 1] = z;
  }
  if (normal) {
    normal[2 * i] = nr;
    normal[2 * i + 1] = nz;
  }
}

// ---------------------------------------------------------------- fill
// Block = 32 columns x 8 rows; the 32 columns' Gauss rings are staged in
// shared memory once and reused by the 8 rows.
constexpr int FILL_COLS = 32;
constexpr int FILL_ROWS = 8;

__global__ void __launch_bounds__(FILL_COLS* FILL_ROWS)
    k_fill_matrix(double* __restrict__ A, int64_t lda, const double* __restrict__ vertices,
                  const uint8_t* __restrict__ types, const double* __restrict__ values,
                  const double* __restrict__ jac, const double* __restrict__ pos, int64_t N, int64_t row0,
                  int64_t row1, int accumulate, int gauss_diagonal) {
  __shared__ double s_r[FILL_COLS][NQ + 1], s_z[FILL_COLS][NQ + 1], s_w[FILL_COLS][NQ + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t j0 = blockIdx.x * (int64_t)FILL_COLS;
  const int tid = ty * FILL_COLS + tx;
  for (int e = tid; e < FILL_COLS * NQ; e += FILL_COLS * FILL_ROWS) {
    int c = e / NQ, k = e % NQ;
    int64_t j = j0 + c;
    double r = 0, z = 0, w = 0;
    if (j < N) {
      r = pos[(j * NQ + k) * 2];
      z = pos[(j * NQ + k) * 2 + 1];
      w = jac[j * NQ + k];
    }
    s_r[c][k] = r;
    s_z[c][k] = z;
    s_w[c][k] = w;
  }
  __syncthreads();
  const int64_t i = row0 + blockIdx.y * (int64_t)FILL_ROWS + ty;
  const int64_t j = j0 + tx;
  if (i >= row1 || j >= N) return;
  if (j == i && !gauss_diagonal) return;
  const double acc = fill_entry(vertices, types, values, i, s_r[tx], s_z[tx], s_w[tx]);
  double* a = A + (i * lda + j);
  *a = accumulate ? *a + acc : acc;
}

// ---------------------------------------------------------------- batched fill
// Many geometries of uneven N in one persistent launch: the tiles (32 columns
// x 8 rows) of all matrices are numbered globally (geometry g owns tiles
// [tile0[g], tile0[g] + tiles_x[g] tiles_y[g])); CTAs stride over them and
// find their geometry by binary search.  Diagonal entries are left to the
// self integrals, as in the single-geometry fill.
__global__ void __launch_bounds__(FILL_COLS* FILL_ROWS)
    k_fill_matrix_batched(const tb_geometry_t* __restrict__ geoms, int n_geoms, int64_t total_tiles) {
  __shared__ double s_r[FILL_COLS][NQ + 1], s_z[FILL_COLS][NQ + 1], s_w[FILL_COLS][NQ + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * FILL_COLS + tx;
  for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    int lo = 0, hi = n_geoms - 1;  // last geometry with tile0 <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (geoms[mid].tile0 <= t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const tb_geometry_t& g = geoms[lo];
    const int64_t N = g.N;
    const int64_t tiles_x = (N + FILL_COLS - 1) / FILL_COLS;
    const int64_t local = t - g.tile0;
    const int64_t j0 = (local % tiles_x) * FILL_COLS, i0 = (local / tiles_x) * FILL_ROWS;
    __syncthreads();  // the previous tile's rings are no longer read
    for (int e = tid; e < FILL_COLS * NQ; e += FILL_COLS * FILL_ROWS) {
      const int c = e / NQ, k = e % NQ;
      const int64_t j = j0 + c;
      double r = 0, z = 0, w = 0;
      if (j < N) {
        r = g.pos[(j * NQ + k) * 2];
        z = g.pos[(j * NQ + k) * 2 + 1];
        w = g.jac[j * NQ + k];
      }
      s_r[c][k] = r;
      s_z[c][k] = z;
      s_w[c][k] = w;
    }
    __syncthreads();
    const int64_t i = i0 + ty, j = j0 + tx;
    if (i < N && j < N && i != j) g.A[i * g.lda + j] = fill_entry(g.vertices, g.types, g.values, i, s_r[tx], s_z[tx], s_w[tx]);
  }
}

// The self terms (one warp per element).
__global__ void k_self_integrals(const double* __restrict__ vertices, const uint8_t* __restrict__ types,
                                 const double* __restrict__ values, double* __restrict__ diag,
                                 double* __restrict__ A, int64_t lda, int64_t N) {
  int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
  int lane = threadIdx.x & 31;
  if (i >= N) return;
  const double v = self_term_warp(vertices, types, values, i, lane);
  if (lane == 0) {
    if (diag) diag[i] = v;
    if (A) A[i * lda + i] = v;
  }
}

// The self terms of all elements of many geometries (one warp per element,
// grid-strided over the global element numbering), onto their matrices'
// diagonals.
__global__ void k_self_integrals_batched(const tb_geometry_t* __restrict__ geoms, int n_geoms, int64_t total) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
  for (int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; e < total; e += warps) {
    int lo = 0, hi = n_geoms - 1;  // last geometry with elem0 <= e
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (geoms[mid].elem0 <= e)
        lo = mid;
      else
        hi = mid - 1;
    }
    const tb_geometry_t& g = geoms[lo];
    const int64_t i = e - g.elem0;
    const double v = self_term_warp(g.vertices, g.types, g.values, i, lane);
    if (lane == 0) g.A[i * g.lda + i] = v;
  }
}

__global__ void k_rhs(const uint8_t* __restrict__ types, const double* __restrict__ values,
                      double* __restrict__ F, int64_t N) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  int t = types[i];
  F[i] = (t == VOLTAGE_FIXED || t == VOLTAGE_FUN || t == MAGNETOSTATIC_POT) ? values[i] : 0.0;
}

// The full right-hand side of solver.py:118-150: voltage rows take their
// value, dielectric rows 0, magnetizable rows -factor(mu) H . n with H the
// pre-existing field at the element's collocation point (field (N, 3) =
// H_x, H_y, H_z at (r, 0, z), or none: zero field) and n its normal.
__global__ void k_rhs_field(const uint8_t* __restrict__ types, const double* __restrict__ values,
                            const double* __restrict__ normal, const double* __restrict__ field,
                            double* __restrict__ F, int64_t N) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int t = types[i];
  double f = 0.0;
  if (t == VOLTAGE_FIXED || t == VOLTAGE_FUN || t == MAGNETOSTATIC_POT) {
    f = values[i];
  } else if (t == MAGNETIZABLE && field) {
    const double hn = field[3 * i] * normal[2 * i] + field[3 * i + 2] * normal[2 * i + 1];
    f = -flux_factor(values[i]) * hn;
  }
  F[i] = f;
}

// ---------------------------------------------------------------- sources
__global__ void k_pack_sources(const double* __restrict__ q, const double* __restrict__ jac,
                               const double* __restrict__ pos, double* __restrict__ src, int64_t N) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t Nq = N * NQ;
  if (g >= Nq) return;
  src[g] = pos[2 * g];
  src[Nq + g] = pos[2 * g + 1];
  src[2 * Nq + g] = q[g / NQ] * jac[g];
}

// ---------------------------------------------------------------- field
// Potential and field at a point from a slice of sources; returns the raw
// sums (see ring_field_acc).
template <bool POT>
__device__ __forceinline__ void source_sums(double r0, double z0, const double* __restrict__ src, int64_t Nq,
                                            int64_t first, int64_t stride, double& Sr, double& Sz, double& Sp) {
  const double* sr = src;
  const double* sz = src + Nq;
  const double* sw = src + 2 * Nq;
  for (int64_t j = first; j < Nq; j += stride) ring_field_acc<POT>(r0, z0, sr[j], sz[j], sw[j], Sr, Sz, Sp);
}

__device__ __forceinline__ void finish_field(const double* p, double Sr, double Sz, double Sp, double* pot,
                                             double* field, int64_t m) {
  double r = sqrt(p[0] * p[0] + p[1] * p[1]);
  if (pot) pot[m] = Sp * INV_PI;
  if (field) {
    double Er = r >= MIN_AXIS ? Sr / (2 * PI * r) : 0.0;
    if (r >= MIN_AXIS) {
      field[3 * m] = p[0] / r * Er;
      field[3 * m + 1] = p[1] / r * Er;
    } else {
      field[3 * m] = 0.0;
      field[3 * m + 1] = 0.0;
    }
    field[3 * m + 2] = -Sz * INV_PI;
  }
}

// One thread per point; source tiles staged through shared memory.
constexpr int FP_THREADS = 256;
template <bool POT>
__global__ void __launch_bounds__(FP_THREADS)
    k_field_points_thread(const double* __restrict__ points, int64_t M, const double* __restrict__ src,
                          int64_t Nq, double* __restrict__ pot, double* __restrict__ field) {
  __shared__ double t_r[FP_THREADS], t_z[FP_THREADS], t_w[FP_THREADS];
  int64_t m = blockIdx.x * (int64_t)FP_THREADS + threadIdx.x;
  double p[3] = {0, 0, 0};
  if (m < M) {
    p[0] = points[3 * m];
    p[1] = points[3 * m + 1];
    p[2] = points[3 * m + 2];
  }
  double r0 = sqrt(p[0] * p[0] + p[1] * p[1]), z0 = p[2];
  double Sr = 0, Sz = 0, Sp = 0;
  for (int64_t base = 0; base < Nq; base += FP_THREADS) {
    int64_t j = base + threadIdx.x;
    __syncthreads();
    if (j < Nq) {
      t_r[threadIdx.x] = src[j];
      t_z[threadIdx.x] = src[Nq + j];
      t_w[threadIdx.x] = src[2 * Nq + j];
    } else {
      t_r[threadIdx.x] = 1.0;  // harmless ring of zero weight
      t_z[threadIdx.x] = 0.0;
      t_w[threadIdx.x] = 0.0;
    }
    __syncthreads();
    int cnt = Nq - base < FP_THREADS ? int(Nq - base) : FP_THREADS;
#pragma unroll 2
    for (int k = 0; k < cnt; k++) ring_field_acc<POT>(r0, z0, t_r[k], t_z[k], t_w[k], Sr, Sz, Sp);
  }
  if (m < M) finish_field(p, Sr, Sz, Sp, pot, field, m);
}

// One team of TEAM threads (a warp or the whole block) per point.
template <bool POT, int TEAM>
__global__ void __launch_bounds__(TEAM >= 256 ? TEAM : 256)
    k_field_points_team(const double* __restrict__ points, int64_t M, const double* __restrict__ src, int64_t Nq,
                        double* __restrict__ pot, double* __restrict__ field) {
  constexpr int TEAMS = (TEAM >= 256 ? TEAM : 256) / TEAM;
  int team = threadIdx.x / TEAM, lane = threadIdx.x % TEAM;
  int64_t m = blockIdx.x * (int64_t)TEAMS + team;
  double p[3] = {0, 0, 0};
  if (m < M) {
    p[0] = points[3 * m];
    p[1] = points[3 * m + 1];
    p[2] = points[3 * m + 2];
  }
  double r0 = sqrt(p[0] * p[0] + p[1] * p[1]);
  double Sr = 0, Sz = 0, Sp = 0;
  if (m < M) source_sums<POT>(r0, p[2], src, Nq, lane, TEAM, Sr, Sz, Sp);
  Sr = warp_sum(Sr);
  Sz = warp_sum(Sz);
  if (POT) Sp = warp_sum(Sp);
  if (TEAM > 32) {
    __shared__ double red[3][TEAM / 32 > 0 ? TEAM / 32 : 1];
    int w = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
      red[0][w] = Sr;
      red[1][w] = Sz;
      red[2][w] = Sp;
    }
    __syncthreads();
    Sr = Sz = Sp = 0;
    for (int k = 0; k < TEAM / 32; k++) {
      Sr += red[0][k];
      Sz += red[1][k];
      Sp += red[2][k];
    }
  }
  if (m < M && lane == 0) finish_field(p, Sr, Sz, Sp, pot, field, m);
}

// ---------------------------------------------------------------- axial
// One block of 256 threads per z point; each thread sums a strided slice of
// the sources, then a block reduction of the 9 partial sums.
__global__ void __launch_bounds__(256)
    k_axial_derivs(const double* __restrict__ z, int64_t Nz, const double* __restrict__ src, int64_t Nq,
                   double* __restrict__ derivs) {
  __shared__ double red[NDERIV][8];
  int64_t iz = blockIdx.x;
  if (iz >= Nz) return;
  double z0 = z[iz];
  double acc[NDERIV];
#pragma unroll
  for (int l = 0; l < NDERIV; l++) acc[l] = 0.0;
  const double* sr = src;
  const double* sz = src + Nq;
  const double* sw = src + 2 * Nq;
  for (int64_t j = threadIdx.x; j < Nq; j += 256) axial_ring(z0, sr[j], sz[j], sw[j], acc);
  int w = threadIdx.x / 32;
#pragma unroll
  for (int l = 0; l < NDERIV; l++) {
    double v = warp_sum(acc[l]);
    if ((threadIdx.x & 31) == 0) red[l][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NDERIV) {
    double s = 0;
    for (int k = 0; k < 8; k++) s += red[threadIdx.x][k];
    derivs[iz * NDERIV + threadIdx.x] = s;
  }
}

// Quintic Hermite on [0, h] through (y, y', y'') at both ends, in the power
// basis of (x - z_i), highest degree first: the form
// PPoly.from_bernstein_basis(BPoly.from_derivatives(...)).c produces
// (field.py:906-911).
__global__ void k_axial_quintic(const double* __restrict__ d, int64_t Nz, double h, double* __restrict__ c) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t iv = g / 7;
  int i = int(g % 7);
  if (iv >= Nz - 1) return;
  const double* a = d + iv * NDERIV;
  const double* b = d + (iv + 1) * NDERIV;
  double c0 = a[i], c1 = a[i + 1], c2 = 0.5 * a[i + 2];
  double D0 = b[i] - (c0 + h * (c1 + h * c2));
  double D1 = (b[i + 1] - (c1 + 2 * h * c2)) * h;
  double D2 = (b[i + 2] - 2 * c2) * h * h;
  double A3 = 10 * D0 - 4 * D1 + 0.5 * D2;  // c3 h^3
  double A4 = -15 * D0 + 7 * D1 - D2;       // c4 h^4
  double A5 = 6 * D0 - 3 * D1 + 0.5 * D2;   // c5 h^5
  double ih = 1.0 / h, ih3 = ih * ih * ih;
  double* o = c + (iv * NDERIV + i) * 6;
  o[0] = A5 * ih3 * ih * ih;
  o[1] = A4 * ih3 * ih;
  o[2] = A3 * ih3;
  o[3] = c2;
  o[4] = c1;
  o[5] = c0;
}

// Not-a-knot cubic spline (scipy.interpolate.CubicSpline default) of the
// columns 7 and 8 of d, one block per column.  Unknowns are the node slopes
// s_0 .. s_{n-1}; on an equal grid with m_i = (y_{i+1} - y_i)/h:
//   s_{i-1} + 4 s_i + s_{i+1} = 3 (m_{i-1} + m_i),      0 < i < n-1
//   not-a-knot at x_1:      s_0 - s_2 = 2 (m_0 - m_1)
//   not-a-knot at x_{n-2}:  s_{n-1} - s_{n-3} = 2 (m_{n-2} - m_{n-3})
// Eliminating s_0 and s_{n-1} leaves a tridiagonal system in s_1..s_{n-2}
// with first row 4 s_1 + 2 s_2 = m_0 + 5 m_1 and last row
// 2 s_{n-3} + 4 s_{n-2} = 5 m_{n-3} + m_{n-2}, solved by the Thomas
// algorithm in shared memory.  n = 3 uses the single parabola through the
// three points, n = 2 the straight line (CubicSpline's special cases).
constexpr int SPLINE_MAX_NZ = 12288;

__global__ void k_axial_cubic(const double* __restrict__ d, int64_t Nz, double h, double* __restrict__ c) {
  extern __shared__ double sm[];
  const int col = 7 + blockIdx.x;
  const int64_t n = Nz;
  if (threadIdx.x != 0) return;
  auto y = [&](int64_t i) { return d[i * NDERIV + col]; };
  auto mm = [&](int64_t i) { return (y(i + 1) - y(i)) / h; };
  double* cp = sm;           // modified super-diagonal, index 1..n-2
  double* dp = sm + n;       // modified rhs / solution slopes, index 0..n-1
  if (n == 2) {
    dp[0] = dp[1] = mm(0);
  } else if (n == 3) {
    // parabola through 3 points: slopes at the nodes
    double m0 = mm(0), m1 = mm(1);
    double a = (m1 - m0) / (2 * h);  // quadratic coefficient
    dp[0] = m0 - a * h;
    dp[1] = m0 + a * h;
    dp[2] = m1 + a * h;
  } else {
    const int64_t K = n - 2;  // unknowns s_1..s_{n-2}
    for (int64_t r = 0; r < K; r++) {
      int64_t i = r + 1;
      double b, a_, cc, rhs;
      if (r == 0) {
        b = 4;
        cc = 2;
        a_ = 0;
        rhs = mm(0) + 5 * mm(1);
      } else if (r == K - 1) {
        a_ = 2;
        b = 4;
        cc = 0;
        rhs = 5 * mm(n - 3) + mm(n - 2);
      } else {
        a_ = 1;
        b = 4;
        cc = 1;
        rhs = 3 * (mm(i - 1) + mm(i));
      }
      if (K == 1) {  // n == 3 handled above; keeps the algebra total
        a_ = 0;
        cc = 0;
      }
      double denom = r == 0 ? b : b - a_ * cp[i - 1];
      cp[i] = cc / denom;
      dp[i] = (r == 0 ? rhs : rhs - a_ * dp[i - 1]) / denom;
    }
    for (int64_t i = n - 3; i >= 1; i--) dp[i] -= cp[i] * dp[i + 1];
    dp[0] = dp[2] + 2 * (mm(0) - mm(1));
    dp[n - 1] = dp[n - 3] + 2 * (mm(n - 2) - mm(n - 3));
  }
  for (int64_t iv = 0; iv < n - 1; iv++) {
    double s0 = dp[iv], s1 = dp[iv + 1], m = mm(iv);
    double* o = c + (iv * NDERIV + col) * 6;
    o[0] = 0.0;
    o[1] = 0.0;
    o[2] = (s0 + s1 - 2 * m) / (h * h);
    o[3] = (3 * m - 2 * s0 - s1) / h;
    o[4] = s0;
    o[5] = y(iv);
  }
}

// ---------------------------------------------------------------- currents
__global__ void k_pack_current_sources(const double* __restrict__ I, const double* __restrict__ jac,
                                       const double* __restrict__ pos, double* __restrict__ src, int64_t N) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t Nc = N * NTRI;
  if (g >= Nc) return;
  src[g] = pos[3 * g];
  src[Nc + g] = pos[3 * g + 2];
  src[2 * Nc + g] = I[g / NTRI] * jac[g];
}

// One warp per point: H from current rings (radial.c:55-83).
__global__ void k_current_field_points(const double* __restrict__ points, int64_t M,
                                       const double* __restrict__ src, int64_t Nc, double* __restrict__ field) {
  int64_t m = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
  int lane = threadIdx.x & 31;
  if (m >= M) return;
  double p[3] = {points[3 * m], points[3 * m + 1], points[3 * m + 2]};
  double r = sqrt(p[0] * p[0] + p[1] * p[1]);
  double Br = 0, Bz = 0;
  for (int64_t j = lane; j < Nc; j += 32) {
    double hr, hz;
    current_field_ring(r, p[2], src[j], src[Nc + j], hr, hz);
    Br = fma(src[2 * Nc + j], hr, Br);
    Bz = fma(src[2 * Nc + j], hz, Bz);
  }
  Br = warp_sum(Br);
  Bz = warp_sum(Bz);
  if (lane == 0) {
    if (r >= MIN_AXIS) {
      field[3 * m] = p[0] / r * Br;
      field[3 * m + 1] = p[1] / r * Br;
    } else {
      field[3 * m] = 0.0;
      field[3 * m + 1] = 0.0;
    }
    field[3 * m + 2] = Bz;
  }
}

__global__ void __launch_bounds__(256)
    k_current_axial(const double* __restrict__ z, int64_t Nz, const double* __restrict__ src, int64_t Nc,
                    double* __restrict__ derivs) {
  __shared__ double red[NDERIV][8];
  int64_t iz = blockIdx.x;
  if (iz >= Nz) return;
  double z0 = z[iz];
  double acc[NDERIV];
#pragma unroll
  for (int l = 0; l < NDERIV; l++) acc[l] = 0.0;
  for (int64_t j = threadIdx.x; j < Nc; j += 256) current_axial_ring(z0, src[j], src[Nc + j], src[2 * Nc + j], acc);
  int w = threadIdx.x / 32;
#pragma unroll
  for (int l = 0; l < NDERIV; l++) {
    double v = warp_sum(acc[l]);
    if ((threadIdx.x & 31) == 0) red[l][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NDERIV) {
    double s = 0;
    for (int k = 0; k < 8; k++) s += red[threadIdx.x][k];
    derivs[iz * NDERIV + threadIdx.x] = s;
  }
}

// Axial series evaluation at points (radial.c:312-384).
__global__ void k_axial_points(const double* __restrict__ points, int64_t M, const double* __restrict__ zi,
                               int64_t Nz, const double* __restrict__ coeff, double* __restrict__ pot,
                               double* __restrict__ field) {
  int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= M) return;
  double p[3] = {points[3 * m], points[3 * m + 1], points[3 * m + 2]};
  double dd[NDERIV];
  bool in = axial_eval(p[2], zi, coeff, Nz, dd);
  double r2 = p[0] * p[0] + p[1] * p[1];
  if (pot) pot[m] = in ? axial_potential(dd, r2) : 0.0;
  if (field) {
    double f[3] = {0, 0, 0};
    if (in) axial_field(dd, p, r2, f);
    field[3 * m] = f[0];
    field[3 * m + 1] = f[1];
    field[3 * m + 2] = f[2];
  }
}

}  // namespace tb

// ====================================================================== C ABI
using namespace tb;

extern "C" int tb_mesh_segments(const double* segments, const int64_t* offsets, int64_t S, double* vertices,
                                int64_t N, tb_stream_t stream) {
  if (S < 1 || N < 0 || !segments || !offsets || (N > 0 && !vertices)) return BAD_ARG;
  if (N == 0) return OK;
  k_mesh_segments<<<unsigned((N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(segments, offsets, S, vertices, N);
  return launch_status();
}

extern "C" int tb_jacobian_buffer_radial(const double* vertices, double* jac, double* pos, int64_t N,
                                         tb_stream_t stream) {
  if (N < 0 || (N > 0 && (!vertices || !jac || !pos))) return BAD_ARG;
  if (N == 0) return OK;
  int64_t n = N * NQ;
  k_jacobian_buffer<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(vertices, jac, pos, N);
  return launch_status();
}

extern "C" int tb_element_targets(const double* vertices, double* target, double* normal, int64_t N,
                                  tb_stream_t stream) {
  if (N < 0 || (N > 0 && !vertices)) return BAD_ARG;
  if (N == 0) return OK;
  k_element_targets<<<unsigned((N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(vertices, target, normal, N);
  return launch_status();
}

extern "C" int tb_fill_matrix_radial(double* A, int64_t lda, const double* vertices, const uint8_t* types,
                                     const double* values, const double* jac, const double* pos, int64_t N,
                                     int64_t row0, int64_t row1, int accumulate, int gauss_diagonal,
                                     tb_stream_t stream) {
  if (N < 0 || lda < N || row0 < 0 || row1 > N || row0 > row1) return BAD_ARG;
  if (N == 0 || row0 == row1) return OK;
  if (!A || !vertices || !types || !values || !jac || !pos) return BAD_ARG;
  dim3 grid(unsigned((N + FILL_COLS - 1) / FILL_COLS), unsigned((row1 - row0 + FILL_ROWS - 1) / FILL_ROWS));
  if (grid.y > 65535u) return BAD_ARG;
  k_fill_matrix<<<grid, dim3(FILL_COLS, FILL_ROWS), 0, (cudaStream_t)stream>>>(
      A, lda, vertices, types, values, jac, pos, N, row0, row1, accumulate, gauss_diagonal);
  return launch_status();
}

extern "C" int tb_self_integrals(const double* vertices, const uint8_t* types, const double* values, double* diag,
                                 double* A, int64_t lda, int64_t N, tb_stream_t stream) {
  if (N < 0 || (A && lda < N)) return BAD_ARG;
  if (N == 0) return OK;
  if (!vertices || !types || !values || (!diag && !A)) return BAD_ARG;
  int64_t threads = N * 32;
  k_self_integrals<<<unsigned((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(vertices, types, values, diag,
                                                                                      A, lda, N);
  return launch_status();
}

extern "C" int64_t tb_batch_plan(tb_geometry_t* geoms, int n_geoms, int64_t* total_elements) {
  if (!geoms || n_geoms <= 0) return -1;
  int64_t tiles = 0, elems = 0;
  for (int g = 0; g < n_geoms; g++) {
    const int64_t N = geoms[g].N;
    if (N <= 0 || geoms[g].lda < N) return -1;
    geoms[g].tile0 = tiles;
    geoms[g].elem0 = elems;
    tiles += ((N + FILL_COLS - 1) / FILL_COLS) * ((N + FILL_ROWS - 1) / FILL_ROWS);
    elems += N;
  }
  if (total_elements) *total_elements = elems;
  return tiles;
}

extern "C" int tb_fill_matrix_radial_batched(const tb_geometry_t* geoms, int n_geoms, int64_t total_tiles,
                                             tb_stream_t stream) {
  if (!geoms || n_geoms <= 0 || total_tiles <= 0) return BAD_ARG;
  // persistent: a few CTAs per SM stride over all tiles of all geometries
  int64_t blocks = (int64_t)num_sms() * 8;
  if (blocks > total_tiles) blocks = total_tiles;
  k_fill_matrix_batched<<<unsigned(blocks), dim3(FILL_COLS, FILL_ROWS), 0, (cudaStream_t)stream>>>(geoms, n_geoms,
                                                                                                  total_tiles);
  return launch_status();
}

extern "C" int tb_self_integrals_batched(const tb_geometry_t* geoms, int n_geoms, int64_t total_elements,
                                         tb_stream_t stream) {
  if (!geoms || n_geoms <= 0 || total_elements <= 0) return BAD_ARG;
  int64_t blocks = (total_elements * 32 + 255) / 256;
  if (blocks > (int64_t)num_sms() * 16) blocks = (int64_t)num_sms() * 16;
  k_self_integrals_batched<<<unsigned(blocks), 256, 0, (cudaStream_t)stream>>>(geoms, n_geoms, total_elements);
  return launch_status();
}

extern "C" int tb_rhs_radial(const uint8_t* types, const double* values, double* F, int64_t N, tb_stream_t stream) {
  if (N < 0 || (N > 0 && (!types || !values || !F))) return BAD_ARG;
  if (N == 0) return OK;
  k_rhs<<<unsigned((N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(types, values, F, N);
  return launch_status();
}

extern "C" int tb_rhs_radial_field(const uint8_t* types, const double* values, const double* normal,
                                   const double* field, double* F, int64_t N, tb_stream_t stream) {
  if (N < 0 || (N > 0 && (!types || !values || !normal || !F))) return BAD_ARG;
  if (N == 0) return OK;
  k_rhs_field<<<unsigned((N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(types, values, normal, field, F, N);
  return launch_status();
}

extern "C" int tb_pack_sources(const double* charges, const double* jac, const double* pos, double* sources,
                               int64_t N, tb_stream_t stream) {
  if (N < 0 || (N > 0 && (!charges || !jac || !pos || !sources))) return BAD_ARG;
  if (N == 0) return OK;
  int64_t n = N * NQ;
  k_pack_sources<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(charges, jac, pos, sources, N);
  return launch_status();
}

extern "C" int tb_pack_current_sources(const double* currents, const double* jac, const double* pos,
                                       double* sources, int64_t N, tb_stream_t stream) {
  if (N < 0 || (N > 0 && (!currents || !jac || !pos || !sources))) return BAD_ARG;
  if (N == 0) return OK;
  int64_t n = N * NTRI;
  k_pack_current_sources<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(currents, jac, pos, sources, N);
  return launch_status();
}

extern "C" int tb_current_field_points(const double* points, int64_t M, const double* sources, int64_t Nc,
                                       double* field, tb_stream_t stream) {
  if (M < 0 || Nc < 0) return BAD_ARG;
  if (M == 0) return OK;
  if (!points || !field || (Nc > 0 && !sources)) return BAD_ARG;
  int64_t threads = M * 32;
  k_current_field_points<<<unsigned((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(points, M, sources, Nc,
                                                                                            field);
  return launch_status();
}

extern "C" int tb_current_axial_derivatives(const double* z, int64_t Nz, const double* sources, int64_t Nc,
                                            double* derivs, tb_stream_t stream) {
  if (Nz < 0 || Nc < 0 || Nz > 0x7fffffff) return BAD_ARG;
  if (Nz == 0) return OK;
  if (!z || !derivs || (Nc > 0 && !sources)) return BAD_ARG;
  k_current_axial<<<unsigned(Nz), 256, 0, (cudaStream_t)stream>>>(z, Nz, sources, Nc, derivs);
  return launch_status();
}

extern "C" int tb_field_radial_points(const double* points, int64_t M, const double* sources, int64_t Nq,
                                      double* pot, double* field, tb_stream_t stream) {
  if (M < 0 || Nq < 0) return BAD_ARG;
  if (M == 0) return OK;
  if (!points || (Nq > 0 && !sources) || (!pot && !field)) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int sms = num_sms();
  // Enough points to fill the GPU one thread per point: stage sources in
  // shared memory.  Otherwise split each point's sum over a warp or a block.
  if (M >= (int64_t)sms * 2048) {
    unsigned g = unsigned((M + FP_THREADS - 1) / FP_THREADS);
    if (pot)
      k_field_points_thread<true><<<g, FP_THREADS, 0, s>>>(points, M, sources, Nq, pot, field);
    else
      k_field_points_thread<false><<<g, FP_THREADS, 0, s>>>(points, M, sources, Nq, pot, field);
  } else if (M >= (int64_t)sms * 16) {
    unsigned g = unsigned((M + 7) / 8);
    if (pot)
      k_field_points_team<true, 32><<<g, 256, 0, s>>>(points, M, sources, Nq, pot, field);
    else
      k_field_points_team<false, 32><<<g, 256, 0, s>>>(points, M, sources, Nq, pot, field);
  } else {
    unsigned g = unsigned(M);
    if (pot)
      k_field_points_team<true, 256><<<g, 256, 0, s>>>(points, M, sources, Nq, pot, field);
    else
      k_field_points_team<false, 256><<<g, 256, 0, s>>>(points, M, sources, Nq, pot, field);
  }
  return launch_status();
}

extern "C" int tb_axial_derivatives_radial(const double* z, int64_t Nz, const double* sources, int64_t Nq,
                                           double* derivs, tb_stream_t stream) {
  if (Nz < 0 || Nq < 0) return BAD_ARG;
  if (Nz == 0) return OK;
  if (!z || !derivs || (Nq > 0 && !sources)) return BAD_ARG;
  if (Nz > 0x7fffffff) return BAD_ARG;
  k_axial_derivs<<<unsigned(Nz), 256, 0, (cudaStream_t)stream>>>(z, Nz, sources, Nq, derivs);
  return launch_status();
}

extern "C" int tb_axial_coefficients(const double* derivs, int64_t Nz, double dz, double* coeffs,
                                     tb_stream_t stream) {
  if (Nz < 2 || Nz > SPLINE_MAX_NZ || !(dz > 0) || !derivs || !coeffs) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t n = (Nz - 1) * 7;
  k_axial_quintic<<<unsigned((n + 255) / 256), 256, 0, s>>>(derivs, Nz, dz, coeffs);
  size_t smem = size_t(2 * Nz) * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_axial_cubic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(2 * SPLINE_MAX_NZ * sizeof(double)));
    if (e != cudaSuccess) return CUDA_ERR;
  }
  k_axial_cubic<<<2, 32, smem, s>>>(derivs, Nz, dz, coeffs);
  return launch_status();
}

extern "C" int tb_axial_field_points(const double* points, int64_t M, const double* z, int64_t Nz,
                                     const double* coeffs, double* pot, double* field, tb_stream_t stream) {
  if (M < 0 || Nz < 2) return BAD_ARG;
  if (M == 0) return OK;
  if (!points || !z || !coeffs || (!pot && !field)) return BAD_ARG;
  k_axial_points<<<unsigned((M + 255) / 256), 256, 0, (cudaStream_t)stream>>>(points, M, z, Nz, coeffs, pot, field);
  return launch_status();
}
