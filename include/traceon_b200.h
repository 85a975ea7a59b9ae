/*
 * traceon_b200.h -- C ABI of libtraceon_b200.so, the B200 (sm_100a) CUDA
 * implementation of Traceon's radially symmetric BEM path.
 *
 * Two families of entry points:
 *
 *  1. Reference-compatible entry points.  Same names, argument order and
 *     meaning as the functions the reference binds with ctypes in its
 *     `backend_functions` table (traceon/backend/__init__.py:287-328).  They
 *     take HOST pointers exactly like the reference C backend, copy to the
 *     device, run the CUDA kernels and copy back, so that a maintainer can
 *     point `backend_lib = C.CDLL(...)` at this library.  Where the reference
 *     would call exit(1) or assert, these leave outputs untouched and record a
 *     status readable with tb_last_status().  Scalar geometry helpers
 *     (elliptic integrals, element points, normals, single ring kernels) are
 *     evaluated on the host by the same __host__ __device__ code the kernels
 *     use; all array work runs on the GPU.
 *
 *  2. Batched device entry points (prefix tb_).  All pointers are DEVICE
 *     pointers (e.g. torch.Tensor.data_ptr()), work is enqueued on `stream`,
 *     and every function returns a status code (TB_OK on success).  Nothing
 *     here allocates device memory unless its comment says so.
 *
 * Array layouts (row-major, FP64 unless noted), N = number of line elements:
 *   vertices  (N, 4, 3)  line4 rows [start, end, 1/3-point, 2/3-point], (r, 0, z)
 *   jac       (N, 16)    Gauss weight x |dx/dalpha|
 *   pos       (N, 16, 2) (r, z) of the Gauss nodes
 *   charges   (N,)       surface charge / eps0 (the reference's unit)
 *   sources   (3, Nq)    packed rings for field sums: r[Nq], z[Nq], w[Nq],
 *                        w = charge * jac, Nq = 16 N (tb_pack_sources)
 */
#ifndef TRACEON_B200_H
#define TRACEON_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *tb_stream_t;

/* status codes */
#define TB_OK 0
#define TB_BAD_ARG 1
#define TB_CUDA_ERR 2
#define TB_NONFINITE 3
#define TB_UNSUPPORTED 4
#define TB_SINGULAR 5
#define TB_TIMEOUT 6     /* a bounded wait inside a kernel ran out (the kernel gave up) */

/* per-particle tracer status */
#define TB_TRACE_EXITED 0
#define TB_TRACE_MAX_ATTEMPTS 1
#define TB_TRACE_ROWS_FULL 2
#define TB_TRACE_NONFINITE 3
#define TB_TRACE_ENGINE_TIMEOUT 4  /* tensor-core engine: bounded MMA wait ran out */

/* ======================================================================
 * 1. Reference-compatible entry points (host pointers)
 * ====================================================================== */

/* Compile-time constants read with ctypes in_dll
 * (traceon/backend/__init__.py:58-66). */
extern const size_t TRACING_BLOCK_SIZE;   /* 100000, tracing.c:7 */
extern const int DERIV_2D_MAX_SYM;        /* 9, radial_ring.c:2 / utilities_2d.c */
extern const int N_QUAD_2D_SYM;           /* 16, utilities_2d.c:2 */
extern const int N_TRIANGLE_QUAD_SYM;     /* 12, utilities_3d.c */
extern const int NU_MAX_SYM;              /* 4, three_d.c:4 */
extern const int M_MAX_SYM;               /* 8, three_d.c:5 */

/* Status of the last reference-compatible call on this thread (TB_OK,
 * TB_BAD_ARG, TB_CUDA_ERR, TB_UNSUPPORTED).  No reference counterpart: the
 * reference reports errors by exit(1) (radial.c:305-308). */
int tb_last_status(void);

/* Elliptic integrals, replaces elliptic.c:9-75 (host scalar). */
double ellipkm1(double p);
double ellipk(double k);
double ellipem1(double p);
double ellipe(double k);

/* Replaces utilities_2d.c:18-29 normal_2d (host scalar). */
void normal_2d(const double *p1, const double *p2, double *normal);
/* Replaces utilities_2d.c:31-48; called with rows v[0], v[2], v[3], v[1]
 * (traceon/backend/__init__.py:373-377). */
void higher_order_normal_radial(double alpha, const double *v1, const double *v2, const double *v3,
                                const double *v4, double *normal);
/* Replace utilities_2d.c:50-66 and :68-87 (host scalar). */
void position_and_jacobian_radial(double alpha, const double *v1, const double *v2, const double *v3,
                                  const double *v4, double *pos, double *jac);
void delta_position_and_jacobian_radial(double alpha, const double *v1, const double *v2, const double *v3,
                                        const double *v4, double *pos, double *jac);

/* Ring kernels, replace radial_ring.c:21-53 (host scalar; the trailing
 * void* is ignored as in the reference). */
double potential_radial_ring(double r0, double z0, double delta_r, double delta_z, void *unused);
double dr1_potential_radial_ring(double r0, double z0, double delta_r, double delta_z, void *unused);
double dz1_potential_radial_ring(double r0, double z0, double delta_r, double delta_z, void *unused);
/* Replaces utilities_2d.c:91-105. */
double flux_density_to_charge_factor(double K);
/* Replaces radial.c:123-148 (host scalar). */
double charge_radial(const double *vertices, double charge);
/* Replaces radial_ring.c:78-107 (host scalar). */
void current_field_radial_ring(double x0, double y0, double x, double y, double *result);
/* Replaces radial_ring.c:73-76 (host scalar). */
double current_potential_axial_radial_ring(double z0, double r, double z);

/* Self-integrands for SciPy LowLevelCallable (radial.c:182-196, :203-222).
 * Host scalar; the solver of this library does not use them -- its
 * diagonal is integrated on the GPU (tb_self_integrals). */
double self_potential_radial(double alpha, void *line_points);
double self_field_dot_normal_radial(double alpha, void *args);

/* GPU: replaces radial.c:224-246 fill_jacobian_buffer_radial. */
void fill_jacobian_buffer_radial(double *jac, double *pos, const double *vertices, size_t N_lines);

/* GPU: replaces radial.c:249-310 fill_matrix_radial.  Accumulates (+=) rows
 * [start, end] of `matrix` (row stride N_matrix) exactly like the reference,
 * including its 16-point Gauss diagonal that the solver later overwrites.
 * Unknown excitation types leave the matrix unchanged and set TB_BAD_ARG. */
void fill_matrix_radial(double *matrix, const double *lines, const uint8_t *types, const double *values,
                        const double *jac, const double *pos, size_t N_lines, size_t N_matrix, int start,
                        int end);

/* GPU: replace radial.c:105-121 and :150-173 (one point per call). */
double potential_radial(const double *point, const double *charges, const double *jac, const double *pos,
                        size_t N);
void field_radial(const double *point, double *result, const double *charges, const double *jac,
                  const double *pos, size_t N);
/* GPU: replaces radial.c:18-36 (accumulates into derivs (N_z, 9)). */
void axial_derivatives_radial(double *derivs, const double *charges, const double *jac, const double *pos,
                              size_t N, const double *z, size_t N_z);
/* GPU: replaces radial.c:55-83 (positions (N, 12, 3)). */
void current_field_radial(const double *point, double *result, const double *currents, const double *jac,
                          const double *pos, size_t N);
/* GPU: replaces radial.c:85-103 (accumulates). */
void current_axial_derivatives_radial(double *derivs, const double *currents, const double *jac,
                                      const double *pos, size_t N, const double *z, size_t N_z);
/* GPU: replaces radial.c:38-53. */
double current_potential_axial(double z0, const double *currents, const double *jac, const double *pos,
                               size_t N);
/* Replace radial.c:312-344 and :347-384 (host scalar: O(1) table lookup). */
double potential_radial_derivs(const double *point, const double *z, const double *coeffs, size_t N_z);
void field_radial_derivs(const double *point, double *field, const double *z, const double *coeffs,
                         size_t N_z);

/* Field callbacks of the tracer, tracing.c:125-174 (field_fun type,
 * traceon/backend/__init__.py:89).  field_radial_traceable evaluates the BEM
 * sums on the GPU; field_radial_derivs_traceable is a host table lookup. */
void field_radial_traceable(const double *position, const double *velocity, void *args, double *elec_out,
                            double *mag_out);
void field_radial_derivs_traceable(const double *position, const double *velocity, void *args,
                                   double *elec_out, double *mag_out);

/* GPU: replaces tracing.c:60-123 trace_particle.  `field` must be one of
 * this library's field_radial_traceable / field_radial_derivs_traceable
 * (with the matching args struct, radial.c:175-180 / three_d.c:26-31); the
 * whole trajectory is then integrated on the GPU.  Any other callback sets
 * TB_UNSUPPORTED and returns 1 (only the start row).  Writes at most
 * TRACING_BLOCK_SIZE rows and returns the row count, like the reference. */
size_t trace_particle(double *times, double *positions, double charge_over_mass, void *field,
                      const double *bounds, double atol, void *args);

/* Replaces tracing.c:184-223 (host: linear crossing on a host trajectory). */
bool plane_intersection(const double *p0, const double *normal, const double *positions, size_t N_p,
                        double *result);

/* Reference entry points outside the radial path (3D geometry, the
 * kronrod_adaptive test helper).  Exported so the reference's import-time
 * getattr loop (traceon/backend/__init__.py:341-352) succeeds; calling them
 * sets TB_UNSUPPORTED and leaves outputs untouched. */
double kronrod_adaptive(void *f, double a, double b, void *args, double abs_tol, double rel_tol);
void normal_3d(const double *points, double *normal);
void position_and_jacobian_3d(double alpha, double beta, const double *triangle, double *pos, double *jac);
void axial_coefficients_3d(const double *charges, const double *jac, const double *pos, double *trig_cos,
                           double *trig_sin, size_t N, const double *z, double *out, size_t N_z);
void fill_jacobian_buffer_current_three_d(const double *lines, double *jac, double *pos, double *dirs,
                                          size_t N);
double potential_3d_derivs(const double *point, const double *z, const double *coeffs, size_t N_z);
void field_3d_derivs(const double *point, double *field, const double *z, const double *coeffs, size_t N_z);
void fill_jacobian_buffer_3d(double *jac, double *pos, const double *vertices, size_t N);
void triangle_areas(const double *triangles, double *out, size_t N);

/* ======================================================================
 * 2. Batched device entry points (device pointers, explicit stream)
 * ====================================================================== */

/* Graded cubic meshes on the device (no reference counterpart: the
 * reference's Path.mesh spaces nodes uniformly, traceon/geometry.py:39-70).
 * Segment s of segments (S, 4) = (r0, z0, r1, z1) gets offsets[s + 1] -
 * offsets[s] elements with Chebyshev-Lobatto nodes (dense toward both ends);
 * vertices (N, 4, 3) in line4 order [start, end, 1/3, 2/3] of (r, 0, z),
 * N = offsets[S], offsets[0] = 0, non-decreasing (device arrays).
 * Coordinates carry the reference Mesh's 16-bit mantissa truncation. */
int tb_mesh_segments(const double *segments, const int64_t *offsets, int64_t S, double *vertices, int64_t N,
                     tb_stream_t stream);

/* Replaces radial.c:224-246 for N elements on the device. */
int tb_jacobian_buffer_radial(const double *vertices, double *jac, double *pos, int64_t N, tb_stream_t stream);

/* Collocation data of each element at alpha = 0: target (N,2) = (r, z) and
 * normal (N,2) (radial.c:266-267, utilities_2d.c:31-48). */
int tb_element_targets(const double *vertices, double *target, double *normal, int64_t N, tb_stream_t stream);

/* Off-diagonal BEM matrix, replaces radial.c:249-310 for rows [row0, row1)
 * of an (N, N) matrix with row stride lda.  types uint8 (N), values (N).
 * accumulate != 0 adds to A (the reference semantics), else overwrites.
 * gauss_diagonal != 0 also writes the reference's 16-point value on the
 * diagonal; otherwise the diagonal entry is left untouched. */
int tb_fill_matrix_radial(double *A, int64_t lda, const double *vertices, const uint8_t *types,
                          const double *values, const double *jac, const double *pos, int64_t N, int64_t row0,
                          int64_t row1, int accumulate, int gauss_diagonal, tb_stream_t stream);

/* One geometry of a batch (device pointers).  tile0 / elem0 are set by
 * tb_batch_plan. */
typedef struct {
  const double *vertices;   /* (N, 4, 3) cubic line elements */
  const uint8_t *types;     /* (N) excitation types */
  const double *values;     /* (N) excitation values */
  const double *jac;        /* (N, 16) from tb_jacobian_buffer_radial */
  const double *pos;        /* (N, 16, 2) */
  double *A;                /* (N, lda) the geometry's matrix */
  int64_t lda;
  int64_t N;
  int64_t tile0;            /* first global fill tile (set by tb_batch_plan) */
  int64_t elem0;            /* first global element (set by tb_batch_plan) */
} tb_geometry_t;

/* Host helper: numbers the fill tiles and elements of n_geoms geometries
 * (host array; sets tile0 / elem0) and returns the total number of tiles
 * (-1 on bad sizes); *total_elements receives the sum of N.  Copy the array
 * to device memory for the two calls below. */
int64_t tb_batch_plan(tb_geometry_t *geoms, int n_geoms, int64_t *total_elements);

/* fill_matrix_radial (radial.c:249-310, off-diagonal entries) of many
 * geometries of uneven N in one persistent launch; geoms is a DEVICE array
 * prepared by tb_batch_plan.  No counterpart in the reference (its Python
 * solver fills one geometry at a time, solver.py:204-232). */
int tb_fill_matrix_radial_batched(const tb_geometry_t *geoms, int n_geoms, int64_t total_tiles, tb_stream_t stream);

/* The singular self terms (as tb_self_integrals) of every element of a batch,
 * stored on each geometry's matrix diagonal; one launch. */
int tb_self_integrals_batched(const tb_geometry_t *geoms, int n_geoms, int64_t total_elements, tb_stream_t stream);

/* ---- Batched solve: many geometries of uneven N filled, factored and
 * solved in ONE persistent launch.  No counterpart in the reference, which
 * fills (solver.py:204-232) and solves (solver.py:160-180, LAPACK dgesv) one
 * geometry at a time.  Each matrix is padded to T x T tiles of 64 x 64 and
 * factored without pivoting (left-looking, tile tasks in dependency order,
 * FP64); a zero or non-finite pivot or charge marks the geometry
 * TB_SINGULAR for the caller to solve with the pivoted LU. */
typedef struct {
  const double *vertices;   /* (N, 4, 3) cubic line elements (device) */
  const uint8_t *types;     /* (N) excitation types */
  const double *values;     /* (N) excitation values */
  const double *rhs;        /* (N) right-hand side */
  double *charges;          /* (N) solution (out) */
  int64_t N;
  /* set by tb_batch_solve_plan: */
  int64_t T;                /* tiles per side, ceil(N / 64) */
  int64_t a_off;            /* workspace offset (doubles) of the padded (64 T)^2 matrix */
  int64_t inv_off;          /* workspace offset of the T inverse tiles (64 x 64) */
  int64_t v_off;            /* workspace offset of the 64 T sweep vector */
  int64_t flag_off;         /* flag offset (int32 words) of T^2 + 2 T + 1 words */
  int64_t ring_off;         /* the geometry's first ring in the packed sources (16 N rings) */
} tb_batch_item_t;

/* Host helper: sets T and the offsets of n_items items (host array), writes
 * the task list (4 int32 per task) when tasks is not NULL and returns the
 * number of tasks (-1 on bad sizes).  sizes[0] = workspace doubles,
 * sizes[1] = flag words, sizes[2] = source rings (16 x sum N).  Copy items
 * and tasks to device memory for tb_batch_solve. */
int64_t tb_batch_solve_plan(tb_batch_item_t *items, int n_items, int32_t *tasks, int64_t *sizes);

/* Fills, factors and solves every item in one persistent launch (items,
 * tasks, work (16-byte aligned), flags, sources, status: device memory).
 * flags (n_flags = sizes[1] words) and status are reset by this call with
 * two memsets on the stream, so a CUDA graph captured around it replays
 * cleanly.  sources: NULL, or (3, total_rings) receiving the charges packed
 * as tb_pack_sources does (r | z | charge x jacobian), geometry g from ring
 * ring_off -- the layout tb_trace_rk45_geometries reads.  status[g]: TB_OK,
 * TB_SINGULAR, or -1 if the launch gave up on a bounded wait (every wait is
 * bounded by tb_set_wait_limit).  blocks_per_sm: 0 = as many as fit. */
int tb_batch_solve(const tb_batch_item_t *items, int n_items, const int32_t *tasks, int64_t n_tasks, double *work,
                   int32_t *flags, int64_t n_flags, double *sources, int64_t total_rings, int32_t *status,
                   int blocks_per_sm, tb_stream_t stream);

/* Singular self terms: diag[i] = integral over alpha in [-1, 1] of the
 * self integrand of element i (self_potential_radial, radial.c:182-196, for
 * voltage rows; self_field_dot_normal_radial - 1, radial.c:203-222 and
 * solver.py:239-244, for dielectric / magnetizable rows), computed by
 * composite 16-point Gauss-Legendre on intervals graded geometrically toward
 * the log singularity at alpha = 0 (FP64, ~1e-15 relative).  If A != NULL the
 * values are also stored on the diagonal of A (stride lda). */
int tb_self_integrals(const double *vertices, const uint8_t *types, const double *values, double *diag,
                      double *A, int64_t lda, int64_t N, tb_stream_t stream);

/* Right-hand side of solver.py:118-150 for voltage / dielectric rows: F = V
 * for types 1, 2, 5; 0 for type 3.  (Magnetizable rows need the
 * pre-existing field and are filled by the caller.) */
int tb_rhs_radial(const uint8_t *types, const double *values, double *F, int64_t N, tb_stream_t stream);

/* The whole right-hand side of solver.py:118-150, magnetizable rows
 * included: F = V for types 1, 2, 5; 0 for type 3; -factor(mu) H . n for
 * type 6 (flux_density_to_charge_factor, utilities_2d.c:91-105), with
 * normal (N, 2) from tb_element_targets and field (N, 3) the pre-existing
 * field (H_x, H_y, H_z) at each element's collocation point (r, 0, z), e.g.
 * from tb_current_field_points, or NULL for none. */
int tb_rhs_radial_field(const uint8_t *types, const double *values, const double *normal, const double *field,
                        double *F, int64_t N, tb_stream_t stream);

/* Dense LU with partial pivoting in FP64, in place on A (N x N, row stride
 * lda): P A = L U.  ipiv (N) int32 receives the pivot row of each step
 * (LAPACK convention, 0-based); perm (N) int32, if not NULL, the resulting
 * row permutation (row i of P A is row perm[i] of A).  Replaces the
 * factorisation inside numpy.linalg.solve (solver.py:173, LAPACK dgesv).
 * A zero pivot yields non-finite factors (checked by the caller, as
 * solver.py:175 checks the charges). */
int tb_lu_factor(double *A, int64_t lda, int32_t *ipiv, int64_t N, tb_stream_t stream);
int tb_lu_factor_perm(double *A, int64_t lda, int32_t *ipiv, int32_t *perm, int64_t N, tb_stream_t stream);

/* Solves A x = f for nrhs right-hand sides stored as rows of F (nrhs, N)
 * (row stride ldf) into the rows of X (nrhs, N) (row stride ldx, X != F),
 * given the factors and permutation of tb_lu_factor_perm. */
int tb_lu_solve_perm(const double *LU, int64_t lda, const int32_t *perm, int64_t N, const double *F, int64_t ldf,
                     double *X, int64_t ldx, int64_t nrhs, tb_stream_t stream);

/* Packs charges (N), jac (N,16), pos (N,16,2) into sources (3, 16 N):
 * r, z and w = charge * jac. */
int tb_pack_sources(const double *charges, const double *jac, const double *pos, double *sources, int64_t N,
                    tb_stream_t stream);

/* Blocked LU without pivoting, in place (A = L U, L unit lower), FP64 or
 * FP32.  The radial BEM matrices need no pivoting (growth factor < 1 on the
 * lens meshes); no reference counterpart beyond the factorisation inside
 * numpy.linalg.solve (solver.py:173). */
int tb_lu_nopiv_f64(double *A, int64_t lda, int64_t N, tb_stream_t stream);
int tb_lu_nopiv_f32(float *A, int64_t lda, int64_t N, tb_stream_t stream);
/* The same FP32 factorisation in 256-column panels with the updates on the
 * tensor cores (tcgen05, 3xTF32: TF32 head/tail split of both operands,
 * FP32 accumulation in tensor memory); the trailing matrix is updated once
 * per panel from operands pre-split into `work`.  work: device scratch of
 * tb_lu_nopiv_f32_tc_workspace(N) bytes, 16-byte aligned (required).  err
 * (device int) is set to 1 if a bounded wait inside a tensor-core kernel ran
 * out.  Used by tb_solve_mixed. */
int64_t tb_lu_nopiv_f32_tc_workspace(int64_t N);
int tb_lu_nopiv_f32_tc(float *A, int64_t lda, int64_t N, void *work, int64_t work_bytes, int *err,
                       tb_stream_t stream);
/* C (M x N, ldc) -= A (M x K, lda) . B (K x N, ldb), FP32 row-major, with
 * the 3xTF32 tensor-core kernels of tb_lu_nopiv_f32_tc (exposed for tests):
 * work == NULL stages and splits the operands in every CTA; otherwise `work`
 * (16-byte aligned, tb_gemm_tf32x3_workspace(M, N, K) bytes) receives the
 * pre-split operands, which the GEMM streams with bulk copies. */
int64_t tb_gemm_tf32x3_workspace(int64_t M, int64_t N, int64_t K);
int tb_gemm_sub_tf32x3(float *C, int64_t ldc, const float *A, int64_t lda, const float *B, int64_t ldb, int64_t M,
                       int64_t N, int64_t K, void *work, int64_t work_bytes, int *err, tb_stream_t stream);

/* Mixed-precision solve of A x = f for the nrhs (<= 16) rows of F (nrhs, N)
 * into X (nrhs, N): FP32 LU without pivoting of A diag(c), c_j = 1 / max_i
 * |A_ij|, then FP64 iterative refinement with the FP64 matrix until, for
 * every right-hand side, max |correction| / max |x| <= tol, or the error
 * left after the last correction, extrapolated from the contraction of the
 * last two, is (at most max_iter rounds; corrections that stall within 100
 * tol count as converged); *last_rel_out gets the last correction's size or
 * that extrapolated error.  `work`
 * is device scratch of tb_solve_mixed_workspace(N, nrhs) bytes.  Returns
 * TB_SINGULAR when refinement does not converge (the caller then solves with
 * tb_lu_factor_perm / tb_lu_solve_perm).  Replaces numpy.linalg.solve
 * (solver.py:173) with the same FP64 answer. */
int64_t tb_solve_mixed_workspace(int64_t N, int64_t nrhs);
int tb_solve_mixed(const double *A, int64_t lda, int64_t N, const double *F, double *X, int64_t nrhs, void *work,
                   int64_t work_bytes, int max_iter, double tol, int *iters_out, double *last_rel_out,
                   tb_stream_t stream);

/* Dense solve that allocates nothing: LU-factorises A in place (as
 * tb_lu_factor_perm) and solves for the nrhs rows of F into the rows of X (as
 * tb_lu_solve_perm), keeping the pivots and permutation in a static device
 * array of the library instead of caller memory.  No counterpart in the
 * reference.  It exists for callers that cannot allocate device memory (a
 * plug-in in a host application that owns the GPU memory pool, a control
 * loop that may not allocate after start-up).  Limit: N <= 32768 (larger N
 * returns TB_BAD_ARG); the array (256 KiB) is held by every GPU that loads
 * the library until the process exits.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture; after a cudaDeviceReset the first call in the
 * new context looks it up again.  All calls share the array: calls that overlap
 * on the GPU (different streams, or other threads) race and must be
 * serialised by the caller.  Calls no cudaMalloc or cudaFree. */
int tb_lu_solve_noalloc(double *A, int64_t lda, int64_t N, const double *F, int64_t ldf, double *X, int64_t ldx,
                        int64_t nrhs, tb_stream_t stream);

/* Packs current rings: currents (N), jac (N,12), pos (N,12,3) (y == 0) into
 * sources (3, 12 N): r, z and w = current * jac. */
int tb_pack_current_sources(const double *currents, const double *jac, const double *pos, double *sources,
                            int64_t N, tb_stream_t stream);

/* Magnetic field H at M points from Nc packed current rings, the batched
 * form of current_field_radial (radial.c:55-83). */
int tb_current_field_points(const double *points, int64_t M, const double *sources, int64_t Nc, double *field,
                            tb_stream_t stream);

/* Axial derivatives of the current scalar potential at N_z points,
 * radial.c:85-103 (overwrites derivs (N_z, 9)).  Column 0 is the on-axis
 * potential, current_potential_axial (radial.c:38-53). */
int tb_current_axial_derivatives(const double *z, int64_t Nz, const double *sources, int64_t Nc, double *derivs,
                                 tb_stream_t stream);

/* Potential and field at M points (M,3) from Nq packed sources: the batched
 * form of potential_radial / field_radial (radial.c:105-173).  pot (M) and/or
 * field (M,3) may be NULL. */
int tb_field_radial_points(const double *points, int64_t M, const double *sources, int64_t Nq, double *pot,
                           double *field, tb_stream_t stream);

/* Axial derivatives at N_z points, radial.c:18-36 (overwrites derivs
 * (N_z, 9)). */
int tb_axial_derivatives_radial(const double *z, int64_t Nz, const double *sources, int64_t Nq,
                                double *derivs, tb_stream_t stream);

/* Interpolation coefficients (N_z - 1, 9, 6) from derivs (N_z, 9) on an
 * equally spaced z grid with spacing dz, replaces field.py:914-937: quintic
 * Hermite through (d_i, d_i+1, d_i+2) for i <= 6, not-a-knot cubic spline
 * for i = 7, 8.  N_z <= 12288. */
int tb_axial_coefficients(const double *derivs, int64_t Nz, double dz, double *coeffs, tb_stream_t stream);

/* Potential / field at M points from axial coefficients, the batched form
 * of radial.c:312-384.  pot and/or field may be NULL. */
int tb_axial_field_points(const double *points, int64_t M, const double *z, int64_t Nz, const double *coeffs,
                          double *pot, double *field, tb_stream_t stream);

/* Field sources of the tracer. */
typedef struct {
  const double *elec_sources;   /* (3, n_elec) packed rings or NULL */
  int64_t n_elec;
  const double *mag_sources;    /* (3, n_mag) packed rings or NULL */
  int64_t n_mag;
  const double *cur_sources;    /* (3, n_cur) packed current rings or NULL */
  int64_t n_cur;
  const double *field_bounds;   /* (3,2) strict field bounds or NULL (tracing.c:136-138) */
  const double *axial_z;        /* axial interpolation: z (N_z) or NULL */
  const double *axial_elec;     /* (N_z-1, 9, 6) */
  const double *axial_mag;      /* (N_z-1, 9, 6) or NULL */
  int64_t axial_nz;
} tb_field_t;

/* Tracing options. */
typedef struct {
  double bounds[6];       /* (xmin, xmax, ymin, ymax, zmin, zmax), inclusive (tracing.c:79-81) */
  double atol;            /* absolute tolerance (tracing.c:106-108) */
  double plane_z;         /* record the last crossing of z = plane_z ... */
  int record_plane;       /* ... when nonzero (cubic Hermite on the bracketing states) */
  int64_t max_attempts;   /* step-attempt cap per particle (> 0) */
  int64_t max_rows;       /* rows per particle in `rows` (>= 2) or 0 for none */
  int team_warps;         /* warps cooperating on one particle's BEM sums: 1, 2, 4 or 8; 0 = auto */
} tb_trace_opts_t;

/* Adaptive RKF45 tracing of n particles (tracing.c:60-123 per particle).
 *   start (n, 6)   x, y, z, vx, vy, vz (SI)
 *   t0 (n) or NULL start times; qm (n) charge/mass per particle
 *   rows (n, max_rows, 7) t, x, y, z, vx, vy, vz (row 0 = start) or NULL
 *   nrows (n) int64 rows written (or NULL), status (n) int32 (TB_TRACE_*)
 *   final (n, 7) last accepted state (t, x..vz) or NULL
 *   plane (n, 7) last crossing of z = plane_z (t, x..vz) or NULL; NaN if none
 *   counters (n, 2) int64 accepted steps / attempts, or NULL
 *   work (1) int32 device scratch, zeroed by the call: the work-queue head.
 * Persistent kernel: teams of warps pull particles from the queue. */
int tb_trace_rk45(const double *start, const double *t0, const double *qm, int64_t n, const tb_field_t *field,
                  const tb_trace_opts_t *opts, double *rows, int64_t *nrows, int32_t *status, double *final_state,
                  double *plane, int64_t *counters, int32_t *work, tb_stream_t stream);

/* Many geometries in one launch (no reference counterpart: the reference
 * traces one field at a time).  As tb_trace_rk45 with a BEM field whose
 * electrostatic sources are the concatenation of n_geoms geometries'
 * sources: particle i sums only the rings src_offsets[geom[i]] ..
 * src_offsets[geom[i] + 1] - 1 of field->elec_sources (n_elec = total).
 *   geom (n) int32 device, ids in [0, n_geoms) (an id outside sums no rings)
 *   src_offsets (n_geoms + 1) int64 device, non-decreasing, last <= n_elec
 *   geom_bounds NULL (opts->bounds for every particle) or (n_geoms, 6)
 *   device: each geometry's own bounding box, as opts->bounds
 * Electrostatic sources only (n_mag = n_cur = 0, no axial table); TB_BAD_ARG
 * otherwise. */
int tb_trace_rk45_geometries(const double *start, const double *t0, const double *qm, const int32_t *geom,
                             int64_t n, const tb_field_t *field, const int64_t *src_offsets, int64_t n_geoms,
                             const double *geom_bounds, const tb_trace_opts_t *opts, double *rows, int64_t *nrows, int32_t *status,
                             double *final_state, double *plane, int64_t *counters, int32_t *work,
                             tb_stream_t stream);

/* Plane crossings of trajectories stored by tb_trace_rk45 (device arrays):
 * per trajectory the crossing nearest its end, by linear interpolation, as
 * plane_intersection (traceon/backend/tracing.c:184-223) finds it.
 *   rows (n, max_rows, 7), nrows (n): as written by tb_trace_rk45
 *   p0, normal: host double[3], a point of the plane and its normal (non-zero)
 *   out (n, 7) t, x..vz at the crossing (NaN where there is none)
 *   found (n) int32 1 / 0 (the reference's bool return) */
int tb_plane_intersection_rows(const double *rows, const int64_t *nrows, int64_t n, int64_t max_rows,
                               const double *p0, const double *normal, double *out, int32_t *found,
                               tb_stream_t stream);

/* Least-squares focus of a beam (focus_position, traceon/focus.py:9-42)
 * from its final states on the device: particle i's x, y, z, vx, vy, vz at
 * states + i * ld (ld >= 6; e.g. ld = 7 on the x column of a (n, 7) t..vz
 * array).  out: device double[3] = (x, y, z) of the focus, NaN when the
 * system is rank deficient (fewer than two particles, or all final
 * directions equal).  work: device scratch of tb_focus_position_workspace()
 * bytes. */
int64_t tb_focus_position_workspace(void);
int tb_focus_position(const double *states, int64_t n, int64_t ld, double *out, void *work, int64_t work_bytes,
                      tb_stream_t stream);

/* ---------------------------------------------------------------------
 * Learned field surrogate (no reference counterpart; see tb_mlp.cuh).
 * Network: 16 input features -> 4 x 128 SiLU -> 16 outputs; parameters in
 * one flat array of 51,344 entries (W1 128x16, b1, W2 128x128, b2, W3, b3,
 * W4, b4, W5 16x128, b5), FP32 master copy plus BF16 copy.  Matrices are
 * BF16 (device pointers passed as void*), accumulators FP32.
 * ------------------------------------------------------------------- */

/* C (M x N, fp32, row stride ldc) (+)= A . B^T on the tensor cores, BF16 in,
 * FP32 accumulate.  A is M x K (a_t = 0: A[m*lda + k]; a_t = 1:
 * A[k*lda + m]); B is N x K likewise with b_t. */
int tb_mlp_gemm(const void *A, int64_t lda, int a_t, const void *B, int64_t ldb, int b_t, float *C, int64_t ldc,
                int64_t M, int64_t N, int64_t K, int accumulate, tb_stream_t stream);
/* Z = C + b (Z may be NULL), Y = silu(Z) as BF16; C, Z, Y are M x N. */
int tb_mlp_bias_silu(const float *C, const float *b, float *Z, void *Y, int64_t M, int64_t N, tb_stream_t stream);
/* Y = C + b (FP32). */
int tb_mlp_bias_out(const float *C, const float *b, float *Y, int64_t M, int64_t N, tb_stream_t stream);
/* dY = 2 (Y - T) w / (M n_out) for the first n_out of N columns (BF16, zero
 * elsewhere); loss_part[block] = partial sums of w (Y - T)^2 (256 entries per
 * block).  T is M x n_out, w (M) or NULL. */
int tb_mlp_mse_grad(const float *Y, const float *T, const float *w, void *dY, float *loss_part, int64_t M, int64_t N,
                    int64_t n_out, tb_stream_t stream);
/* dZ = dA * silu'(Z) (BF16), n elements. */
int tb_mlp_silu_back(const float *dA, const float *Z, void *dZ, int64_t n, tb_stream_t stream);
/* db[c] = sum over the M rows of dZ (BF16, M x N). */
int tb_mlp_colsum(const void *dZ, float *db, int64_t M, int64_t N, tb_stream_t stream);
/* Adam step (bias-corrected, step >= 1) on n FP32 parameters, refreshing the
 * BF16 copy pb. */
int tb_mlp_adam(float *p, const float *g, float *m, float *v, void *pb, int64_t n, float lr, float b1, float b2,
                float eps, int64_t step, tb_stream_t stream);
/* Input features (M x 16, BF16) of M points (M,3): rho = r / r_max,
 * zeta = (z - z_c) / z_half. */
int tb_mlp_features(const double *points, int64_t M, double r_max, double z_c, double z_half, void *X,
                    tb_stream_t stream);

/* Surrogate description for tb_trace_surrogate. */
typedef struct {
  const void *weights_bf16;     /* flat BF16 parameters */
  const float *params_f32;      /* flat FP32 parameters (biases are read from here) */
  double r_max, z_c, z_half;    /* input normalisation; also the domain in r */
  double z_lo, z_hi;            /* domain in z */
  int n_electrodes;             /* field sources: first the electrodes, outputs 3s..3s+2 = (phi, E_r, E_z)
                                   of electrode s at 1 V ... */
  int n_coils;                  /* ... then the current coils, (magnetostatic potential, H_r, H_z) of coil
                                   s at 1 A-turn; 1 <= n_electrodes + n_coils <= 10 */
  double strengths[10];         /* electrode voltages (V), then coil currents (A-turns) */
  float scale[32];              /* output scales */
  int env_power;                /* correction = strength * scale * y * rho^p (radial part: rho^(p+1)) */
  const double *segments;       /* (n_segments, 4) electrode segments r0, z0, r1, z1 (device) */
  int n_segments;               /* <= 64 */
  double fallback_dist;         /* exact BEM within this distance of a segment */
  int engine;                   /* network engine: 0 = tcgen05 (groups of 128 particles, accumulators in
                                   tensor memory), 1 = warp-level mma.sync (32 particles per warp) */
} tb_surrogate_t;

/* RKF45 tracing (tracing.c:60-123 step control) through the surrogate field:
 * axial-series field of `field->axial_elec` (the table for the actual
 * voltages) plus the network's correction, exact BEM sums of
 * `field->elec_sources` near electrodes and outside the network's domain.
 * With a magnetic part (n_coils > 0, `field->axial_mag` -- the table for the
 * actual currents -- or magnetostatic / current sources) the magnetic field
 * H is built the same way and the force is q/m (E + mu0 v x H)
 * (tracing.c:20-57, 141-163).  Endpoint mode only (no trajectories);
 * counters (n, 3): accepted steps, attempts, field evaluations that fell
 * back to BEM. */
int tb_trace_surrogate(const double *start, const double *t0, const double *qm, int64_t n, const tb_field_t *field,
                       const tb_surrogate_t *sur, const tb_trace_opts_t *opts, int32_t *status, double *final_state,
                       double *plane, int64_t *counters, int32_t *work, tb_stream_t stream);

/* The surrogate field E (M,3) at M points (M,3) exactly as the tracer sees
 * it (fallback included), and the magnetic field H (M,3) into out_h unless
 * NULL (zero without a magnetic part); used_bem (M) int32 flags BEM
 * fallbacks (-1: the engine's wait ran out), or NULL. */
int tb_surrogate_field_points(const double *points, int64_t M, const tb_field_t *field, const tb_surrogate_t *sur,
                              double *out, double *out_h, int32_t *used_bem, tb_stream_t stream);

/* Number of SMs of the current device (grid sizing helper). */
int tb_num_sms(void);

/* Lookahead of the mixed solve's factorisation (tb_solve_mixed,
 * tb_lu_nopiv_f32_tc): the trailing update of each 256-column panel is split
 * into the next panel's columns (on every SM) and the remaining columns, which
 * run on a second stream on all but reserve_sms SMs while the next panel is
 * factored on the caller's stream.  Default: one SM in five; 0 turns it
 * off, a negative value restores the default.  One value per process;
 * returns the previous one.  The factors are the same either way, bit for
 * bit. */
int tb_set_solve_lookahead(int reserve_sms);

/* Bound, in SM clock cycles, of the progress waits inside this library's
 * kernels: the tensor-core engines' waits for their MMA chains and copy
 * stages, and the triangular sweeps' waits for blocks other CTAs publish.
 * No reference counterpart (the reference has no GPU code).  A wait that
 * runs out makes the kernel give up cleanly: the mixed solve returns
 * TB_TIMEOUT, the surrogate tracer ends the particles in hand with
 * TB_TRACE_ENGINE_TIMEOUT.  Work already in flight (MMAs, bulk copies) is
 * always drained under the default bound before a CTA releases its memory.
 * cycles >= 1 sets the bound for launches made after the call (one value
 * per process); cycles <= 0 restores the default (2e9, about 1 s).
 * Returns the previous bound. */
int64_t tb_set_wait_limit(int64_t cycles);

#ifdef __cplusplus
}
#endif

#endif /* TRACEON_B200_H */
