// tb_lu_mixed.cu -- blocked LU without pivoting (FP32 or FP64) and the
// mixed-precision charge solve: FP32 factors of the column-equilibrated BEM
// matrix, FP64 iterative refinement against the FP64 matrix.
//
// Why no pivoting: the collocation matrices of the radial BEM are close to
// a positive single-layer operator; on the lens meshes the growth factor of
// unpivoted elimination is below 1 and the unpivoted FP64 solution agrees
// with LAPACK dgesv to ~1e-13 (tests/test_gpu_solve.py checks both).  The
// column scaling c_j = 1 / max_i |A_ij| removes the element-size spread of
// graded meshes from the condition number (about 9.6e4 -> 2.3e3 at
// N = 1000), which is what lets FP32 factors converge under refinement.
//
// Blocked right-looking factorisation, per panel of NB columns:
//   k_diag_lu      one CTA factors the NB x NB diagonal block in shared memory
//   k_trsm_right   L21 = A21 U11^-1   (one thread per row)
//   k_trsm_left    U12 = L11^-1 A12   (one thread per column)
//   k_gemm_update  A22 -= L21 U12     (register-tiled SIMT GEMM)
#include <cstring>

#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

constexpr int MX_NB = 64;

template <class T>
__global__ void __launch_bounds__(256) k_diag_lu(T* __restrict__ A, int64_t lda, int64_t k0, int nb) {
  __shared__ T D[MX_NB][MX_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) D[e / nb][e % nb] = A[(k0 + e / nb) * lda + k0 + e % nb];
  __syncthreads();
  for (int k = 0; k < nb - 1; k++) {
    const T piv = D[k][k];
    for (int e = threadIdx.x; e < (nb - k - 1) * (nb - k - 1); e += blockDim.x) {
      int i = k + 1 + e / (nb - k - 1), j = k + 1 + e % (nb - k - 1);
      T l = D[i][k] / piv;
      D[i][j] -= l * D[k][j];
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < nb; i += blockDim.x) D[i][k] /= piv;
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) A[(k0 + e / nb) * lda + k0 + e % nb] = D[e / nb][e % nb];
}

// rows i >= k0 + nb: A[i, k0:k0+nb] <- A[i, k0:k0+nb] U11^-1
template <class T>
__global__ void __launch_bounds__(128) k_trsm_right(T* __restrict__ A, int64_t lda, int64_t N, int64_t k0, int nb) {
  __shared__ T U[MX_NB][MX_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) U[e / nb][e % nb] = A[(k0 + e / nb) * lda + k0 + e % nb];
  __syncthreads();
  int64_t i = k0 + nb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  T* row = A + i * lda + k0;
  T x[MX_NB];
#pragma unroll
  for (int j = 0; j < MX_NB; j++) {
    if (j < nb) {
      T v = row[j];
      for (int m = 0; m < j; m++) v -= x[m] * U[m][j];
      x[j] = v / U[j][j];
      row[j] = x[j];
    }
  }
}

// columns j >= k0 + nb: A[k0:k0+nb, j] <- L11^-1 A[k0:k0+nb, j] (L11 unit lower)
template <class T>
__global__ void __launch_bounds__(128) k_trsm_left(T* __restrict__ A, int64_t lda, int64_t N, int64_t k0, int nb) {
  __shared__ T L[MX_NB][MX_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) L[e / nb][e % nb] = A[(k0 + e / nb) * lda + k0 + e % nb];
  __syncthreads();
  int64_t c = k0 + nb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  T x[MX_NB];
#pragma unroll
  for (int i = 0; i < MX_NB; i++) {
    if (i < nb) {
      T v = A[(k0 + i) * lda + c];
      for (int m = 0; m < i; m++) v -= L[i][m] * x[m];
      x[i] = v;
      A[(k0 + i) * lda + c] = v;
    }
  }
}

// C (M x Nc) -= A (M x K) B (K x Nc), K <= MX_NB; 128 x 128 tile per block,
// 256 threads, 8 x 8 outputs per thread; K staged through shared memory in
// slices of 32 (FP32) or 16 (FP64) to stay within 48 KB of static shared
// memory.
template <class T>
__global__ void __launch_bounds__(256)
    k_gemm_update(T* __restrict__ C, int64_t ldc, const T* __restrict__ A, int64_t lda, const T* __restrict__ B,
                  int64_t ldb, int64_t M, int64_t Nc, int K) {
  constexpr int BK = sizeof(T) == 4 ? 32 : 16;
  __shared__ T sA[BK][128 + 4];  // sA[k][row]
  __shared__ T sB[BK][128 + 4];  // sB[k][col]
  const int64_t row0 = blockIdx.y * 128, col0 = blockIdx.x * 128;
  const int t = threadIdx.x, tr = t / 16, tc = t % 16;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = T(0);
  for (int k0 = 0; k0 < K; k0 += BK) {
    const int kk = K - k0 < BK ? K - k0 : BK;
    __syncthreads();
    for (int e = t; e < 128 * BK; e += 256) {
      int r = e / BK, k = e % BK;
      int64_t gr = row0 + r;
      sA[k][r] = (gr < M && k < kk) ? A[gr * lda + k0 + k] : T(0);
    }
    for (int e = t; e < 128 * BK; e += 256) {
      int k = e / 128, cc = e % 128;
      int64_t gc = col0 + cc;
      sB[k][cc] = (gc < Nc && k < kk) ? B[(k0 + k) * ldb + gc] : T(0);
    }
    __syncthreads();
    for (int k = 0; k < kk; k++) {
      T a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = sA[k][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; j++) b[j] = sB[k][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int64_t gr = row0 + tr + 16 * i;
    if (gr >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      int64_t gc = col0 + tc + 16 * j;
      if (gc < Nc) C[gr * ldc + gc] -= acc[i][j];
    }
  }
}

// ---------------------------------------------------------------- mixed solve
// c[j] = 1 / max_i |A[i, j]| (one block of 8 warps per 32 columns, rows strided over the warps)
__global__ void k_col_maxabs(const double* __restrict__ A, int64_t lda, int64_t N, double* __restrict__ c) {
  __shared__ double red[8][32];
  int64_t j = blockIdx.x * 32 + (threadIdx.x & 31);
  int w = threadIdx.x / 32;
  double m = 0.0;
  if (j < N)
    for (int64_t i = w; i < N; i += 8) m = fmax(m, fabs(A[i * lda + j]));
  red[w][threadIdx.x & 31] = m;
  __syncthreads();
  if (w == 0 && j < N) {
    for (int k = 1; k < 8; k++) m = fmax(m, red[k][threadIdx.x & 31]);
    c[j] = m > 0 ? 1.0 / m : 1.0;
  }
}

// S (float) = A diag(c)
__global__ void k_scale_to_f32(const double* __restrict__ A, int64_t lda, const double* __restrict__ c,
                               float* __restrict__ S, int64_t N) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= N * N) return;
  int64_t i = g / N, j = g % N;
  S[g] = float(A[i * lda + j] * c[j]);
}

// R[r, i] = F[r, i] - sum_j A[i, j] X[r, j]; one warp per row i, all right-hand
// sides at once (A read once; nrhs <= 16).
constexpr int MX_MAX_RHS = 16;
__global__ void k_residual(const double* __restrict__ A, int64_t lda, const double* __restrict__ X,
                           const double* __restrict__ F, double* __restrict__ R, int64_t N, int nrhs) {
  int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
  int lane = threadIdx.x & 31;
  if (i >= N) return;
  double acc[MX_MAX_RHS];
#pragma unroll
  for (int r = 0; r < MX_MAX_RHS; r++) acc[r] = 0.0;
  const double* row = A + i * lda;
  for (int64_t j = lane; j < N; j += 32) {
    double a = row[j];
#pragma unroll
    for (int r = 0; r < MX_MAX_RHS; r++)
      if (r < nrhs) acc[r] = fma(a, X[r * N + j], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < MX_MAX_RHS; r++) {
    if (r < nrhs) {
      double v = warp_sum(acc[r]);
      if (lane == 0) R[r * N + i] = F[r * N + i] - v;
    }
  }
}

// Triangular solves with FP32 factors and FP64 right-hand sides (the
// correction equation of the refinement), blocked like tb_lu_solve_perm.
template <bool LOWER>
__global__ void k_trsv_block_f32(const float* __restrict__ LU, int64_t lda, double* __restrict__ X, int64_t N,
                                 int64_t b0, int nb, int nrhs) {
  __shared__ double Tm[MX_NB][MX_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) Tm[e / nb][e % nb] = LU[(b0 + e / nb) * lda + b0 + e % nb];
  __syncthreads();
  int r = threadIdx.x;
  if (r >= nrhs) return;
  double* x = X + r * N + b0;
  if (LOWER) {
    for (int i = 0; i < nb; i++) {
      double v = x[i];
      for (int m = 0; m < i; m++) v = fma(-Tm[i][m], x[m], v);
      x[i] = v;
    }
  } else {
    for (int i = nb - 1; i >= 0; i--) {
      double v = x[i];
      for (int m = i + 1; m < nb; m++) v = fma(-Tm[i][m], x[m], v);
      x[i] = v / Tm[i][i];
    }
  }
}

__global__ void k_trsv_update_f32(const float* __restrict__ LU, int64_t lda, double* __restrict__ X, int64_t N,
                                  int64_t b0, int nb, int64_t i0, int64_t i1, int nrhs) {
  __shared__ double xs[MX_MAX_RHS][MX_NB];
  for (int e = threadIdx.x; e < nrhs * nb; e += blockDim.x) xs[e / nb][e % nb] = X[(e / nb) * N + b0 + e % nb];
  __syncthreads();
  int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= i1) return;
  const float* row = LU + i * lda + b0;
  double acc[MX_MAX_RHS];
#pragma unroll
  for (int r = 0; r < MX_MAX_RHS; r++) acc[r] = 0.0;
  for (int m = 0; m < nb; m++) {
    double l = row[m];
#pragma unroll
    for (int r = 0; r < MX_MAX_RHS; r++)
      if (r < nrhs) acc[r] = fma(l, xs[r][m], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < MX_MAX_RHS; r++)
    if (r < nrhs) X[r * N + i] -= acc[r];
}

// X[r, j] += c[j] D[r, j]; also the largest |c D| / |X| over all entries
// (bits of a non-negative double compare like integers).
__global__ void k_apply_correction(double* __restrict__ X, const double* __restrict__ D, const double* __restrict__ c,
                                   int64_t N, int nrhs, unsigned long long* __restrict__ maxes) {
  // maxes[2 r] = max_j |correction|, maxes[2 r + 1] = max_j |x| of right-hand side r
  // (non-negative doubles order like their bit patterns)
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= N * nrhs) return;
  int64_t j = g % N, r = g / N;
  double d = c[j] * D[g];
  double x = X[g] + d;
  X[g] = x;
  double ad = fabs(d), ax = fabs(x);
  if (!(ad == ad) || !(ax == ax)) ad = 1e300;
  atomicMax(&maxes[2 * r], (unsigned long long)__double_as_longlong(ad));
  atomicMax(&maxes[2 * r + 1], (unsigned long long)__double_as_longlong(ax));
}

template <class T>
static int lu_nopiv(T* A, int64_t lda, int64_t N, cudaStream_t s) {
  for (int64_t k0 = 0; k0 < N; k0 += MX_NB) {
    int nb = N - k0 < MX_NB ? int(N - k0) : MX_NB;
    k_diag_lu<T><<<1, 256, 0, s>>>(A, lda, k0, nb);
    int64_t rest = N - k0 - nb;
    if (rest > 0) {
      unsigned g = unsigned((rest + 127) / 128);
      k_trsm_right<T><<<g, 128, 0, s>>>(A, lda, N, k0, nb);
      k_trsm_left<T><<<g, 128, 0, s>>>(A, lda, N, k0, nb);
      dim3 grid(unsigned((rest + 127) / 128), unsigned((rest + 127) / 128));
      k_gemm_update<T><<<grid, 256, 0, s>>>(A + (k0 + nb) * lda + k0 + nb, lda, A + (k0 + nb) * lda + k0, lda,
                                            A + k0 * lda + k0 + nb, lda, rest, rest, nb);
    }
  }
  return launch_status();
}

}  // namespace tb

using namespace tb;

extern "C" int tb_lu_nopiv_f64(double* A, int64_t lda, int64_t N, tb_stream_t stream) {
  if (N < 0 || lda < N || (N > 0 && !A) || N > 0x7fffffff) return BAD_ARG;
  if (N == 0) return OK;
  return lu_nopiv<double>(A, lda, N, (cudaStream_t)stream);
}

extern "C" int tb_lu_nopiv_f32(float* A, int64_t lda, int64_t N, tb_stream_t stream) {
  if (N < 0 || lda < N || (N > 0 && !A) || N > 0x7fffffff) return BAD_ARG;
  if (N == 0) return OK;
  return lu_nopiv<float>(A, lda, N, (cudaStream_t)stream);
}

extern "C" int64_t tb_solve_mixed_workspace(int64_t N, int64_t nrhs) {
  if (N <= 0 || nrhs <= 0) return 0;
  // FP32 factors, column scales, correction / residual block, 2 * nrhs maxima
  return N * N * 4 + 256 + N * 8 + 256 + nrhs * N * 8 + 256 + 256;
}

extern "C" int tb_solve_mixed(const double* A, int64_t lda, int64_t N, const double* F, double* X, int64_t nrhs,
                              void* work, int64_t work_bytes, int max_iter, double tol, int* iters_out,
                              double* last_rel_out, tb_stream_t stream) {
  if (N <= 0 || nrhs <= 0 || nrhs > MX_MAX_RHS || lda < N || !A || !F || !X || !work || max_iter < 1)
    return BAD_ARG;
  if (work_bytes < tb_solve_mixed_workspace(N, nrhs)) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  char* w = static_cast<char*>(work);
  float* S = reinterpret_cast<float*>(w);
  w += ((N * N * 4 + 255) / 256) * 256;
  double* c = reinterpret_cast<double*>(w);
  w += ((N * 8 + 255) / 256) * 256;
  double* D = reinterpret_cast<double*>(w);
  w += ((nrhs * N * 8 + 255) / 256) * 256;
  unsigned long long* maxes = reinterpret_cast<unsigned long long*>(w);

  k_col_maxabs<<<unsigned((N + 31) / 32), 256, 0, s>>>(A, lda, N, c);
  k_scale_to_f32<<<unsigned((N * N + 255) / 256), 256, 0, s>>>(A, lda, c, S, N);
  int st = lu_nopiv<float>(S, N, N, s);
  if (st != OK) return st;
  if (cudaMemsetAsync(X, 0, sizeof(double) * N * nrhs, s) != cudaSuccess) return CUDA_ERR;
  const int nr = int(nrhs);
  int it = 0;
  double rel = 1e300;
  for (it = 1; it <= max_iter; it++) {
    // D = F - A X (FP64), then D <- (L U)^-1 D with the FP32 factors
    k_residual<<<unsigned((N * 32 + 255) / 256), 256, 0, s>>>(A, lda, X, F, D, N, nr);
    for (int64_t b0 = 0; b0 < N; b0 += MX_NB) {
      int nb = N - b0 < MX_NB ? int(N - b0) : MX_NB;
      k_trsv_block_f32<true><<<1, 32, 0, s>>>(S, N, D, N, b0, nb, nr);
      int64_t i0 = b0 + nb;
      if (i0 < N) k_trsv_update_f32<<<unsigned((N - i0 + 127) / 128), 128, 0, s>>>(S, N, D, N, b0, nb, i0, N, nr);
    }
    for (int64_t b = (N + MX_NB - 1) / MX_NB - 1; b >= 0; b--) {
      int64_t b0 = b * MX_NB;
      int nb = N - b0 < MX_NB ? int(N - b0) : MX_NB;
      k_trsv_block_f32<false><<<1, 32, 0, s>>>(S, N, D, N, b0, nb, nr);
      if (b0 > 0) k_trsv_update_f32<<<unsigned((b0 + 127) / 128), 128, 0, s>>>(S, N, D, N, b0, nb, 0, b0, nr);
    }
    if (cudaMemsetAsync(maxes, 0, sizeof(unsigned long long) * 2 * nr, s) != cudaSuccess) return CUDA_ERR;
    k_apply_correction<<<unsigned((N * nrhs + 255) / 256), 256, 0, s>>>(X, D, c, N, nr, maxes);
    unsigned long long bits[2 * MX_MAX_RHS];
    if (cudaMemcpyAsync(bits, maxes, sizeof(unsigned long long) * 2 * nr, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return CUDA_ERR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CUDA_ERR;
    const double prev = rel;
    rel = 0.0;
    for (int r = 0; r < nr; r++) {
      double md, mx;
      std::memcpy(&md, &bits[2 * r], sizeof(md));
      std::memcpy(&mx, &bits[2 * r + 1], sizeof(mx));
      double q = md / (mx > 1e-300 ? mx : 1e-300);
      rel = (q > rel || !(q == q)) ? q : rel;
    }
    if (!(rel == rel) || rel > 1e200) {
      st = NONFINITE;
      break;
    }
    if (rel <= tol) break;
    // Corrections that stop shrinking just above tol have reached the FP64
    // rounding floor of the residual (about cond * 1e-16): converged.
    if (it >= 3 && rel <= 100.0 * tol && rel > 0.5 * prev) {
      rel = tol;
      break;
    }
  }
  if (iters_out) *iters_out = it > max_iter ? max_iter : it;
  if (last_rel_out) *last_rel_out = rel;
  if (st != OK) return st;
  if (rel > tol) return SINGULAR;  // did not converge: the caller falls back to the pivoted FP64 LU
  return launch_status();
}
