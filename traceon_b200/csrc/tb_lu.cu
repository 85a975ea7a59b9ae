// tb_lu.cu -- dense FP64 LU with partial pivoting and the triangular solves:
// the charge solve of traceon/solver.py:160-180 (numpy.linalg.solve, LAPACK
// dgesv) as a right-looking blocked factorisation.
//
// Per panel of LU_NB columns:
//   for each column k of the panel
//     k_lu_pivot   (1 block)  pivot search in column k, full-row swap, ipiv/perm
//     k_lu_column  (grid)     multipliers of column k and their update of the
//                             rest of the panel
//   k_lu_trsm     (grid)      U12 = L11^-1 A12
//   k_gemm_sub    (grid)      A22 -= L21 U12   (FP64 register-tiled GEMM)
#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

constexpr int LU_NB = 32;

// Pivot of column k: the first row of largest |A[r, k]|, r >= k (LAPACK
// idamax picks the first maximum).  Swaps rows k and p over all N columns.
__global__ void __launch_bounds__(1024)
    k_lu_pivot(double* __restrict__ A, int64_t lda, int64_t N, int64_t k, int32_t* __restrict__ ipiv,
               int32_t* __restrict__ perm) {
  __shared__ double s_v[32];
  __shared__ int64_t s_i[32];
  __shared__ int64_t s_p;
  double best = -1.0;
  int64_t bi = k;
  for (int64_t r = k + threadIdx.x; r < N; r += blockDim.x) {
    double v = fabs(A[r * lda + k]);
    if (v > best) {
      best = v;
      bi = r;
    }
  }
  // warp argmax, ties to the smaller row
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, best, o);
    int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) {
      best = ov;
      bi = oi;
    }
  }
  int w = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
    s_v[w] = best;
    s_i[w] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = -1.0;
    int64_t p = k;
    int nw = (blockDim.x + 31) / 32;
    for (int i = 0; i < nw; i++)
      if (s_v[i] > b || (s_v[i] == b && s_i[i] < p)) {
        b = s_v[i];
        p = s_i[i];
      }
    s_p = p;
    ipiv[k] = int32_t(p);
    if (perm && p != k) {
      int32_t t = perm[k];
      perm[k] = perm[p];
      perm[p] = t;
    }
  }
  __syncthreads();
  int64_t p = s_p;
  if (p != k) {
    for (int64_t c = threadIdx.x; c < N; c += blockDim.x) {
      double t = A[k * lda + c];
      A[k * lda + c] = A[p * lda + c];
      A[p * lda + c] = t;
    }
  }
}

// Rows r > k: l = A[r,k] / A[k,k], then A[r, k+1 .. kend) -= l A[k, k+1 .. kend).
__global__ void k_lu_column(double* __restrict__ A, int64_t lda, int64_t N, int64_t k, int64_t kend) {
  int64_t r = k + 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= N) return;
  const double* pr = A + k * lda;
  double l = A[r * lda + k] / pr[k];
  double* row = A + r * lda;
  row[k] = l;
  for (int64_t c = k + 1; c < kend; c++) row[c] = fma(-l, pr[c], row[c]);
}

// U12 = L11^-1 A12, L11 unit lower (nb x nb at (k0, k0)); one thread per column.
__global__ void k_lu_trsm(double* __restrict__ A, int64_t lda, int64_t N, int64_t k0, int nb) {
  __shared__ double L[LU_NB][LU_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e / nb, j = e % nb;
    L[i][j] = A[(k0 + i) * lda + k0 + j];
  }
  __syncthreads();
  int64_t c = k0 + nb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  double x[LU_NB];
#pragma unroll
  for (int i = 0; i < LU_NB; i++) {
    if (i < nb) {
      double v = A[(k0 + i) * lda + c];
      for (int m = 0; m < i; m++) v = fma(-L[i][m], x[m], v);
      x[i] = v;
      A[(k0 + i) * lda + c] = v;
    }
  }
}

// C (M x Nc, ldc) -= Am (M x K, lda) * B (K x Nc, ldb), K <= LU_NB.
// 64 x 64 output tile per block, 256 threads, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256)
    k_gemm_sub(double* __restrict__ C, int64_t ldc, const double* __restrict__ Am, int64_t lda,
               const double* __restrict__ B, int64_t ldb, int64_t M, int64_t Nc, int K) {
  __shared__ double sA[LU_NB][64 + 1];  // transposed: sA[k][row]
  __shared__ double sB[LU_NB][64 + 1];  // sB[k][col]
  const int64_t row0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
  const int t = threadIdx.x;
  for (int e = t; e < 64 * K; e += 256) {
    int rr = e / K, kk = e % K;
    int64_t gr = row0 + rr;
    sA[kk][rr] = gr < M ? Am[gr * lda + kk] : 0.0;
  }
  for (int e = t; e < 64 * K; e += 256) {
    int kk = e / 64, cc = e % 64;
    int64_t gc = col0 + cc;
    sB[kk][cc] = gc < Nc ? B[kk * ldb + gc] : 0.0;
  }
  __syncthreads();
  const int tr = t / 16, tc = t % 16;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  for (int kk = 0; kk < K; kk++) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; i++) a[i] = sA[kk][tr + 16 * i];
#pragma unroll
    for (int j = 0; j < 4; j++) b[j] = sB[kk][tc + 16 * j];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int64_t gr = row0 + tr + 16 * i;
    if (gr >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int64_t gc = col0 + tc + 16 * j;
      if (gc < Nc) C[gr * ldc + gc] -= acc[i][j];
    }
  }
}

__global__ void k_iota(int32_t* __restrict__ p, int64_t N) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < N) p[i] = int32_t(i);
}

// ------------------------------------------------------------- solve
// X (nrhs, N) = F gathered by the row permutation: X[r, i] = F[r, perm[i]].
__global__ void k_gather_rhs(const double* __restrict__ F, int64_t ldf, const int32_t* __restrict__ perm,
                             double* __restrict__ X, int64_t ldx, int64_t N, int64_t nrhs) {
  int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= N * nrhs) return;
  int64_t r = g / N, i = g % N;
  X[r * ldx + i] = F[r * ldf + perm[i]];
}

// Diagonal block of the forward (lower, unit) or backward (upper) solve for
// all right-hand sides: one thread per right-hand side, block rows in smem.
constexpr int TS_NB = 64;
template <bool LOWER>
__global__ void k_trsv_block(const double* __restrict__ LU, int64_t lda, double* __restrict__ X, int64_t ldx,
                             int64_t b0, int nb, int64_t nrhs) {
  __shared__ double T[TS_NB][TS_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e / nb, j = e % nb;
    T[i][j] = LU[(b0 + i) * lda + b0 + j];
  }
  __syncthreads();
  int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  double* x = X + r * ldx + b0;
  if (LOWER) {
    for (int i = 0; i < nb; i++) {
      double v = x[i];
      for (int m = 0; m < i; m++) v = fma(-T[i][m], x[m], v);
      x[i] = v;
    }
  } else {
    for (int i = nb - 1; i >= 0; i--) {
      double v = x[i];
      for (int m = i + 1; m < nb; m++) v = fma(-T[i][m], x[m], v);
      x[i] = v / T[i][i];
    }
  }
}

// X[r, i] -= sum_m LU[i, b0 + m] X[r, b0 + m] for rows i in [i0, i1):
// one thread per (rhs, row); rows of the panel read once per rhs.
__global__ void k_trsv_update(const double* __restrict__ LU, int64_t lda, double* __restrict__ X, int64_t ldx,
                              int64_t b0, int nb, int64_t i0, int64_t i1, int64_t nrhs) {
  __shared__ double xs[8][TS_NB];
  int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t rbase = blockIdx.y * 8;
  for (int e = threadIdx.x; e < 8 * nb; e += blockDim.x) {
    int rr = e / nb, m = e % nb;
    xs[rr][m] = (rbase + rr < nrhs) ? X[(rbase + rr) * ldx + b0 + m] : 0.0;
  }
  __syncthreads();
  if (i >= i1) return;
  const double* row = LU + i * lda + b0;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int m = 0; m < nb; m++) {
    double l = row[m];
#pragma unroll
    for (int rr = 0; rr < 8; rr++) acc[rr] = fma(l, xs[rr][m], acc[rr]);
  }
#pragma unroll
  for (int rr = 0; rr < 8; rr++)
    if (rbase + rr < nrhs) X[(rbase + rr) * ldx + i] -= acc[rr];
}

}  // namespace tb

using namespace tb;

extern "C" int tb_lu_factor_perm(double* A, int64_t lda, int32_t* ipiv, int32_t* perm, int64_t N,
                                 tb_stream_t stream) {
  if (N < 0 || lda < N || (N > 0 && (!A || !ipiv))) return BAD_ARG;
  if (N == 0) return OK;
  if (N > 0x7fffffff) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (perm) k_iota<<<unsigned((N + 255) / 256), 256, 0, s>>>(perm, N);
  for (int64_t k0 = 0; k0 < N; k0 += LU_NB) {
    int nb = N - k0 < LU_NB ? int(N - k0) : LU_NB;
    int64_t kend = k0 + nb;
    for (int64_t k = k0; k < kend; k++) {
      k_lu_pivot<<<1, 1024, 0, s>>>(A, lda, N, k, ipiv, perm);
      int64_t rows = N - k - 1;
      if (rows > 0) k_lu_column<<<unsigned((rows + 127) / 128), 128, 0, s>>>(A, lda, N, k, kend);
    }
    int64_t rest = N - kend;
    if (rest > 0) {
      k_lu_trsm<<<unsigned((rest + 127) / 128), 128, 0, s>>>(A, lda, N, k0, nb);
      dim3 g(unsigned((rest + 63) / 64), unsigned((rest + 63) / 64));
      k_gemm_sub<<<g, 256, 0, s>>>(A + kend * lda + kend, lda, A + kend * lda + k0, lda, A + k0 * lda + kend, lda,
                                   rest, rest, nb);
    }
    int st = launch_status();
    if (st != OK) return st;
  }
  return launch_status();
}

extern "C" int tb_lu_factor(double* A, int64_t lda, int32_t* ipiv, int64_t N, tb_stream_t stream) {
  return tb_lu_factor_perm(A, lda, ipiv, nullptr, N, stream);
}

extern "C" int tb_lu_solve_perm(const double* LU, int64_t lda, const int32_t* perm, int64_t N, const double* F,
                                int64_t ldf, double* X, int64_t ldx, int64_t nrhs, tb_stream_t stream) {
  if (N < 0 || nrhs < 0 || lda < N || ldf < N || ldx < N) return BAD_ARG;
  if (N == 0 || nrhs == 0) return OK;
  if (!LU || !perm || !F || !X || F == X) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int64_t tot = N * nrhs;
  k_gather_rhs<<<unsigned((tot + 255) / 256), 256, 0, s>>>(F, ldf, perm, X, ldx, N, nrhs);
  unsigned ry = unsigned((nrhs + 7) / 8);
  unsigned rb = unsigned((nrhs + 127) / 128);
  // forward: L y = P f
  for (int64_t b0 = 0; b0 < N; b0 += TS_NB) {
    int nb = N - b0 < TS_NB ? int(N - b0) : TS_NB;
    k_trsv_block<true><<<rb, 128, 0, s>>>(LU, lda, X, ldx, b0, nb, nrhs);
    int64_t i0 = b0 + nb;
    if (i0 < N) k_trsv_update<<<dim3(unsigned((N - i0 + 127) / 128), ry), 128, 0, s>>>(LU, lda, X, ldx, b0, nb, i0, N, nrhs);
  }
  // backward: U x = y
  int64_t nblk = (N + TS_NB - 1) / TS_NB;
  for (int64_t b = nblk - 1; b >= 0; b--) {
    int64_t b0 = b * TS_NB;
    int nb = N - b0 < TS_NB ? int(N - b0) : TS_NB;
    k_trsv_block<false><<<rb, 128, 0, s>>>(LU, lda, X, ldx, b0, nb, nrhs);
    if (b0 > 0) k_trsv_update<<<dim3(unsigned((b0 + 127) / 128), ry), 128, 0, s>>>(LU, lda, X, ldx, b0, nb, 0, b0, nrhs);
  }
  return launch_status();
}

// ============================================================================
// Dense solve that allocates nothing.
//
// For callers that cannot allocate device memory: a plug-in inside a host
// application that owns the GPU's memory pool, or a control loop that must
// not allocate after start-up (e.g. re-solving lens charges whenever the
// electrode voltages change).  The pivot steps and the row permutation of
// the factorisation live in this file-scope device array instead of caller
// or library allocations: every GPU that loads the library holds it
// (256 KiB) until the process exits, and it bounds N to NOALLOC_MAX_N.
// ============================================================================
#include <cuda.h>
#include <mutex>

namespace tb {
constexpr int64_t NOALLOC_MAX_N = 32768;
static __device__ __align__(256) int32_t g_lu_noalloc_scratch[2 * NOALLOC_MAX_N];

// Per device: the array's device address and the id of the CUDA context it
// was looked up in.  A device's address belongs to its context: after a
// cudaDeviceReset the next call runs in a new context and looks it up again.
struct NoallocSlot {
  unsigned long long ctx_id;
  int32_t* addr;
};
static std::mutex g_noalloc_mutex;
static NoallocSlot g_noalloc[64] = {};

// Id of the calling thread's current context, or 0 when there is none or the
// driver cannot tell (then the address is looked up on every call).  The two
// driver calls are fetched through the runtime, so the library does not link
// the driver library itself.
static unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}
}  // namespace tb

extern "C" int tb_lu_solve_noalloc(double* A, int64_t lda, int64_t N, const double* F, int64_t ldf, double* X,
                                   int64_t ldx, int64_t nrhs, tb_stream_t stream) {
  if (N < 0 || N > tb::NOALLOC_MAX_N) return tb::BAD_ARG;
  if (nrhs < 0 || lda < N || ldf < N || ldx < N) return tb::BAD_ARG;
  if (N == 0 || nrhs == 0) return tb::OK;
  if (!A || !F || !X || F == X) return tb::BAD_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return tb::CUDA_ERR;
  int32_t* scratch = nullptr;
  {
    // Once per device (and context), with that device current: the
    // host-side name of the array is not a device address, so look the
    // address up.
    std::lock_guard<std::mutex> lock(tb::g_noalloc_mutex);
    tb::NoallocSlot& slot = tb::g_noalloc[dev];
    const unsigned long long ctx = tb::current_context_id();
    if (!slot.addr || ctx == 0 || slot.ctx_id != ctx) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, tb::g_lu_noalloc_scratch) != cudaSuccess || !p) return tb::CUDA_ERR;
      slot.addr = static_cast<int32_t*>(p);
      slot.ctx_id = tb::current_context_id();  // the lookup made the device's context current
    }
    scratch = slot.addr;
  }
  int32_t* ipiv = scratch;
  int32_t* perm = scratch + tb::NOALLOC_MAX_N;  // reset to the identity by every factorisation
  int st = tb_lu_factor_perm(A, lda, ipiv, perm, N, stream);
  if (st != tb::OK) return st;
  return tb_lu_solve_perm(A, lda, perm, N, F, ldf, X, ldx, nrhs, stream);
}
