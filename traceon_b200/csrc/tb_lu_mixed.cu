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
// The mixed solve factors with lu_nopiv_f32_tc (256-column panels, trailing
// updates on the tensor cores, below; its kernels are launched as
// programmatic dependents of one another, see pdl_launch); tb_lu_nopiv_f32 /
// _f64 keep the plain one-level blocking.  Blocked right-looking factorisation, per panel of NB
// columns:
//   k_diag_lu      one CTA factors the NB x NB diagonal block in shared memory
//   k_trsm_right   L21 = A21 U11^-1   (one thread per row)
//   k_trsm_left    U12 = L11^-1 A12   (one thread per column)
//   k_gemm_update  A22 -= L21 U12     (register-tiled SIMT GEMM)
#include <cstdint>
#include <cstring>

#include <atomic>
#include <mutex>
#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "tb_tc.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

constexpr int MX_NB = 64;

// Programmatic dependent launch of the factorisation's kernels.  A kernel
// launched by pdl_launch may be scheduled while its predecessor in the
// stream is still finishing; it calls pdl_wait() before its first memory
// access, and that returns once the predecessor grid has completed and its
// writes are visible.  The data order of the stream is therefore unchanged;
// only the gap between dependent launches is overlapped.  In a launch
// without the attribute pdl_wait() returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
static void pdl_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);  // errors: launch_status() / cudaGetLastError
}

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

// columns c0 <= j < c1: A[k0:k0+nb, j] <- L11^-1 A[k0:k0+nb, j] (L11 unit lower)
template <class T>
__global__ void __launch_bounds__(128)
    k_trsm_left(T* __restrict__ A, int64_t lda, int64_t c0, int64_t c1, int64_t k0, int nb) {
  __shared__ T L[MX_NB][MX_NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) L[e / nb][e % nb] = A[(k0 + e / nb) * lda + k0 + e % nb];
  __syncthreads();
  int64_t c = c0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= c1) return;
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

// ---------------------------------------------------------------- FP32 panel kernels
// Panel kernels of lu_nopiv_f32_tc (64-wide blocks).

// D (the nb x nb diagonal block at (k0, k0)) <- its LU factors in place.
// Thread t owns column j = t % 64 of rows t / 64 + 4 s (s = 0..15) in
// registers; at step k the owners publish column k and row k to shared
// memory (double-buffered by the parity of k: one barrier per step) and
// every thread updates its elements with the pivot's reciprocal.  Fully
// unrolled (k and s are constants in every iteration, so no dynamic
// register indexing).  Rows and columns beyond nb are the identity.
__global__ void __launch_bounds__(256) k_diag_lu_f32(float* __restrict__ A, int64_t lda, int64_t k0, int nb) {
  pdl_wait();
  __shared__ float colk[2][MX_NB], rowk[2][MX_NB];
  const int j = threadIdx.x % MX_NB, i0 = threadIdx.x / MX_NB;
  float v[16];
#pragma unroll
  for (int sI = 0; sI < 16; sI++) {
    const int i = i0 + 4 * sI;
    v[sI] = (i < nb && j < nb) ? A[(k0 + i) * lda + k0 + j] : (i == j ? 1.f : 0.f);
  }
#pragma unroll
  for (int k = 0; k < MX_NB - 1; k++) {
    if (k >= nb - 1) break;
    const int buf = k & 1;
    if (j == k) {
#pragma unroll
      for (int sI = 0; sI < 16; sI++) colk[buf][i0 + 4 * sI] = v[sI];
    }
    if (i0 == (k & 3)) rowk[buf][j] = v[k >> 2];
    __syncthreads();
    const float inv = 1.f / rowk[buf][k];
    const float u = rowk[buf][j];
#pragma unroll
    for (int sI = 0; sI < 16; sI++) {
      const int i = i0 + 4 * sI;
      if (i > k) {
        const float l = colk[buf][i] * inv;
        if (j == k)
          v[sI] = l;
        else if (j > k)
          v[sI] = fmaf(-l, u, v[sI]);
      }
    }
  }
#pragma unroll
  for (int sI = 0; sI < 16; sI++) {
    const int i = i0 + 4 * sI;
    if (i < nb && j < nb) A[(k0 + i) * lda + k0 + j] = v[sI];
  }
}

// Forward substitution on the 64-long vectors V[.][t] (one per thread, in
// shared memory, V[m][t] = element m): x_i = (v_i - sum_{p < i} C[p][i] x_p)
// times C[i][i] when DIAG (the caller stores the reciprocal pivots on the
// diagonal of C), unit diagonal otherwise.  Blocked by 8: the 8 unknowns of
// a block stay in registers while every finished unknown p < block is
// applied to all 8 (two 16-byte broadcast reads of C per p), then the block
// is solved in registers.
constexpr int TRSM_COLS = 128;
template <bool DIAG>
__device__ __forceinline__ void solve_vectors(float (*V)[TRSM_COLS], const float (*C)[MX_NB], int t) {
#pragma unroll 1
  for (int b0 = 0; b0 < MX_NB; b0 += 8) {
    float x[8];
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = V[b0 + c][t];
#pragma unroll 4
    for (int p = 0; p < b0; p++) {
      const float xp = V[p][t];
      const float4 c0 = *reinterpret_cast<const float4*>(&C[p][b0]);
      const float4 c1 = *reinterpret_cast<const float4*>(&C[p][b0 + 4]);
      x[0] = fmaf(-c0.x, xp, x[0]);
      x[1] = fmaf(-c0.y, xp, x[1]);
      x[2] = fmaf(-c0.z, xp, x[2]);
      x[3] = fmaf(-c0.w, xp, x[3]);
      x[4] = fmaf(-c1.x, xp, x[4]);
      x[5] = fmaf(-c1.y, xp, x[5]);
      x[6] = fmaf(-c1.z, xp, x[6]);
      x[7] = fmaf(-c1.w, xp, x[7]);
    }
#pragma unroll
    for (int c = 0; c < 8; c++) {
#pragma unroll
      for (int q = 0; q < c; q++) x[c] = fmaf(-C[b0 + q][b0 + c], x[q], x[c]);
      if (DIAG) x[c] *= C[b0 + c][b0 + c];
      V[b0 + c][t] = x[c];
    }
  }
}

// rows r0 <= i < r1: A[i, k0:k0+nb] <- A[i, k0:k0+nb] U11^-1.  x U = a is
// x_m = (a_m - sum_{p < m} x_p U[p][m]) / U[m][m]: solve_vectors with
// C = U (row-major, as stored; reciprocal pivots on its diagonal).  128 rows
// per CTA (thread = row), staged through shared memory (48 KB in all); all
// loads of a thread are issued before the first use (one memory latency).
__global__ void __launch_bounds__(TRSM_COLS)
    k_trsm_right_f32(float* __restrict__ A, int64_t lda, int64_t r0, int64_t r1, int64_t k0, int nb) {
  pdl_wait();
  __shared__ __align__(16) float U[MX_NB][MX_NB];
  __shared__ float V[MX_NB][TRSM_COLS];  // V[m][r]: element m of row r of the CTA
  const int64_t rb = r0 + blockIdx.x * (int64_t)TRSM_COLS;
  const int nrow = r1 - rb < TRSM_COLS ? int(r1 - rb) : TRSM_COLS;
  const int r = threadIdx.x;  // lanes over rows: conflict-free shared stores
  const bool vec = nb == MX_NB && lda % 4 == 0 && k0 % 4 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0;
  float* arow = A + (rb + r) * lda + k0;
  {
    float a[MX_NB];
    if (vec && r < nrow) {
#pragma unroll
      for (int q = 0; q < MX_NB / 4; q++) {
        const float4 f = *reinterpret_cast<const float4*>(arow + 4 * q);
        a[4 * q] = f.x;
        a[4 * q + 1] = f.y;
        a[4 * q + 2] = f.z;
        a[4 * q + 3] = f.w;
      }
    } else {
#pragma unroll
      for (int m = 0; m < MX_NB; m++) a[m] = (r < nrow && m < nb) ? arow[m] : 0.f;
    }
    float u[MX_NB * MX_NB / TRSM_COLS];
#pragma unroll
    for (int q = 0; q < MX_NB * MX_NB / TRSM_COLS; q++) {
      const int e = threadIdx.x + TRSM_COLS * q, m = e / MX_NB, jj = e % MX_NB;
      u[q] = (m < nb && jj < nb) ? A[(k0 + m) * lda + k0 + jj] : 0.f;
    }
#pragma unroll
    for (int m = 0; m < MX_NB; m++) V[m][r] = a[m];
#pragma unroll
    for (int q = 0; q < MX_NB * MX_NB / TRSM_COLS; q++) {
      const int e = threadIdx.x + TRSM_COLS * q, m = e / MX_NB, jj = e % MX_NB;
      U[m][jj] = m == jj ? (m < nb ? __frcp_rn(u[q]) : 1.f) : u[q];
    }
  }
  __syncthreads();
  solve_vectors<true>(V, U, r);
  if (r < nrow) {
    if (vec) {
#pragma unroll
      for (int q = 0; q < MX_NB / 4; q++)
        *reinterpret_cast<float4*>(arow + 4 * q) =
            make_float4(V[4 * q][r], V[4 * q + 1][r], V[4 * q + 2][r], V[4 * q + 3][r]);
    } else {
      for (int m = 0; m < nb; m++) arow[m] = V[m][r];
    }
  }
}

// columns c0 <= c < c1: A[k0:k0+nb, c] <- L11^-1 A[k0:k0+nb, c] (L11 unit
// lower): x_i = a_i - sum_{m < i} L[i][m] x_m, solve_vectors with
// C[m][i] = L[i][m] (L transposed into shared memory).  128 columns per CTA;
// all loads of a thread are issued before the first use.
__global__ void __launch_bounds__(TRSM_COLS)
    k_trsm_left_f32(float* __restrict__ A, int64_t lda, int64_t c0, int64_t c1, int64_t k0, int nb) {
  pdl_wait();
  __shared__ __align__(16) float Lt[MX_NB][MX_NB];
  __shared__ float V[MX_NB][TRSM_COLS];  // V[i][c]: row i of column c of the CTA
  const int64_t cb = c0 + blockIdx.x * (int64_t)TRSM_COLS;
  const int ncol = c1 - cb < TRSM_COLS ? int(c1 - cb) : TRSM_COLS;
  {
    float a[MX_NB], l[MX_NB * MX_NB / TRSM_COLS];
#pragma unroll
    for (int ii = 0; ii < MX_NB; ii++)
      a[ii] = (ii < nb && threadIdx.x < ncol) ? A[(k0 + ii) * lda + cb + threadIdx.x] : 0.f;
#pragma unroll
    for (int q = 0; q < MX_NB * MX_NB / TRSM_COLS; q++) {
      const int e = threadIdx.x + TRSM_COLS * q, m = e / MX_NB, ii = e % MX_NB;  // lanes over ii
      l[q] = (ii < nb && m < nb && m < ii) ? A[(k0 + ii) * lda + k0 + m] : 0.f;
    }
#pragma unroll
    for (int ii = 0; ii < MX_NB; ii++) V[ii][threadIdx.x] = a[ii];
#pragma unroll
    for (int q = 0; q < MX_NB * MX_NB / TRSM_COLS; q++) {
      const int e = threadIdx.x + TRSM_COLS * q;
      Lt[e / MX_NB][e % MX_NB] = l[q];
    }
  }
  __syncthreads();
  solve_vectors<false>(V, Lt, threadIdx.x);
  for (int ii = 0; ii < nb; ii++)
    if (threadIdx.x < ncol) A[(k0 + ii) * lda + cb + threadIdx.x] = V[ii][threadIdx.x];
}

// ---------------------------------------------------------------- tensor cores
// C (M x Nc, ldc) -= A (M x K, lda) . B (K x Nc, ldb), FP32 row-major, on
// the 5th-generation tensor cores (tcgen05.mma kind::tf32) with 3xTF32:
// every operand is split into a TF32 head (cvt.rna.tf32) and the FP32 tail
// x - head, and head.head + head.tail + tail.head is accumulated in FP32 in
// tensor memory -- about FP32 accuracy at tensor-core speed.  CTA tile
// 128 x 256 (TMEM: 256 FP32 columns), K in chunks of 32 (one SWIZZLE_128B
// atom of FP32 per row), staged by all 256 threads into two buffers so that
// the staging of chunk k + 1 overlaps the MMAs of chunk k.  B is staged
// transposed (N rows x K), so both operands are K-major.
constexpr int GT_M = 128, GT_N = 256, GT_K = 32, GT_THREADS = 256;

struct GemmSmem {
  uint8_t a_hi[2][GT_M * 128];
  uint8_t a_lo[2][GT_M * 128];
  uint8_t b_hi[2][GT_N * 128];
  uint8_t b_lo[2][GT_N * 128];
  uint64_t mbar[2];
  uint32_t tmem_base;
};
constexpr int GT_SMEM_BYTES = int(sizeof(GemmSmem)) + 1024;

__device__ __forceinline__ void split_tf32(float v, float& hi, float& lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
  hi = __uint_as_float(h);
  lo = v - hi;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Global -> register staging of one K chunk (prefetched while the previous
// chunk's MMAs run).  A: 128 rows x 32 k, item (row r = i / 8, k-quad i % 8):
// the 8 lanes of a row read its 128 contiguous bytes.  B: 32 k x 256 n, thread
// t owns column n = t, all 8 k-quads: each load is coalesced along n.
template <bool VEC>
__device__ __forceinline__ void gt_load(const float* __restrict__ A, int64_t lda, const float* __restrict__ B,
                                        int64_t ldb, int64_t M, int64_t Nc, int K, int64_t m0, int64_t n0, int k0,
                                        float (&ra)[16], float (&rb)[32]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int it = tid + GT_THREADS * j, r = it >> 3, kq = it & 7;
    const int64_t gr = m0 + r;
    const int k = k0 + 4 * kq;
    if (VEC && gr < M && k + 3 < K) {
      const float4 v = *reinterpret_cast<const float4*>(A + gr * lda + k);
      ra[4 * j] = v.x;
      ra[4 * j + 1] = v.y;
      ra[4 * j + 2] = v.z;
      ra[4 * j + 3] = v.w;
    } else {
#pragma unroll
      for (int u = 0; u < 4; u++) ra[4 * j + u] = (gr < M && k + u < K) ? A[gr * lda + k + u] : 0.f;
    }
  }
  const int64_t gn = n0 + tid;
#pragma unroll
  for (int kq = 0; kq < 8; kq++)
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = k0 + 4 * kq + u;
      rb[4 * kq + u] = (k < K && gn < Nc) ? B[(int64_t)k * ldb + gn] : 0.f;
    }
}

// Registers -> shared memory (TF32 head and tail), 16-byte swizzled stores:
// eight consecutive lanes write eight different chunk positions, no bank
// conflicts.
__device__ __forceinline__ void gt_store(uint32_t ah, uint32_t al, uint32_t bh, uint32_t bl, const float (&ra)[16],
                                         const float (&rb)[32]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int it = tid + GT_THREADS * j, r = it >> 3, kq = it & 7;
    float h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; u++) split_tf32(ra[4 * j + u], h[u], l[u]);
    const uint32_t off = tc::sw128(r, kq);
    tc::st_shared_v4(ah + off, __float_as_uint(h[0]), __float_as_uint(h[1]), __float_as_uint(h[2]),
                     __float_as_uint(h[3]));
    tc::st_shared_v4(al + off, __float_as_uint(l[0]), __float_as_uint(l[1]), __float_as_uint(l[2]),
                     __float_as_uint(l[3]));
  }
#pragma unroll
  for (int kq = 0; kq < 8; kq++) {
    float h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; u++) split_tf32(rb[4 * kq + u], h[u], l[u]);
    const uint32_t off = tc::sw128(tid, kq);
    tc::st_shared_v4(bh + off, __float_as_uint(h[0]), __float_as_uint(h[1]), __float_as_uint(h[2]),
                     __float_as_uint(h[3]));
    tc::st_shared_v4(bl + off, __float_as_uint(l[0]), __float_as_uint(l[1]), __float_as_uint(l[2]),
                     __float_as_uint(l[3]));
  }
}

template <bool VEC>
__global__ void __launch_bounds__(GT_THREADS, 1)
    k_gemm_sub_tf32x3(float* __restrict__ C, int64_t ldc, const float* __restrict__ A, int64_t lda,
                      const float* __restrict__ B, int64_t ldb, int64_t M, int64_t Nc, int K, int* __restrict__ err,
                      long long wait_cycles) {
  extern __shared__ __align__(1024) unsigned char gt_raw[];
  pdl_wait();
  const uint32_t raw = tc::smem_u32(gt_raw);
  GemmSmem& sm = *reinterpret_cast<GemmSmem*>(gt_raw + (((raw + 1023u) & ~1023u) - raw));
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int64_t m0 = (int64_t)blockIdx.y * GT_M, n0 = (int64_t)blockIdx.x * GT_N;
  if (tid < 2) tc::mbar_init(&sm.mbar[tid], 1);
  if (tid == 0) tc::fence_mbar_init();
  if (warp == 0) {
    tc::tmem_alloc(&sm.tmem_base, GT_N);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t dtm = sm.tmem_base;
  // kind::tf32: A, B TF32 (format 2), D FP32, K-major, M = 128, N = 256
  constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(GT_N >> 3) << 17) |
                             (uint32_t(GT_M >> 4) << 24);
  const int nk = (K + GT_K - 1) / GT_K;
  bool ok = true;
  int committed = 0;  // chunks whose MMAs were committed (uniform over the CTA)
  float ra[16], rb[32];
  gt_load<VEC>(A, lda, B, ldb, M, Nc, K, m0, n0, 0, ra, rb);
  for (int kc = 0; kc < nk; kc++) {
    const int b = kc & 1;
    if (kc >= 2) {  // the MMAs of chunk kc - 2 read buffer b
      const bool w = tc::mbar_wait_warp(&sm.mbar[b], uint32_t((kc - 2) >> 1) & 1u, wait_cycles);
      if (__syncthreads_or(!w)) {
        ok = false;
        break;
      }
    }
    const uint32_t ah = tc::smem_u32(sm.a_hi[b]), al = tc::smem_u32(sm.a_lo[b]);
    const uint32_t bh = tc::smem_u32(sm.b_hi[b]), bl = tc::smem_u32(sm.b_lo[b]);
    gt_store(ah, al, bh, bl, ra, rb);
    if (kc + 1 < nk) gt_load<VEC>(A, lda, B, ldb, M, Nc, K, m0, n0, (kc + 1) * GT_K, ra, rb);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < GT_K / 8; ks++) {  // K = 8 (32 bytes) per instruction
        const uint64_t dah = tc::desc_sw128(ah + 32 * ks), dal = tc::desc_sw128(al + 32 * ks);
        const uint64_t dbh = tc::desc_sw128(bh + 32 * ks), dbl = tc::desc_sw128(bl + 32 * ks);
        mma_tf32(dtm, dal, dbh, IDESC, (kc > 0 || ks > 0) ? 1u : 0u);
        mma_tf32(dtm, dah, dbl, IDESC, 1u);
        mma_tf32(dtm, dah, dbh, IDESC, 1u);
      }
      tc::mma_commit(&sm.mbar[b]);
    }
    committed = kc + 1;
  }
  if (ok && nk > 0) {
    const int bl = (nk - 1) & 1;
    const bool w = tc::mbar_wait_warp(&sm.mbar[bl], uint32_t((nk - 1) >> 1) & 1u, wait_cycles);
    ok = !__syncthreads_or(!w);
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // the committed MMAs must have finished before TMEM is freed
      if (committed > 0)
        tc::mbar_wait_bounded(&sm.mbar[(committed - 1) & 1], uint32_t((committed - 1) >> 1) & 1u,
                              DRAIN_WAIT_CYCLES);
    }
  } else if (nk > 0) {
    tc::fence_after_sync();
    // warp w: TMEM lanes 32 (w % 4) .. (rows), columns 128 (w / 4) ..
    const int row = 32 * (warp % 4) + lane;
    const int64_t gr = m0 + row;
    const uint32_t tbase = dtm + (uint32_t(32 * (warp % 4)) << 16) + uint32_t(128 * (warp / 4));
#pragma unroll 1
    for (int c = 0; c < 8; c++) {
      uint32_t v[16];
      tc::tmem_ld16(tbase + 16 * c, v);
      tc::tmem_wait_ld();
      const int64_t col0 = n0 + 128 * (warp / 4) + 16 * c;
      if (gr < M && col0 < Nc) {
        float* crow = C + gr * ldc + col0;
        if (VEC && col0 + 16 <= Nc) {
#pragma unroll
          for (int q = 0; q < 4; q++) {
            float4 x = *reinterpret_cast<float4*>(crow + 4 * q);
            x.x -= __uint_as_float(v[4 * q]);
            x.y -= __uint_as_float(v[4 * q + 1]);
            x.z -= __uint_as_float(v[4 * q + 2]);
            x.w -= __uint_as_float(v[4 * q + 3]);
            *reinterpret_cast<float4*>(crow + 4 * q) = x;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++)
            if (col0 + j < Nc) crow[j] -= __uint_as_float(v[j]);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(dtm, GT_N);
  }
}

static int gemm_sub_tf32x3(float* C, int64_t ldc, const float* A, int64_t lda, const float* B, int64_t ldb,
                           int64_t M, int64_t Nc, int K, int* err, cudaStream_t s) {
  if (M <= 0 || Nc <= 0 || K <= 0) return OK;
  if (cudaFuncSetAttribute(k_gemm_sub_tf32x3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, GT_SMEM_BYTES) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_gemm_sub_tf32x3<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, GT_SMEM_BYTES) !=
          cudaSuccess)
    return CUDA_ERR;
  dim3 grid(unsigned((Nc + GT_N - 1) / GT_N), unsigned((M + GT_M - 1) / GT_M));
  // 16-byte vector access of A rows and C rows when every row start is aligned
  const bool vec = (lda % 4 == 0) && (ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(C) % 16 == 0);
  if (vec)
    pdl_launch(k_gemm_sub_tf32x3<true>, grid, dim3(GT_THREADS), GT_SMEM_BYTES, s, C, ldc, A, lda, B, ldb, M, Nc, K,
               err, wait_limit());
  else
    pdl_launch(k_gemm_sub_tf32x3<false>, grid, dim3(GT_THREADS), GT_SMEM_BYTES, s, C, ldc, A, lda, B, ldb, M, Nc, K,
               err, wait_limit());
  return launch_status();
}

// ---------------------------------------------------------------- pre-split operands
// For the large updates the operands are split once, not per CTA: A (M x K)
// and B (K x N) FP32 become TF32 head / tail blocks already in the
// tensor-core operand layout -- A block (mb, kc) = [head atom | tail atom] of
// 128 rows x 32 k (16 KB each), B block (nb, kc) = [head | tail] of 256 rows
// (n) x 32 k (32 KB each); rows or k beyond the matrix are zero.  The GEMM
// below then moves whole blocks into shared memory with asynchronous bulk
// copies (cp.async.bulk, completion counted on an mbarrier).
constexpr uint32_t PA_BLOCK = 2u * GT_M * 128u;  // 32 KB
constexpr uint32_t PB_BLOCK = 2u * GT_N * 128u;  // 64 KB

__device__ __forceinline__ void st_global_v4(uint8_t* p, const float (&v)[4]) {
  *reinterpret_cast<uint4*>(p) =
      make_uint4(__float_as_uint(v[0]), __float_as_uint(v[1]), __float_as_uint(v[2]), __float_as_uint(v[3]));
}

__global__ void __launch_bounds__(256) k_split_a(const float* __restrict__ A, int64_t lda, int64_t M, int K,
                                                uint8_t* __restrict__ out) {
  pdl_wait();
  const int nk = (K + GT_K - 1) / GT_K;
  const int kc = blockIdx.x;
  const int64_t mb = blockIdx.y;
  uint8_t* blk = out + (mb * nk + kc) * (int64_t)PA_BLOCK;
  for (int it = threadIdx.x; it < GT_M * 8; it += blockDim.x) {
    const int r = it >> 3, kq = it & 7;
    const int64_t gr = mb * GT_M + r;
    const int k = kc * GT_K + 4 * kq;
    float h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; u++) split_tf32((gr < M && k + u < K) ? A[gr * lda + k + u] : 0.f, h[u], l[u]);
    st_global_v4(blk + tc::sw128(r, kq), h);
    st_global_v4(blk + GT_M * 128 + tc::sw128(r, kq), l);
  }
}

__global__ void __launch_bounds__(256) k_split_b(const float* __restrict__ B, int64_t ldb, int K, int64_t N,
                                                uint8_t* __restrict__ out) {
  pdl_wait();
  const int nk = (K + GT_K - 1) / GT_K;
  const int kc = blockIdx.x;
  const int64_t nb = blockIdx.y;
  uint8_t* blk = out + (nb * nk + kc) * (int64_t)PB_BLOCK;
  const int n = threadIdx.x;  // 256 threads: one column each, coalesced along n
  const int64_t gn = nb * GT_N + n;
#pragma unroll
  for (int kq = 0; kq < 8; kq++) {
    float h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = kc * GT_K + 4 * kq + u;
      split_tf32((k < K && gn < N) ? B[(int64_t)k * ldb + gn] : 0.f, h[u], l[u]);
    }
    st_global_v4(blk + tc::sw128(n, kq), h);
    st_global_v4(blk + GT_N * 128 + tc::sw128(n, kq), l);
  }
}

// C (M x Nc) -= A B from pre-split blocks, persistent: one CTA per SM walks
// the 128 x 256 tiles (t = blockIdx.x, + gridDim.x, ...) with two
// accumulators in tensor memory (512 columns), so the epilogue of one tile
// overlaps the MMAs of the next.  Warp 0 lane 0 streams the K chunks' blocks
// into two shared-memory stages with bulk copies (waiting for a stage to be
// released by the MMAs two chunks back), warp 1 lane 0 issues the 3 x 4 MMAs
// of each chunk (3xTF32) into accumulator t & 1 once the epilogue has
// released it (acc_empty), releases each stage with tcgen05.commit and
// signals the tile's end the same way (acc_full);
// warps 4..11 are the epilogue: warp w drains TMEM lanes 32 (w % 4).. and
// columns 128 ((w - 4) / 4).. of the tile into C.  Before waiting for an
// accumulator the epilogue warps prefetch their C rows into L2, so the
// read-modify-write of C mostly hits L2.  Every wait is bounded; a role
// whose wait runs out sets the failure flag and the others stop at their
// next wait.
constexpr int GQ_THREADS = 384;

struct GemmPersistSmem {
  uint8_t a[2][PA_BLOCK];
  uint8_t b[2][PB_BLOCK];
  uint64_t full[2], empty[2], acc_full[2], acc_empty[2];
  uint32_t tmem_base;
  int fail;
};
constexpr int GQ_SMEM_BYTES = int(sizeof(GemmPersistSmem)) + 1024;

__global__ void __launch_bounds__(GQ_THREADS, 1)
    k_gemm_sub_persist(float* __restrict__ C, int64_t ldc, const uint8_t* __restrict__ Apre,
                       const uint8_t* __restrict__ Bpre, int64_t M, int64_t Nc, int nk, int64_t nbn, int64_t ntiles,
                       int* __restrict__ err, long long wait_cycles) {
  extern __shared__ __align__(1024) unsigned char gq_raw[];
  pdl_wait();
  const uint32_t raw = tc::smem_u32(gq_raw);
  GemmPersistSmem& sm = *reinterpret_cast<GemmPersistSmem*>(gq_raw + (((raw + 1023u) & ~1023u) - raw));
  volatile int* fail = &sm.fail;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  if (tid < 2) {
    tc::mbar_init(&sm.full[tid], 1);
    tc::mbar_init(&sm.empty[tid], 1);
    tc::mbar_init(&sm.acc_full[tid], 1);
    tc::mbar_init(&sm.acc_empty[tid], 8);  // one arrive per epilogue warp
  }
  if (tid == 0) {
    sm.fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(&sm.tmem_base, 2 * GT_N);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t dtm = sm.tmem_base;
  constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(GT_N >> 3) << 17) |
                             (uint32_t(GT_M >> 4) << 24);
  int issued = 0;  // MMA chunks issued by this thread (warp 1 lane 0)
  int filled = 0;  // chunks whose copies this thread started (warp 0 lane 0)
  if (warp == 0) {
    if (lane == 0) {  // producer
      int it = 0;
      for (int64_t t = blockIdx.x; t < ntiles && !*fail; t += gridDim.x) {
        const uint8_t* Ab = Apre + (t / nbn) * nk * (int64_t)PA_BLOCK;
        const uint8_t* Bb = Bpre + (t % nbn) * nk * (int64_t)PB_BLOCK;
        for (int kc = 0; kc < nk; kc++, it++) {
          const int st = it & 1;
          if (it >= 2 && !tc::mbar_wait_bounded(&sm.empty[st], uint32_t((it - 2) >> 1) & 1u, wait_cycles)) {
            *fail = 1;
            break;
          }
          tc::mbar_arrive_expect_tx(&sm.full[st], PA_BLOCK + PB_BLOCK);
          const uint32_t da = tc::smem_u32(sm.a[st]), db = tc::smem_u32(sm.b[st]);
          for (uint32_t o = 0; o < PA_BLOCK; o += 16384u)
            tc::bulk_copy_g2s(da + o, Ab + kc * (int64_t)PA_BLOCK + o, 16384u, &sm.full[st]);
          for (uint32_t o = 0; o < PB_BLOCK; o += 16384u)
            tc::bulk_copy_g2s(db + o, Bb + kc * (int64_t)PB_BLOCK + o, 16384u, &sm.full[st]);
          filled = it + 1;
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int it = 0, tl = 0;
      for (int64_t t = blockIdx.x; t < ntiles && !*fail; t += gridDim.x, tl++) {
        const int buf = tl & 1;
        if (tl >= 2 && !tc::mbar_wait_bounded(&sm.acc_empty[buf], uint32_t((tl - 2) >> 1) & 1u, wait_cycles)) {
          *fail = 1;
          break;
        }
        tc::fence_after_sync();
        const uint32_t d = dtm + uint32_t(buf * GT_N);
        bool ok = true;
        for (int kc = 0; kc < nk; kc++, it++) {
          const int st = it & 1;
          if (!tc::mbar_wait_bounded(&sm.full[st], uint32_t(it >> 1) & 1u, wait_cycles)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t ah = tc::smem_u32(sm.a[st]), al = ah + GT_M * 128;
          const uint32_t bh = tc::smem_u32(sm.b[st]), bl = bh + GT_N * 128;
#pragma unroll
          for (int ks = 0; ks < GT_K / 8; ks++) {
            const uint64_t dah = tc::desc_sw128(ah + 32 * ks), dal = tc::desc_sw128(al + 32 * ks);
            const uint64_t dbh = tc::desc_sw128(bh + 32 * ks), dbl = tc::desc_sw128(bl + 32 * ks);
            mma_tf32(d, dal, dbh, IDESC, (kc > 0 || ks > 0) ? 1u : 0u);
            mma_tf32(d, dah, dbl, IDESC, 1u);
            mma_tf32(d, dah, dbh, IDESC, 1u);
          }
          tc::mma_commit(&sm.empty[st]);
          issued = it + 1;
        }
        if (!ok) {
          *fail = 1;
          break;
        }
        tc::mma_commit(&sm.acc_full[buf]);
      }
    }
    __syncwarp();
  } else if (warp >= 4) {  // epilogue
    const int quarter = warp % 4, half = (warp - 4) / 4;
    const int row = 32 * quarter + lane;
    const bool vec = (ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(C) % 16 == 0);
    int tl = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, tl++) {
      const int buf = tl & 1;
      const int64_t gr = (t / nbn) * GT_M + row;
      const int64_t c0 = (t % nbn) * GT_N + 128 * half;
      if (gr < M && c0 < Nc) {  // this thread's 128 columns of C, 4 lines of 128 bytes
        const float* crow = C + gr * ldc + c0;
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (c0 + 32 * q < Nc) asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + 32 * q));
      }
      const bool stop = __shfl_sync(0xffffffffu, *fail, 0) != 0;  // warp-uniform
      if (stop || !tc::mbar_wait_warp(&sm.acc_full[buf], uint32_t(tl >> 1) & 1u, wait_cycles)) {
        if (lane == 0) *fail = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t tbase = dtm + (uint32_t(32 * quarter) << 16) + uint32_t(buf * GT_N + 128 * half);
#pragma unroll 1
      for (int c = 0; c < 8; c++) {
        uint32_t v[16];
        tc::tmem_ld16(tbase + 16 * c, v);
        tc::tmem_wait_ld16(v);
        const int64_t col0 = c0 + 16 * c;
        if (gr < M && col0 < Nc) {
          float* crow = C + gr * ldc + col0;
          if (vec && col0 + 16 <= Nc) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
              float4 x = *reinterpret_cast<float4*>(crow + 4 * q);
              x.x -= __uint_as_float(v[4 * q]);
              x.y -= __uint_as_float(v[4 * q + 1]);
              x.z -= __uint_as_float(v[4 * q + 2]);
              x.w -= __uint_as_float(v[4 * q + 3]);
              *reinterpret_cast<float4*>(crow + 4 * q) = x;
            }
          } else {
#pragma unroll
            for (int j = 0; j < 16; j++)
              if (col0 + j < Nc) crow[j] -= __uint_as_float(v[j]);
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.acc_empty[buf]);
    }
  }
  // teardown: the MMAs issued and the copies started must have completed
  // before TMEM is freed and the CTA exits (after a failure too; all of
  // this has already happened on the normal path)
  if (warp == 1 && lane == 0 && issued > 0)
    tc::mbar_wait_bounded(&sm.empty[(issued - 1) & 1], uint32_t((issued - 1) >> 1) & 1u, DRAIN_WAIT_CYCLES);
  if (warp == 0 && lane == 0)
    for (int j = filled - 1; j >= 0 && j >= filled - 2; j--)
      tc::mbar_wait_bounded(&sm.full[j & 1], uint32_t(j >> 1) & 1u, DRAIN_WAIT_CYCLES);
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0 && sm.fail) atomicExch(err, 1);
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(dtm, 2 * GT_N);
  }
}

static int64_t round256(int64_t b) { return (b + 255) / 256 * 256; }

// Workspace of the pre-split GEMM for an M x N x K update.
static int64_t gemm_pre_bytes(int64_t M, int64_t N, int64_t K) {
  const int64_t nk = (K + GT_K - 1) / GT_K;
  return ((M + GT_M - 1) / GT_M) * nk * PA_BLOCK + ((N + GT_N - 1) / GT_N) * nk * PB_BLOCK;
}

static bool g_attr_gemm_pre[64];

static int gemm_pre_attr() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CUDA_ERR;
  if (dev >= 0 && dev < 64 && !g_attr_gemm_pre[dev]) {
    if (cudaFuncSetAttribute(k_gemm_sub_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, GQ_SMEM_BYTES) !=
        cudaSuccess)
      return CUDA_ERR;
    g_attr_gemm_pre[dev] = true;
  }
  return OK;
}

// Operands of C (M x Nc) -= A (M x K) B (K x Nc) split into TF32 head / tail
// blocks in `work` (A blocks first, then B blocks).
static void gemm_split(const float* A, int64_t lda, const float* B, int64_t ldb, int64_t M, int64_t Nc, int K,
                       uint8_t* work, cudaStream_t s) {
  const int nk = (K + GT_K - 1) / GT_K;
  const int64_t mbk = (M + GT_M - 1) / GT_M, nbk = (Nc + GT_N - 1) / GT_N;
  k_split_a<<<dim3(unsigned(nk), unsigned(mbk)), 256, 0, s>>>(A, lda, M, K, work);
  k_split_b<<<dim3(unsigned(nk), unsigned(nbk)), 256, 0, s>>>(B, ldb, K, Nc, work + mbk * nk * (int64_t)PA_BLOCK);
}

// The update from split operands, restricted to the row blocks [mb0, mb1)
// of 128 rows and the column blocks [nb0, nb1) of 256 columns, on at most
// max_ctas CTAs (0: one per SM).
static int gemm_persist_part(float* C, int64_t ldc, const uint8_t* work, int64_t M, int64_t Nc, int K, int64_t mb0,
                             int64_t mb1, int64_t nb0, int64_t nb1, int max_ctas, int* err, cudaStream_t s) {
  const int nk = (K + GT_K - 1) / GT_K;
  const int64_t mbk = (M + GT_M - 1) / GT_M;
  const int64_t nbk = (Nc + GT_N - 1) / GT_N;
  if (mb1 > mbk) mb1 = mbk;
  if (nb1 > nbk) nb1 = nbk;
  if (mb0 >= mb1 || nb0 >= nb1) return OK;
  const uint8_t* pa = work + mb0 * nk * (int64_t)PA_BLOCK;
  const uint8_t* pb = work + mbk * nk * (int64_t)PA_BLOCK + nb0 * nk * (int64_t)PB_BLOCK;
  const int64_t nrows = (mb1 == mbk ? M : mb1 * GT_M) - mb0 * GT_M;
  const int64_t ncols = (nb1 == nbk ? Nc : nb1 * GT_N) - nb0 * GT_N;
  const int64_t nbn = nb1 - nb0, ntiles = (mb1 - mb0) * nbn;
  int64_t grid = max_ctas > 0 && max_ctas < num_sms() ? max_ctas : num_sms();
  if (grid > ntiles) grid = ntiles;
  pdl_launch(k_gemm_sub_persist, dim3(unsigned(grid)), dim3(GQ_THREADS), GQ_SMEM_BYTES, s,
             C + mb0 * GT_M * ldc + nb0 * GT_N, ldc, pa, pb, nrows, ncols, nk, nbn, ntiles, err, wait_limit());
  return launch_status();
}

static int gemm_sub_pre(float* C, int64_t ldc, const float* A, int64_t lda, const float* B, int64_t ldb, int64_t M,
                        int64_t Nc, int K, uint8_t* work, int* err, cudaStream_t s) {
  if (M <= 0 || Nc <= 0 || K <= 0) return OK;
  if (gemm_pre_attr() != OK) return CUDA_ERR;
  gemm_split(A, lda, B, ldb, M, Nc, K, work, s);
  return gemm_persist_part(C, ldc, work, M, Nc, K, 0, (M + GT_M - 1) / GT_M, 0, (Nc + GT_N - 1) / GT_N, 0, err, s);
}

// Lookahead of the panel factorisation: SMs left free of the trailing update
// (0: no lookahead).  With lookahead the trailing update of a panel is split:
// the next panel's 256 columns first, on every SM, then the remaining columns
// on a second stream with all but this many SMs, while the next panel is
// factored on the first stream.  Set by tb_set_solve_lookahead.
static std::atomic<int> g_lookahead{-1};  // -1: one SM in five

static int lookahead_reserve() {
  const int v = g_lookahead.load(std::memory_order_relaxed);
  return v < 0 ? num_sms() / 5 : v;
}

struct SideStream {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, top = nullptr, bottom = nullptr;
};
static std::mutex g_side_mutex;
static SideStream g_side[64];

static int side_stream(SideStream*& out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CUDA_ERR;
  std::lock_guard<std::mutex> lock(g_side_mutex);
  SideStream& ss = g_side[dev];
  if (!ss.side) {
    if (cudaStreamCreateWithFlags(&ss.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.top, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.bottom, cudaEventDisableTiming) != cudaSuccess)
      return CUDA_ERR;
  }
  out = &ss;
  return OK;
}

// FP32 LU without pivoting, two-level blocked: panels of 256 columns are
// factored with the 64-wide kernels above (diagonal block, triangular
// solves) and tensor-core updates (K = 64) inside the panel and its row
// block; the trailing matrix is updated once per panel by the persistent
// tensor-core GEMM (K = 256) from operands pre-split into `work`.  err
// receives 1 if a tensor-core wait ran out.
constexpr int TC_PANEL = 256;
static int lu_nopiv_f32_tc(float* A, int64_t lda, int64_t N, int* err, uint8_t* work, cudaStream_t s) {
  const int reserve = lookahead_reserve();
  SideStream* ss = nullptr;
  if (reserve > 0 && side_stream(ss) != OK) return CUDA_ERR;
  if (gemm_pre_attr() != OK) return CUDA_ERR;
  // With lookahead the trailing update of panel p runs in three parts: the
  // next panel's 256 columns first, on every SM, on the caller's stream;
  // then, on the side stream with all but `reserve` SMs, the remaining
  // columns of the next panel's 256 rows (the row block it factors next,
  // event `top`) and of all rows below (event `bottom`).  The next panel's
  // column factorisation runs beside `top`, its row block beside `bottom`.
  // The split operands alternate between two buffers, so a panel's split
  // never overwrites the operands of an update still running.
  const int64_t buf_bytes = round256(gemm_pre_bytes(N, N, TC_PANEL));
  bool top_pending = false, bottom_pending = false;
  int buf = 0;
  for (int64_t p0 = 0; p0 < N; p0 += TC_PANEL) {
    const int64_t pe = p0 + TC_PANEL < N ? p0 + TC_PANEL : N;
    for (int64_t k0 = p0; k0 < pe; k0 += MX_NB) {
      const int nb = pe - k0 < MX_NB ? int(pe - k0) : MX_NB;
      pdl_launch(k_diag_lu_f32, dim3(1), dim3(256), 0, s, A, lda, k0, nb);
      const int64_t below = N - k0 - nb, right = pe - k0 - nb;
      if (below > 0)
        pdl_launch(k_trsm_right_f32, dim3(unsigned((below + TRSM_COLS - 1) / TRSM_COLS)), dim3(TRSM_COLS), 0, s, A,
                   lda, k0 + nb, N, k0, nb);
      if (right > 0) {
        pdl_launch(k_trsm_left_f32, dim3(unsigned((right + TRSM_COLS - 1) / TRSM_COLS)), dim3(TRSM_COLS), 0, s, A,
                   lda, k0 + nb, pe, k0, nb);
        const int st = gemm_sub_tf32x3(A + (k0 + nb) * lda + k0 + nb, lda, A + (k0 + nb) * lda + k0, lda,
                                       A + k0 * lda + k0 + nb, lda, below, right, nb, err, s);
        if (st != OK) return st;
      }
    }
    const int64_t rest = N - pe;
    if (rest <= 0) break;
    if (top_pending) {  // the row block reads the columns `top` updates
      if (cudaStreamWaitEvent(s, ss->top, 0) != cudaSuccess) return CUDA_ERR;
      top_pending = false;
    }
    // row block right of the panel: U12 = L11^-1 A12, 64 rows at a time
    for (int64_t k0 = p0; k0 < pe; k0 += MX_NB) {
      const int nb = pe - k0 < MX_NB ? int(pe - k0) : MX_NB;
      pdl_launch(k_trsm_left_f32, dim3(unsigned((rest + TRSM_COLS - 1) / TRSM_COLS)), dim3(TRSM_COLS), 0, s, A, lda,
                 pe, N, k0, nb);
      const int64_t rows = pe - k0 - nb;
      if (rows > 0) {
        const int st = gemm_sub_tf32x3(A + (k0 + nb) * lda + pe, lda, A + (k0 + nb) * lda + k0, lda, A + k0 * lda + pe,
                                       lda, rows, rest, nb, err, s);
        if (st != OK) return st;
      }
    }
    const int K = int(pe - p0);
    float* C = A + pe * lda + pe;
    uint8_t* w = work + (ss ? buf * buf_bytes : 0);
    const int nk = (K + GT_K - 1) / GT_K;
    const int64_t mbk = (rest + GT_M - 1) / GT_M, nbk = (rest + GT_N - 1) / GT_N;
    const float* L21 = A + pe * lda + p0;
    const float* U12 = A + p0 * lda + pe;
    uint8_t* wb = w + mbk * nk * (int64_t)PA_BLOCK;
    // split operands: L21 and the next panel's columns of U12 here; the rest
    // of U12 on the side stream when it runs the rest of the update
    pdl_launch(k_split_a, dim3(unsigned(nk), unsigned(mbk)), dim3(256), 0, s, L21, lda, rest, K, w);
    pdl_launch(k_split_b, dim3(unsigned(nk), 1u), dim3(256), 0, s, U12, lda, K, rest < GT_N ? rest : GT_N, wb);
    if (bottom_pending) {  // the update below reads rows `bottom` updates
      if (cudaStreamWaitEvent(s, ss->bottom, 0) != cudaSuccess) return CUDA_ERR;
      bottom_pending = false;
    }
    if (ss && nbk > 1) {
      constexpr int64_t TOP = TC_PANEL / GT_M;  // row blocks of the next panel
      int st = gemm_persist_part(C, lda, w, rest, rest, K, 0, mbk, 0, 1, 0, err, s);
      if (st != OK) return st;
      if (cudaEventRecord(ss->fork, s) != cudaSuccess || cudaStreamWaitEvent(ss->side, ss->fork, 0) != cudaSuccess)
        return CUDA_ERR;
      k_split_b<<<dim3(unsigned(nk), unsigned(nbk - 1)), 256, 0, ss->side>>>(U12 + GT_N, lda, K, rest - GT_N,
                                                                          wb + nk * (int64_t)PB_BLOCK);
      const int ctas = num_sms() - reserve;
      st = gemm_persist_part(C, lda, w, rest, rest, K, 0, TOP, 1, nbk, ctas, err, ss->side);
      if (st != OK) return st;
      if (cudaEventRecord(ss->top, ss->side) != cudaSuccess) return CUDA_ERR;
      st = gemm_persist_part(C, lda, w, rest, rest, K, TOP, mbk, 1, nbk, ctas, err, ss->side);
      if (st != OK) return st;
      if (cudaEventRecord(ss->bottom, ss->side) != cudaSuccess) return CUDA_ERR;
      top_pending = bottom_pending = true;
      buf ^= 1;
    } else {
      if (nbk > 1)
        k_split_b<<<dim3(unsigned(nk), unsigned(nbk - 1)), 256, 0, s>>>(U12 + GT_N, lda, K, rest - GT_N,
                                                                     wb + nk * (int64_t)PB_BLOCK);
      const int st = gemm_persist_part(C, lda, w, rest, rest, K, 0, mbk, 0, nbk, 0, err, s);
      if (st != OK) return st;
    }
  }
  if (top_pending && cudaStreamWaitEvent(s, ss->top, 0) != cudaSuccess) return CUDA_ERR;
  if (bottom_pending && cudaStreamWaitEvent(s, ss->bottom, 0) != cudaSuccess) return CUDA_ERR;
  return launch_status();
}

// ---------------------------------------------------------------- mixed solve
// Column maxima of |A| as the bits of non-negative doubles (which order as
// unsigned integers): a 2-D grid of column blocks (64 columns, two per lane,
// 16-byte loads) x row slices, one atomicMax per column and CTA.
constexpr int CM_SLICES = 16;
__global__ void __launch_bounds__(256) k_col_maxabs(const double* __restrict__ A, int64_t lda, int64_t N,
                                                    unsigned long long* __restrict__ maxbits) {
  __shared__ double red[8][64];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t j = blockIdx.x * 64 + 2 * lane;
  const int64_t per = (N + CM_SLICES - 1) / CM_SLICES;
  const int64_t r0 = blockIdx.y * per, r1 = r0 + per < N ? r0 + per : N;
  const bool vec = (lda % 2) == 0 && (reinterpret_cast<uintptr_t>(A) % 16) == 0 && j + 1 < N;
  double m0 = 0.0, m1 = 0.0;
  if (vec) {
#pragma unroll 4
    for (int64_t i = r0 + w; i < r1; i += 8) {
      const double2 a = *reinterpret_cast<const double2*>(A + i * lda + j);
      m0 = fmax(m0, fabs(a.x));
      m1 = fmax(m1, fabs(a.y));
    }
  } else {
    for (int64_t i = r0 + w; i < r1; i += 8) {
      if (j < N) m0 = fmax(m0, fabs(A[i * lda + j]));
      if (j + 1 < N) m1 = fmax(m1, fabs(A[i * lda + j + 1]));
    }
  }
  red[w][2 * lane] = m0;
  red[w][2 * lane + 1] = m1;
  __syncthreads();
  if (threadIdx.x < 64) {
    double m = red[0][threadIdx.x];
    for (int k = 1; k < 8; k++) m = fmax(m, red[k][threadIdx.x]);
    const int64_t col = blockIdx.x * 64 + threadIdx.x;
    if (col < N) atomicMax(maxbits + col, (unsigned long long)__double_as_longlong(m));
  }
}

// c[j] = 1 / max_i |A[i, j]| (1 for a zero column)
__global__ void k_col_scale(const unsigned long long* __restrict__ maxbits, double* __restrict__ c, int64_t N) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= N) return;
  const double m = __longlong_as_double((long long)maxbits[j]);
  c[j] = m > 0 ? 1.0 / m : 1.0;
}

// S (float) = A diag(c): one CTA per (row, 512-column chunk), two columns
// per thread with 16-byte loads and 8-byte stores.
constexpr int SC_COLS = 512;
__global__ void __launch_bounds__(256) k_scale_to_f32(const double* __restrict__ A, int64_t lda,
                                                      const double* __restrict__ c, float* __restrict__ S,
                                                      int64_t N) {
  const int64_t chunks = (N + SC_COLS - 1) / SC_COLS;
  const int64_t i = blockIdx.x / chunks, j = (blockIdx.x % chunks) * SC_COLS + 2 * threadIdx.x;
  if (i >= N || j >= N) return;
  const double* a = A + i * lda + j;
  float* o = S + i * N + j;
  if (j + 1 < N && (lda % 2) == 0 && (N % 2) == 0 && (reinterpret_cast<uintptr_t>(A) % 16) == 0) {
    const double2 v = *reinterpret_cast<const double2*>(a);
    const double2 cc = *reinterpret_cast<const double2*>(c + j);
    *reinterpret_cast<float2*>(o) = make_float2(float(v.x * cc.x), float(v.y * cc.y));
  } else {
    o[0] = float(a[0] * c[j]);
    if (j + 1 < N) o[1] = float(a[1] * c[j + 1]);
  }
}

// R[r, i] = F[r, i] - sum_j A[i, j] X[r, j] (nrhs <= 16), streaming A once.
// A persistent grid (one CTA of 8 warps per SM) walks groups of 8 RPW rows;
// X is staged through shared memory in column chunks, double-buffered with
// cp.async so the next chunk arrives while this one is used, and each
// staged value serves the RPW rows of a warp.  A full chunk of in-range rows
// reads two columns per lane with 16-byte loads, all of the chunk's loads
// independent (enough bytes in flight to keep HBM busy).
constexpr int MX_MAX_RHS = 16;
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int RPW>
constexpr int residual_cols() { return RPW == 4 ? 512 : 256; }  // 32 KB of X per chunk
template <int RPW>
constexpr int residual_smem() { return 2 * (RPW == 4 ? 8 : 16) * residual_cols<RPW>() * int(sizeof(double)); }

template <int RPW>  // rows per warp: 4 for nrhs <= 8, 2 for nrhs <= 16
__global__ void __launch_bounds__(256, 1) k_residual(const double* __restrict__ A, int64_t lda,
                                                    const double* __restrict__ X, const double* __restrict__ F,
                                                    double* __restrict__ R, int64_t N, int nrhs) {
  constexpr int NR = RPW == 4 ? 8 : 16;
  constexpr int RES_COLS = residual_cols<RPW>();
  extern __shared__ __align__(16) double res_dyn[];  // [2][NR][RES_COLS]
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const bool avec = (lda % 2) == 0 && (reinterpret_cast<uintptr_t>(A) % 16) == 0;
  const int64_t nchunk = (N + RES_COLS - 1) / RES_COLS;
  auto stage = [&](int64_t ch, int buf) {  // chunk ch of X into buffer buf (zeros outside)
    double* xb = res_dyn + buf * NR * RES_COLS;
    const int64_t c0 = ch * RES_COLS;
    for (int e = threadIdx.x; e < NR * RES_COLS; e += blockDim.x) {
      const int r = e / RES_COLS, c = e % RES_COLS;
      const bool in = r < nrhs && c0 + c < N;
      cp_async8(xb + e, in ? X + (int64_t)r * N + c0 + c : X, in ? 8 : 0);
    }
    cp_async_commit_group();
  };
  for (int64_t grp = blockIdx.x; grp * 8 * RPW < N; grp += gridDim.x) {
    const int64_t row0 = (grp * 8 + warp) * RPW;
    const bool vec = avec && row0 + RPW <= N;
    double acc[RPW][NR];
#pragma unroll
    for (int q = 0; q < RPW; q++)
#pragma unroll
      for (int r = 0; r < NR; r++) acc[q][r] = 0.0;
    __syncthreads();  // the previous group is done with both buffers
    stage(0, 0);
    for (int64_t ch = 0; ch < nchunk; ch++) {
      if (ch + 1 < nchunk) {
        stage(ch + 1, int((ch + 1) & 1));
        cp_async_wait_group<1>();
      } else {
        cp_async_wait_group<0>();
      }
      __syncthreads();
      const double* xb = res_dyn + (ch & 1) * NR * RES_COLS;
      const int64_t c0 = ch * RES_COLS;
      if (vec && c0 + RES_COLS <= N) {
#pragma unroll
        for (int c = 2 * lane; c < RES_COLS; c += 64) {
          double2 a[RPW];
#pragma unroll
          for (int q = 0; q < RPW; q++) a[q] = *reinterpret_cast<const double2*>(A + (row0 + q) * lda + c0 + c);
#pragma unroll
          for (int r = 0; r < NR; r++) {
            const double2 x = *reinterpret_cast<const double2*>(xb + r * RES_COLS + c);
#pragma unroll
            for (int q = 0; q < RPW; q++) acc[q][r] = fma(a[q].y, x.y, fma(a[q].x, x.x, acc[q][r]));
          }
        }
      } else {
#pragma unroll 4
        for (int c = lane; c < RES_COLS; c += 32) {
          if (c0 + c >= N) break;
          double a[RPW];
#pragma unroll
          for (int q = 0; q < RPW; q++) a[q] = row0 + q < N ? A[(row0 + q) * lda + c0 + c] : 0.0;
#pragma unroll
          for (int r = 0; r < NR; r++) {
            const double x = xb[r * RES_COLS + c];
#pragma unroll
            for (int q = 0; q < RPW; q++) acc[q][r] = fma(a[q], x, acc[q][r]);
          }
        }
      }
      __syncthreads();  // this buffer is staged again two chunks on
    }
#pragma unroll
    for (int q = 0; q < RPW; q++) {
      const int64_t i = row0 + q;
#pragma unroll
      for (int r = 0; r < NR; r++) {
        const double v = warp_sum(acc[q][r]);
        if (lane == 0 && i < N && r < nrhs) R[(int64_t)r * N + i] = F[(int64_t)r * N + i] - v;
      }
    }
  }
}

// ---------------------------------------------------------------- sweeps
// One launch per triangular sweep of the refinement's correction equation.
// CTA q owns row block b (64 rows; b = q for the forward sweep with the unit
// lower factor, b = nblk - 1 - q for the backward sweep with the upper
// factor), so every block it depends on belongs to a CTA launched before it.
//
// Lookahead form.  With T the triangle, D_b = T_bb^-1 and g the block
// published last before b (g = b - 1 forward, b + 1 backward):
//   x_b = y_b - M_b x_g,   y_b = D_b (r_b - sum_{j != g} T_bj x_j),   M_b = D_b T_bg.
// y_b needs only blocks published before g, so the CTA finishes it while it
// waits; the step that gates the next block is one 64 x 64 FP64
// matrix-vector product with the freshly published x_g.  D_b and M_b are
// computed once per factorisation (k_diag_inverse) in FP64 from the FP32
// factor values.  Published blocks: the sweep writes its solution into an
// output vector that was filled with a sentinel bit pattern (all bytes 0xFF,
// a NaN no arithmetic produces) before the launch; a consumer polls the
// values of the block it needs until none is the sentinel (relaxed GPU-scope
// stores and loads, each value single-copy atomic), so no flag, fence or
// second read of the data sits on the chain.  A CTA's place in the chain is the ticket it draws
// from a counter when it starts (not its block index), so it only ever
// waits on CTAs that are already running, whatever order the hardware
// starts them in.  Waits are bounded (the library's wait limit): when one
// runs out the CTA records an error and writes NaN, and the solve returns
// TB_TIMEOUT.
constexpr int TS_B = 64;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Sweep outputs: relaxed GPU-scope 8-byte accesses (single-copy atomic, and
// never served from a stale L1 line).
constexpr long long SWEEP_SENTINEL = -1LL;  // all bytes 0xFF
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// Bounded wait of one thread for flags[j] == epoch; false (and err set) when
// it ran out.  The sleep between polls doubles up to max_ns.
__device__ __forceinline__ bool wait_flag(const int* flags, int j, int epoch, int* err, unsigned max_ns,
                                          long long max_cycles) {
  const long long t0 = clock64();
  unsigned ns = 32;
  while (ld_acquire(flags + j) != epoch) {
    if (clock64() - t0 > max_cycles) {
      atomicExch(err, 1);
      return false;
    }
    __nanosleep(ns);
    ns = ns < max_ns ? 2 * ns : max_ns;
  }
  return true;
}

// For row block b of the unit lower (LOWER) or upper triangle of LU:
// Dinv[b] = T_bb^-1 and Mla[b] = T_bb^-1 T_bg (g = b - 1 / b + 1; zero when
// b has no such neighbour), both 64 x 64 FP64 stored column-major
// (element (i, m) at m * 64 + i); rows / columns beyond N are the identity
// in T_bb and zero in T_bg.  One CTA of 64 threads per block, one column per
// thread.
template <bool LOWER>
__global__ void __launch_bounds__(TS_B) k_diag_inverse(const float* __restrict__ LU, int64_t lda, int64_t N,
                                                      double* __restrict__ Dinv, double* __restrict__ Mla) {
  __shared__ float T[TS_B][TS_B];    // the factor block (FP32 values, exact)
  __shared__ double Xc[TS_B][TS_B];  // Xc[row][col]; thread k owns column k
  const int nblk = int((N + TS_B - 1) / TS_B);
  const int64_t b0 = (int64_t)blockIdx.x * TS_B;
  const int nb = N - b0 < TS_B ? int(N - b0) : TS_B;
  for (int e = threadIdx.x; e < TS_B * TS_B; e += blockDim.x) {
    const int i = e / TS_B, j = e % TS_B;
    float v = (i == j) ? 1.f : 0.f;
    if (i < nb && j < nb) {
      const float a = LU[(b0 + i) * lda + b0 + j];
      if (LOWER ? (i > j) : (i <= j)) v = a;
    }
    T[i][j] = v;
  }
  __syncthreads();
  const int k = threadIdx.x;  // column k of the inverse: T x = e_k
  if (LOWER) {
    for (int i = 0; i < TS_B; i++) {
      double v = (i == k) ? 1.0 : 0.0;
      for (int m = 0; m < i; m++) v = fma(-double(T[i][m]), Xc[m][k], v);
      Xc[i][k] = v;
    }
  } else {
    for (int i = TS_B - 1; i >= 0; i--) {
      double v = (i == k) ? 1.0 : 0.0;
      for (int m = i + 1; m < TS_B; m++) v = fma(-double(T[i][m]), Xc[m][k], v);
      Xc[i][k] = v / double(T[i][i]);
    }
  }
  __syncthreads();
  double* D = Dinv + (int64_t)blockIdx.x * TS_B * TS_B;
  for (int e = threadIdx.x; e < TS_B * TS_B; e += blockDim.x) D[e] = Xc[e % TS_B][e / TS_B];
  // the lookahead product with the neighbour block of the same block row
  const int g = LOWER ? int(blockIdx.x) - 1 : int(blockIdx.x) + 1;
  double* Mo = Mla + (int64_t)blockIdx.x * TS_B * TS_B;
  if (g < 0 || g >= nblk) {
    for (int e = threadIdx.x; e < TS_B * TS_B; e += blockDim.x) Mo[e] = 0.0;
    return;
  }
  const int64_t g0 = (int64_t)g * TS_B;
  for (int e = threadIdx.x; e < TS_B * TS_B; e += blockDim.x) {
    const int i = e / TS_B, j = e % TS_B;
    T[i][j] = (i < nb && g0 + j < N) ? LU[(b0 + i) * lda + g0 + j] : 0.f;
  }
  __syncthreads();
  for (int i = 0; i < TS_B; i++) {
    double v0 = 0.0, v1 = 0.0;
#pragma unroll 8
    for (int m = 0; m < TS_B; m += 2) {
      v0 = fma(Xc[i][m], double(T[m][k]), v0);
      v1 = fma(Xc[i][m + 1], double(T[m + 1][k]), v1);
    }
    Mo[(int64_t)k * TS_B + i] = v0 + v1;
  }
}

// X (nrhs x N, row r at X + r N) <- T^-1 X with T the unit lower (LOWER) or
// upper triangle of LU, in the lookahead form above.  256 threads: thread
// (i, grp) = (tid % 64, tid / 64) accumulates row i of the block over
// columns 16 grp .. 16 grp + 15 of every tile before the gate (16 factor
// values prefetched into registers one tile ahead, NR right-hand sides in
// registers; the four column groups meet in shared memory once, in a fixed
// order), and owns right-hand sides NR/4 grp .. NR/4 grp + NR/4 - 1 of row i
// in the two matrix-vector products.  Dynamic shared memory: D_b, M_b
// (64 KB) and the column groups' partial sums (NR * 2 KB).
// In holds the right-hand sides, Out (sentinel-filled) receives the
// solution.  flags[nblk] is the ticket counter (every launch of a solve
// draws nblk tickets, so the launch of epoch e draws (e - 1) nblk ..
// e nblk - 1).
template <int NR>
constexpr int sweep_dyn_bytes() {
  return 2 * TS_B * TS_B * int(sizeof(double)) + 4 * NR * TS_B * int(sizeof(double));
}

template <bool LOWER, int NR>
__global__ void __launch_bounds__(256, 2) k_trsv_sweep(const float* __restrict__ LU, int64_t lda, int64_t N,
                                                   const double* __restrict__ Dinv, const double* __restrict__ Mla,
                                                   const double* __restrict__ In, double* __restrict__ Out, int nrhs,
                                                   int* __restrict__ flags, int epoch, int* __restrict__ err,
                                                   long long wait_cycles) {
  extern __shared__ __align__(16) double sw_dyn[];
  double* Ds = sw_dyn;                    // D_b, column-major
  double* Ms = sw_dyn + TS_B * TS_B;      // M_b, column-major
  double* part = Ms + TS_B * TS_B;        // part[(grp * NR + r) * 64 + i]
  __shared__ __align__(16) double xs[NR][TS_B];  // a published block's solution
  __shared__ double rs[NR][TS_B];                // this block's right-hand side
  __shared__ int s_fail, s_ticket;
  constexpr int RPT = NR / 4;  // right-hand sides per thread in the products
  const int nblk = int((N + TS_B - 1) / TS_B);
  if (threadIdx.x == 0) s_ticket = atomicAdd(flags + nblk, 1) - (epoch - 1) * nblk;
  __syncthreads();
  const int q = s_ticket;  // this CTA's place in the chain
  const int b = LOWER ? q : nblk - 1 - q;
  const int64_t b0 = (int64_t)b * TS_B;
  const int i = threadIdx.x % TS_B, grp = threadIdx.x / TS_B;
  // everything that does not depend on other blocks first
  {
    const double* Dg = Dinv + (int64_t)b * TS_B * TS_B;
    const double* Mg = Mla + (int64_t)b * TS_B * TS_B;
    for (int e = threadIdx.x; e < TS_B * TS_B; e += blockDim.x) {
      Ds[e] = Dg[e];
      Ms[e] = Mg[e];
    }
  }
  for (int e = threadIdx.x; e < NR * TS_B; e += blockDim.x) {
    const int r = e / TS_B, c = e % TS_B;
    rs[r][c] = (r < nrhs && b0 + c < N) ? In[(int64_t)r * N + b0 + c] : 0.0;
  }
  if (threadIdx.x == 0) s_fail = 0;
  __syncthreads();
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) acc[r] = 0.0;
  const int64_t row = b0 + i;
  const bool vec4 = (lda % 4) == 0 && (reinterpret_cast<uintptr_t>(LU) % 16) == 0;
  float lv[16];  // row i, columns 16 grp .. 16 grp + 15 of the next tile
  auto load_lu = [&](int j) {
    const int64_t j0 = (int64_t)j * TS_B + 16 * grp;
    if (vec4 && row < N && j0 + 16 <= N) {
      const float4* p = reinterpret_cast<const float4*>(LU + row * lda + j0);
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const float4 f = __ldg(p + v);
        lv[4 * v] = f.x;
        lv[4 * v + 1] = f.y;
        lv[4 * v + 2] = f.z;
        lv[4 * v + 3] = f.w;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 16; c++) lv[c] = (row < N && j0 + c < N) ? LU[row * lda + j0 + c] : 0.f;
    }
  };
  // A block published by another CTA, polled until none of its values is the
  // sentinel (every thread of the CTA calls it; false if the bounded wait ran
  // out, after which s_fail is set).  Ends with the values in xs.
  auto poll_x = [&](int64_t j0, unsigned max_ns) -> bool {
    const long long t0 = clock64();
    unsigned ns = 32;
    for (;;) {
      bool ready = true;
      for (int e = threadIdx.x; e < NR * TS_B; e += blockDim.x) {
        const int r = e / TS_B, c = e % TS_B;
        double v = 0.0;
        if (r < nrhs && j0 + c < N) {
          v = ld_relaxed_f64(Out + (int64_t)r * N + j0 + c);
          ready = ready && __double_as_longlong(v) != SWEEP_SENTINEL;
        }
        xs[r][c] = v;
      }
      if (__syncthreads_and(ready)) return true;
      if (threadIdx.x == 0 && clock64() - t0 > wait_cycles) {
        atomicExch(err, 1);
        s_fail = 1;
      }
      __syncthreads();
      if (s_fail) return false;
      __nanosleep(ns);
      ns = ns < max_ns ? 2 * ns : max_ns;
    }
  };
  const int nacc = q > 0 ? q - 1 : 0;  // tiles accumulated before the gate
  if (nacc > 0) load_lu(LOWER ? 0 : nblk - 1);
  for (int t = 0; t < nacc; t++) {
    const int j = LOWER ? t : nblk - 1 - t;  // finished blocks in publication order
    __syncthreads();  // every thread is done with the previous tile's xs
    if (!poll_x((int64_t)j * TS_B, 256)) break;
    float lc[16];
#pragma unroll
    for (int c = 0; c < 16; c++) lc[c] = lv[c];
    if (t + 1 < nacc) load_lu(LOWER ? t + 1 : nblk - 2 - t);
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
#pragma unroll
      for (int r = 0; r < NR; r++) {
        const double2 x = *reinterpret_cast<const double2*>(&xs[r][16 * grp + c]);
        acc[r] = fma(double(lc[c]), x.x, acc[r]);
        acc[r] = fma(double(lc[c + 1]), x.y, acc[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < NR; r++) part[(grp * NR + r) * TS_B + i] = acc[r];
  __syncthreads();
  // y_b = D_b (r_b - sum): this thread's right-hand sides of row i
#pragma unroll
  for (int u = 0; u < RPT; u++) {
    const int r = RPT * grp + u;
    double v = rs[r][i];
#pragma unroll
    for (int h = 0; h < 4; h++) v -= part[(h * NR + r) * TS_B + i];
    rs[r][i] = v;
  }
  __syncthreads();
  double y[RPT];
  {
    double y0[RPT], y1[RPT];
#pragma unroll
    for (int u = 0; u < RPT; u++) y0[u] = y1[u] = 0.0;
#pragma unroll 4
    for (int m = 0; m < TS_B; m += 2) {
      const double d0 = Ds[m * TS_B + i], d1 = Ds[(m + 1) * TS_B + i];
#pragma unroll
      for (int u = 0; u < RPT; u++) {
        y0[u] = fma(d0, rs[RPT * grp + u][m], y0[u]);
        y1[u] = fma(d1, rs[RPT * grp + u][m + 1], y1[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < RPT; u++) y[u] = y0[u] + y1[u];
  }
  // the gate: x_b = y_b - M_b x_g
  if (q > 0) {
    const int g = LOWER ? b - 1 : b + 1;
    __syncthreads();  // every thread is done with the previous tile's xs
    if (!s_fail && poll_x((int64_t)g * TS_B, 64)) {
      double z0[RPT], z1[RPT];
#pragma unroll
      for (int u = 0; u < RPT; u++) z0[u] = z1[u] = 0.0;
#pragma unroll 4
      for (int m = 0; m < TS_B; m += 2) {
        const double m0 = Ms[m * TS_B + i], m1 = Ms[(m + 1) * TS_B + i];
#pragma unroll
        for (int u = 0; u < RPT; u++) {
          z0[u] = fma(m0, xs[RPT * grp + u][m], z0[u]);
          z1[u] = fma(m1, xs[RPT * grp + u][m + 1], z1[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < RPT; u++) y[u] -= z0[u] + z1[u];
    }
  }
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
  for (int u = 0; u < RPT; u++) {
    const int r = RPT * grp + u;
    if (r < nrhs && row < N) st_relaxed_f64(Out + (int64_t)r * N + row, s_fail ? nan : y[u]);
  }
}

// X[r, j] += c[j] D[r, j]; also, per right-hand side r, the largest
// |c D| (maxes[2 r]) and |X| (maxes[2 r + 1]) -- non-negative doubles order
// like their bit patterns.  Grid (blocks, nrhs): one warp-reduced atomic per
// warp and quantity.
__global__ void k_apply_correction(double* __restrict__ X, const double* __restrict__ D, const double* __restrict__ c,
                                   int64_t N, unsigned long long* __restrict__ maxes) {
  const int r = blockIdx.y;
  unsigned long long md = 0, mx = 0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < N; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = (int64_t)r * N + j;
    const double d = c[j] * D[g];
    const double x = X[g] + d;
    X[g] = x;
    double ad = fabs(d);
    const double ax = fabs(x);
    if (!(ad == ad) || !(ax == ax)) ad = 1e300;
    const unsigned long long bd = (unsigned long long)__double_as_longlong(ad);
    const unsigned long long bx = (unsigned long long)__double_as_longlong(ax);
    md = bd > md ? bd : md;
    mx = bx > mx ? bx : mx;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long od = __shfl_xor_sync(0xffffffffu, md, o);
    const unsigned long long ox = __shfl_xor_sync(0xffffffffu, mx, o);
    md = od > md ? od : md;
    mx = ox > mx ? ox : mx;
  }
  if (threadIdx.x % 32 == 0) {
    atomicMax(&maxes[2 * r], md);
    atomicMax(&maxes[2 * r + 1], mx);
  }
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
      k_trsm_left<T><<<g, 128, 0, s>>>(A, lda, k0 + nb, N, k0, nb);
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


extern "C" int tb_set_solve_lookahead(int reserve_sms) {
  const int prev = lookahead_reserve();
  g_lookahead.store(reserve_sms < 0 ? -1 : (reserve_sms < num_sms() ? reserve_sms : 0));
  return prev;
}

extern "C" int64_t tb_gemm_tf32x3_workspace(int64_t M, int64_t N, int64_t K) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  return gemm_pre_bytes(M, N, K);
}

extern "C" int64_t tb_lu_nopiv_f32_tc_workspace(int64_t N) {
  if (N <= 0) return 0;
  return 2 * round256(gemm_pre_bytes(N, N, TC_PANEL));  // two alternating split-operand buffers
}

extern "C" int tb_lu_nopiv_f32_tc(float* A, int64_t lda, int64_t N, void* work, int64_t work_bytes, int* err,
                                  tb_stream_t stream) {
  if (N < 0 || lda < N || (N > 0 && (!A || !err)) || N > 0x7fffffff) return BAD_ARG;
  if (N == 0) return OK;
  if (!work || work_bytes < tb_lu_nopiv_f32_tc_workspace(N) || reinterpret_cast<uintptr_t>(work) % 16 != 0)
    return BAD_ARG;
  return lu_nopiv_f32_tc(A, lda, N, err, static_cast<uint8_t*>(work), (cudaStream_t)stream);
}

extern "C" int tb_gemm_sub_tf32x3(float* C, int64_t ldc, const float* A, int64_t lda, const float* B, int64_t ldb,
                                  int64_t M, int64_t N, int64_t K, void* work, int64_t work_bytes, int* err,
                                  tb_stream_t stream) {
  if (M < 0 || N < 0 || K < 0 || K > 0x7fffffff || !err) return BAD_ARG;
  if (M == 0 || N == 0 || K == 0) return OK;
  if (!C || !A || !B || ldc < N || lda < K || ldb < N) return BAD_ARG;
  if (work) {
    if (work_bytes < gemm_pre_bytes(M, N, K) || reinterpret_cast<uintptr_t>(work) % 16 != 0) return BAD_ARG;
    return gemm_sub_pre(C, ldc, A, lda, B, ldb, M, N, int(K), static_cast<uint8_t*>(work), err,
                        (cudaStream_t)stream);
  }
  return gemm_sub_tf32x3(C, ldc, A, lda, B, ldb, M, N, int(K), err, (cudaStream_t)stream);
}

extern "C" int64_t tb_solve_mixed_workspace(int64_t N, int64_t nrhs) {
  if (N <= 0 || nrhs <= 0) return 0;
  const int64_t nblk = (N + TS_B - 1) / TS_B;
  // FP32 factors, column scales, correction / residual block, the forward
  // sweep's output, 2 * nrhs maxima, inverses of the diagonal blocks of both
  // factors and their lookahead products, sweep flags and the error word
  return round256(N * N * 4) + round256(N * 8) + 2 * round256(nrhs * N * 8) + 256 +
         4 * round256(nblk * TS_B * TS_B * 8) + round256((nblk + 1) * 4) + 256 +
         round256(tb_lu_nopiv_f32_tc_workspace(N));
}

extern "C" int tb_solve_mixed(const double* A, int64_t lda, int64_t N, const double* F, double* X, int64_t nrhs,
                              void* work, int64_t work_bytes, int max_iter, double tol, int* iters_out,
                              double* last_rel_out, tb_stream_t stream) {
  if (N <= 0 || nrhs <= 0 || nrhs > MX_MAX_RHS || lda < N || !A || !F || !X || !work || max_iter < 1)
    return BAD_ARG;
  if (work_bytes < tb_solve_mixed_workspace(N, nrhs)) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  char* w = static_cast<char*>(work);
  const int64_t nblk = (N + TS_B - 1) / TS_B;
  float* S = reinterpret_cast<float*>(w);
  w += round256(N * N * 4);
  double* c = reinterpret_cast<double*>(w);
  w += round256(N * 8);
  double* D = reinterpret_cast<double*>(w);
  w += round256(nrhs * N * 8);
  double* Y = reinterpret_cast<double*>(w);  // the forward sweep's output
  w += round256(nrhs * N * 8);
  unsigned long long* maxes = reinterpret_cast<unsigned long long*>(w);
  w += 256;
  double* dinv_l = reinterpret_cast<double*>(w);
  w += round256(nblk * TS_B * TS_B * 8);
  double* dinv_u = reinterpret_cast<double*>(w);
  w += round256(nblk * TS_B * TS_B * 8);
  double* mla_l = reinterpret_cast<double*>(w);
  w += round256(nblk * TS_B * TS_B * 8);
  double* mla_u = reinterpret_cast<double*>(w);
  w += round256(nblk * TS_B * TS_B * 8);
  int* flags = reinterpret_cast<int*>(w);  // nblk publication flags + the ticket counter
  w += round256((nblk + 1) * 4);
  int* err = reinterpret_cast<int*>(w);
  w += 256;
  uint8_t* gemm_work = reinterpret_cast<uint8_t*>(w);  // pre-split operands of the trailing updates

  // column maxima (bits gathered in the correction buffer D, N words), scales
  unsigned long long* maxbits = reinterpret_cast<unsigned long long*>(D);
  if (cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long) * N, s) != cudaSuccess) return CUDA_ERR;
  k_col_maxabs<<<dim3(unsigned((N + 63) / 64), CM_SLICES), 256, 0, s>>>(A, lda, N, maxbits);
  k_col_scale<<<unsigned((N + 255) / 256), 256, 0, s>>>(maxbits, c, N);
  {
    const int64_t chunks = (N + SC_COLS - 1) / SC_COLS;
    k_scale_to_f32<<<unsigned(N * chunks), SC_COLS / 2, 0, s>>>(A, lda, c, S, N);
  }
  if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return CUDA_ERR;
  int st = lu_nopiv_f32_tc(S, N, N, err, gemm_work, s);
  if (st != OK) return st;
  k_diag_inverse<true><<<unsigned(nblk), TS_B, 0, s>>>(S, N, N, dinv_l, mla_l);
  k_diag_inverse<false><<<unsigned(nblk), TS_B, 0, s>>>(S, N, N, dinv_u, mla_u);
  if (cudaMemsetAsync(flags, 0, sizeof(int) * (nblk + 1), s) != cudaSuccess) return CUDA_ERR;
  constexpr int SW8 = sweep_dyn_bytes<8>(), SW16 = sweep_dyn_bytes<16>();
  if (cudaFuncSetAttribute(k_residual<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, residual_smem<4>()) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_residual<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, residual_smem<2>()) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_trsv_sweep<true, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, SW8) != cudaSuccess ||
      cudaFuncSetAttribute(k_trsv_sweep<false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, SW8) != cudaSuccess ||
      cudaFuncSetAttribute(k_trsv_sweep<true, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, SW16) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_trsv_sweep<false, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, SW16) !=
          cudaSuccess)
    return CUDA_ERR;
  int epoch = 0;
  const long long wcyc = wait_limit();
  if (cudaMemsetAsync(X, 0, sizeof(double) * N * nrhs, s) != cudaSuccess) return CUDA_ERR;
  const int nr = int(nrhs);
  int it = 0;
  double rel = 1e300;
  for (it = 1; it <= max_iter; it++) {
    // D = F - A X (FP64; F itself while X is still zero), then
    // D <- (L U)^-1 D with the FP32 factors
    if (it == 1) {
      if (cudaMemcpyAsync(D, F, sizeof(double) * N * nrhs, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return CUDA_ERR;
    } else {
      // one CTA per SM, at most one per group of rows
      const int64_t rows = nr <= 8 ? 32 : 16;
      int64_t grid = (N + rows - 1) / rows;
      if (grid > num_sms()) grid = num_sms();
      if (nr <= 8)
        k_residual<4><<<unsigned(grid), 256, residual_smem<4>(), s>>>(A, lda, X, F, D, N, nr);
      else
        k_residual<2><<<unsigned(grid), 256, residual_smem<2>(), s>>>(A, lda, X, F, D, N, nr);
    }
    // D -> Y (forward, unit lower), Y -> D (backward, upper); each output
    // filled with the sentinel first
    const size_t vec_bytes = sizeof(double) * N * nrhs;
    if (cudaMemsetAsync(Y, 0xff, vec_bytes, s) != cudaSuccess) return CUDA_ERR;
    if (nr <= 8)
      k_trsv_sweep<true, 8><<<unsigned(nblk), 256, SW8, s>>>(S, N, N, dinv_l, mla_l, D, Y, nr, flags, ++epoch, err,
                                                                  wcyc);
    else
      k_trsv_sweep<true, 16><<<unsigned(nblk), 256, SW16, s>>>(S, N, N, dinv_l, mla_l, D, Y, nr, flags, ++epoch, err,
                                                                   wcyc);
    if (cudaMemsetAsync(D, 0xff, vec_bytes, s) != cudaSuccess) return CUDA_ERR;
    if (nr <= 8)
      k_trsv_sweep<false, 8><<<unsigned(nblk), 256, SW8, s>>>(S, N, N, dinv_u, mla_u, Y, D, nr, flags, ++epoch, err,
                                                                   wcyc);
    else
      k_trsv_sweep<false, 16><<<unsigned(nblk), 256, SW16, s>>>(S, N, N, dinv_u, mla_u, Y, D, nr, flags, ++epoch,
                                                                    err, wcyc);
    if (cudaMemsetAsync(maxes, 0, sizeof(unsigned long long) * 2 * nr, s) != cudaSuccess) return CUDA_ERR;
    {
      const int64_t bx = (N + 255) / 256;
      k_apply_correction<<<dim3(unsigned(bx < 256 ? bx : 256), unsigned(nr)), 256, 0, s>>>(X, D, c, N, maxes);
    }
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
    // Refinement contracts the error linearly: with q = rel / prev the error
    // left after this correction is about rel * q, so when that is already
    // below tol the round that would only confirm it is skipped.
    if (it >= 2 && rel < 0.5 * prev && rel * (rel / prev) <= tol) {
      rel *= rel / prev;  // reported: the estimated remaining error
      break;
    }
    // Corrections that stop shrinking just above tol have reached the FP64
    // rounding floor of the residual (about cond * 1e-16): converged.
    if (it >= 3 && rel <= 100.0 * tol && rel > 0.5 * prev) {
      rel = tol;
      break;
    }
  }
  if (iters_out) *iters_out = it > max_iter ? max_iter : it;
  if (last_rel_out) *last_rel_out = rel;
  int err_h = 0;  // a bounded wait in the factorisation or a sweep ran out
  if (cudaMemcpyAsync(&err_h, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUDA_ERR;
  if (err_h) return TIMEOUT;
  if (st != OK) return st;
  if (rel > tol) return SINGULAR;  // did not converge: the caller falls back to the pivoted FP64 LU
  return launch_status();
}
