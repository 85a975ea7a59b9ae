// tb_mlp.cu -- the learned field surrogate: a small MLP (4 hidden layers of
// 128, SiLU) trained on the GPU from BEM samples, in BF16 with FP32
// accumulation.  No reference counterpart (the reference has no learned
// part); it is checked against the FP64 BEM field of tb_bem.cu.
//
// Kernels:
//   k_gemm_bf16<AT, BT>  C[M x N] (fp32) = A[M x K] . B[N x K]^T on the tensor
//                        cores (mma.sync m16n8k16, BF16 in, FP32 accumulate);
//                        AT / BT select operands stored with K as the slow
//                        index (the transposed products of the backward pass)
//   k_bias_silu          Z = C + b (kept for the backward pass), Y = silu(Z) (bf16)
//   k_bias_out           Y = C + b (fp32 network output)
//   k_mse_grad           dY = 2 (Y - T) w / (B n), per-block loss partials
//   k_silu_back          dZ = dA * silu'(Z) (bf16)
//   k_colsum             db = sum over rows of dZ
//   k_adam               FP32 master weights, BF16 copies
//   k_features           (r, z) -> 16 input features
#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "tb_mlp.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

// ------------------------------------------------------------------ GEMM
constexpr int GM = 64, GN = 64, GK = 32;

template <bool AT, bool BT>
__global__ void __launch_bounds__(128)
    k_gemm_bf16(const __nv_bfloat16* __restrict__ A, int64_t lda, const __nv_bfloat16* __restrict__ B, int64_t ldb,
                float* __restrict__ C, int64_t ldc, int M, int N, int K, int accumulate, int kchunk) {
  __shared__ __align__(16) __nv_bfloat16 sA[GM][GK + 8];
  __shared__ __align__(16) __nv_bfloat16 sB[GN][GK + 8];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int wm = (warp / 2) * 32, wn = (warp % 2) * 32;  // warp tile origin in the block tile
  const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[i][j][c] = 0.f;
  const int g = lane >> 2, q = lane & 3;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  for (int k0 = kbeg; k0 < kend; k0 += GK) {
    __syncthreads();
    for (int e = threadIdx.x; e < GM * GK; e += 128) {
      int mm = e / GK, kk = e % GK;
      if (AT) {  // A(m, k) at A[k * lda + m]: walk m fastest for coalescing
        mm = e % GM;
        kk = e / GM;
      }
      int gm = m0 + mm, gk = k0 + kk;
      __nv_bfloat16 v = __float2bfloat16(0.f);
      if (gm < M && gk < kend) v = AT ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk];
      sA[mm][kk] = v;
    }
    for (int e = threadIdx.x; e < GN * GK; e += 128) {
      int nn = e / GK, kk = e % GK;
      if (BT) {
        nn = e % GN;
        kk = e / GN;
      }
      int gn = n0 + nn, gk = k0 + kk;
      __nv_bfloat16 v = __float2bfloat16(0.f);
      if (gn < N && gk < kend) v = BT ? B[(int64_t)gk * ldb + gn] : B[(int64_t)gn * ldb + gk];
      sB[nn][kk] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; kk += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&sA[r][kk + 2 * q]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][kk + 2 * q]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&sA[r][kk + 8 + 2 * q]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][kk + 8 + 2 * q]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        int n = wn + j * 8 + g;
        bf[j][0] = *reinterpret_cast<const uint32_t*>(&sB[n][kk + 2 * q]);
        bf[j][1] = *reinterpret_cast<const uint32_t*>(&sB[n][kk + 8 + 2 * q]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16_16816(acc[i][j], af[i], bf[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        int r = m0 + wm + i * 16 + g + (c >= 2 ? 8 : 0);
        int col = n0 + wn + j * 8 + 2 * q + (c & 1);
        if (r < M && col < N) {
          float* p = C + (int64_t)r * ldc + col;
          if (accumulate == 2)
            atomicAdd(p, acc[i][j][c]);  // split-K partial
          else
            *p = accumulate ? *p + acc[i][j][c] : acc[i][j][c];
        }
      }
}

// ------------------------------------------------------------------ elementwise
// One pair of adjacent elements per thread (the packed SiLU works on pairs);
// an odd last element is paired with a zero.
__global__ void k_bias_silu(const float* __restrict__ C, const float* __restrict__ b, float* __restrict__ Z,
                            __nv_bfloat16* __restrict__ Y, int64_t M, int N) {
  const int64_t n = M * N;
  const int64_t i = 2 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float z0 = C[i] + b[i % N];
  const bool two = i + 1 < n;
  const float z1 = two ? C[i + 1] + b[(i + 1) % N] : 0.f;
  if (Z) {
    Z[i] = z0;
    if (two) Z[i + 1] = z1;
  }
  const uint32_t y = silu2_bf16(z0, z1);
  Y[i] = __ushort_as_bfloat16((unsigned short)(y & 0xffffu));
  if (two) Y[i + 1] = __ushort_as_bfloat16((unsigned short)(y >> 16));
}

__global__ void k_bias_out(const float* __restrict__ C, const float* __restrict__ b, float* __restrict__ Y,
                           int64_t M, int N) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  Y[i] = C[i] + b[i % N];
}

// MSE over the first n_out columns of Y (M x N): loss = mean_(i, c<n_out) w_i (Y - T)^2.
__global__ void k_mse_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ w,
                           __nv_bfloat16* __restrict__ dY, float* __restrict__ loss_part, int64_t M, int N,
                           int n_out) {
  __shared__ float red[256];
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < M * N) {
    int c = int(i % N);
    int64_t row = i / N;
    float g = 0.f;
    if (c < n_out) {
      float d = Y[i] - T[row * n_out + c];
      float wi = w ? w[row] : 1.f;
      g = 2.f * d * wi / float(M * n_out);
      l = d * d * wi;
    }
    dY[i] = __float2bfloat16(g);
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

__global__ void k_silu_back(const float* __restrict__ dA, const float* __restrict__ Z,
                            __nv_bfloat16* __restrict__ dZ, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  dZ[i] = __float2bfloat16(dA[i] * silu_grad(Z[i]));
}

// db[c] = sum_r dZ[r, c]; one block per column.
__global__ void k_colsum(const __nv_bfloat16* __restrict__ dZ, float* __restrict__ db, int64_t M, int N) {
  __shared__ float red[256];
  int c = blockIdx.x;
  float s = 0.f;
  for (int64_t r = threadIdx.x; r < M; r += 256) s += __bfloat162float(dZ[r * N + c]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = red[0];
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ pb, int64_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  pb[i] = __float2bfloat16(pi);
}

__global__ void k_features(const double* __restrict__ pts, int64_t M, MlpDomain dom, __nv_bfloat16* __restrict__ X) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= M) return;
  double r = sqrt(pts[3 * i] * pts[3 * i] + pts[3 * i + 1] * pts[3 * i + 1]);
  float f[MLP_IN];
  mlp_features(r, pts[3 * i + 2], dom, f);
#pragma unroll
  for (int c = 0; c < MLP_IN; c++) X[i * MLP_IN + c] = __float2bfloat16(f[c]);
}

}  // namespace tb

using namespace tb;

extern "C" int tb_mlp_gemm(const void* A, int64_t lda, int a_t, const void* B, int64_t ldb, int b_t, float* C,
                           int64_t ldc, int64_t M, int64_t N, int64_t K, int accumulate, tb_stream_t stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return BAD_ARG;
  if (M > (int64_t)65535 * GM || N > (int64_t)65535 * GN || K > 0x7fffffff) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  // Few output tiles and a long reduction (the weight gradients, K = batch):
  // split K over blockIdx.z and add the partial tiles atomically into C,
  // which is cleared first.
  const int64_t tiles = ((N + GN - 1) / GN) * ((M + GM - 1) / GM);
  int kchunk = int(K);
  if (tiles < 64 && K >= 1024 && accumulate == 0) {
    kchunk = 512;
    accumulate = 2;
    if (cudaMemset2DAsync(C, size_t(ldc) * sizeof(float), 0, size_t(N) * sizeof(float), size_t(M), s) != cudaSuccess)
      return CUDA_ERR;
  }
  dim3 grid(unsigned((N + GN - 1) / GN), unsigned((M + GM - 1) / GM), unsigned((K + kchunk - 1) / kchunk));
  auto a = static_cast<const __nv_bfloat16*>(A);
  auto b = static_cast<const __nv_bfloat16*>(B);
  const int acc = accumulate;
  if (!a_t && !b_t)
    k_gemm_bf16<false, false><<<grid, 128, 0, s>>>(a, lda, b, ldb, C, ldc, int(M), int(N), int(K), acc, kchunk);
  else if (!a_t && b_t)
    k_gemm_bf16<false, true><<<grid, 128, 0, s>>>(a, lda, b, ldb, C, ldc, int(M), int(N), int(K), acc, kchunk);
  else if (a_t && !b_t)
    k_gemm_bf16<true, false><<<grid, 128, 0, s>>>(a, lda, b, ldb, C, ldc, int(M), int(N), int(K), acc, kchunk);
  else
    k_gemm_bf16<true, true><<<grid, 128, 0, s>>>(a, lda, b, ldb, C, ldc, int(M), int(N), int(K), acc, kchunk);
  return launch_status();
}

extern "C" int tb_mlp_bias_silu(const float* C, const float* b, float* Z, void* Y, int64_t M, int64_t N,
                                tb_stream_t stream) {
  if (M <= 0 || N <= 0 || !C || !b || !Y) return BAD_ARG;
  int64_t n = M * N;
  k_bias_silu<<<unsigned(((n + 1) / 2 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(C, b, Z,
                                                                                     static_cast<__nv_bfloat16*>(Y),
                                                                         M, int(N));
  return launch_status();
}

extern "C" int tb_mlp_bias_out(const float* C, const float* b, float* Y, int64_t M, int64_t N, tb_stream_t stream) {
  if (M <= 0 || N <= 0 || !C || !b || !Y) return BAD_ARG;
  int64_t n = M * N;
  k_bias_out<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(C, b, Y, M, int(N));
  return launch_status();
}

extern "C" int tb_mlp_mse_grad(const float* Y, const float* T, const float* w, void* dY, float* loss_part, int64_t M,
                               int64_t N, int64_t n_out, tb_stream_t stream) {
  if (M <= 0 || N <= 0 || n_out <= 0 || n_out > N || !Y || !T || !dY || !loss_part) return BAD_ARG;
  int64_t n = M * N;
  k_mse_grad<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      Y, T, w, static_cast<__nv_bfloat16*>(dY), loss_part, M, int(N), int(n_out));
  return launch_status();
}

extern "C" int tb_mlp_silu_back(const float* dA, const float* Z, void* dZ, int64_t n, tb_stream_t stream) {
  if (n <= 0 || !dA || !Z || !dZ) return BAD_ARG;
  k_silu_back<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(dA, Z, static_cast<__nv_bfloat16*>(dZ), n);
  return launch_status();
}

extern "C" int tb_mlp_colsum(const void* dZ, float* db, int64_t M, int64_t N, tb_stream_t stream) {
  if (M <= 0 || N <= 0 || !dZ || !db) return BAD_ARG;
  k_colsum<<<unsigned(N), 256, 0, (cudaStream_t)stream>>>(static_cast<const __nv_bfloat16*>(dZ), db, M, int(N));
  return launch_status();
}

extern "C" int tb_mlp_adam(float* p, const float* g, float* m, float* v, void* pb, int64_t n, float lr, float b1,
                           float b2, float eps, int64_t step, tb_stream_t stream) {
  if (n <= 0 || !p || !g || !m || !v || !pb || step < 1) return BAD_ARG;
  float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  k_adam<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, static_cast<__nv_bfloat16*>(pb), n,
                                                                     lr, b1, b2, eps, c1, c2);
  return launch_status();
}

extern "C" int tb_mlp_features(const double* points, int64_t M, double r_max, double z_c, double z_half, void* X,
                               tb_stream_t stream) {
  if (M <= 0 || !points || !X || !(r_max > 0) || !(z_half > 0)) return BAD_ARG;
  MlpDomain d{r_max, z_c, z_half};
  k_features<<<unsigned((M + 255) / 256), 256, 0, (cudaStream_t)stream>>>(points, M, d,
                                                                          static_cast<__nv_bfloat16*>(X));
  return launch_status();
}
