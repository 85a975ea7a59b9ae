// tb_mlp.cuh -- the field-surrogate network: sizes, parameter layout, input
// features, activation, and the warp-level forward pass used inside the
// tracer.  The network is 16 features -> 4 x 128 (SiLU) -> 32 outputs, BF16
// weights and activations with FP32 accumulation on the tensor cores
// (mma.sync m16n8k16).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace tb {

constexpr int MLP_IN = 16;
constexpr int MLP_H = 128;
constexpr int MLP_OUT = 32;
// Field sources of a surrogate: electrodes (per unit voltage) and current
// coils (per unit current), 3 outputs each -- (phi, E_r, E_z) of an
// electrode, (magnetostatic potential, H_r, H_z) of a coil -- in columns
// 3 s .. 3 s + 2 of source s (electrodes first).
constexpr int MLP_MAX_SOURCES = MLP_OUT / 3;  // 10

// Flat parameter layout: W1 (H x IN), b1 (H), W2, b2, W3, b3, W4, b4 (H x H, H),
// W5 (OUT x H), b5 (OUT).  Weights are row-major [out][in].
constexpr int64_t MLP_OFF_W1 = 0;
constexpr int64_t MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN;
constexpr int64_t MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int64_t MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int64_t MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int64_t MLP_OFF_B3 = MLP_OFF_W3 + MLP_H * MLP_H;
constexpr int64_t MLP_OFF_W4 = MLP_OFF_B3 + MLP_H;
constexpr int64_t MLP_OFF_B4 = MLP_OFF_W4 + MLP_H * MLP_H;
constexpr int64_t MLP_OFF_W5 = MLP_OFF_B4 + MLP_H;
constexpr int64_t MLP_OFF_B5 = MLP_OFF_W5 + MLP_OUT * MLP_H;
constexpr int64_t MLP_NPARAM = MLP_OFF_B5 + MLP_OUT;

// Normalisation of the inputs: rho = r / r_max, zeta = (z - z_c) / z_half.
struct MlpDomain {
  double r_max, z_c, z_half;
};

// SiLU through a single hardware tanh: silu(z) = z sigmoid(z) = h + h tanh(h)
// with h = z / 2, in FP32 (tanh.approx.f32, one MUFU operation; maximum
// relative error about 2^-11, below the BF16 rounding of the activations
// that follows), the pair rounded to BF16 once at the end.  Training (the
// forward pass of k_bias_silu) and both tracer engines evaluate the same
// function; the backward pass uses its FP32 derivative.  (A packed form --
// h rounded to BF16, tanh.approx.bf16x2, fma.rn.bf16x2 -- halves the MUFU
// operations but raised the trained network's held-out error by 30-40 %
// with no measurable gain in tracer speed, so it is not used.)
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// BF16 pair {silu(z0), silu(z1)} from the halved pre-activations
// h0 = z0 / 2, h1 = z1 / 2 (h0 in the low half).
__device__ __forceinline__ uint32_t silu2_bf16_half(float h0, float h1) {
  __nv_bfloat162 v = __floats2bfloat162_rn(fmaf(h0, tanh_fast(h0), h0), fmaf(h1, tanh_fast(h1), h1));
  return *reinterpret_cast<uint32_t*>(&v);
}
// The same from the accumulators a0, a1 and the halved biases b0, b1
// (h = a + b), with the additions and the multiply-adds as packed FP32x2
// operations (add.rn.f32x2, fma.rn.f32x2: each half rounded exactly as the
// scalar operation, so the result equals silu2_bf16_half(a0 + b0, a1 + b1)).
__device__ __forceinline__ uint32_t silu2_bf16_half_bias(float a0, float a1, float b0, float b1) {
  float h0 = a0, h1 = a1;
  asm("{.reg .b64 x, y;\n mov.b64 x, {%0, %1};\n mov.b64 y, {%2, %3};\n add.rn.f32x2 x, x, y;\n"
      " mov.b64 {%0, %1}, x;}"
      : "+f"(h0), "+f"(h1)
      : "f"(b0), "f"(b1));
  const float t0 = tanh_fast(h0), t1 = tanh_fast(h1);
  float y0 = h0, y1 = h1;
  asm("{.reg .b64 x, y, z;\n mov.b64 x, {%2, %3};\n mov.b64 y, {%4, %5};\n mov.b64 z, {%0, %1};\n"
      " fma.rn.f32x2 z, x, y, z;\n mov.b64 {%0, %1}, z;}"
      : "+f"(y0), "+f"(y1)
      : "f"(h0), "f"(h1), "f"(t0), "f"(t1));
  __nv_bfloat162 v = __floats2bfloat162_rn(y0, y1);
  return *reinterpret_cast<uint32_t*>(&v);
}
// BF16 pair {silu(z0), silu(z1)} (z0 in the low half).
__device__ __forceinline__ uint32_t silu2_bf16(float z0, float z1) { return silu2_bf16_half(0.5f * z0, 0.5f * z1); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = fmaf(0.5f, tanh_fast(0.5f * z), 0.5f);  // sigmoid(z)
  return s * fmaf(z, 1.f - s, 1.f);
}

// Input features of a point (r, z): polynomial terms in rho^2 and zeta (the
// field is even in r) and five Fourier pairs in zeta, sin/cos(k pi zeta) for
// k = 1..5, the higher harmonics by the angle-addition recurrence.
__device__ __forceinline__ void mlp_features(double r, double z, const MlpDomain& d, float* f) {
  float rho = float(r / d.r_max), zeta = float((z - d.z_c) / d.z_half);
  float p = rho * rho;
  f[0] = p;
  f[1] = zeta;
  f[2] = p * zeta;
  f[3] = zeta * zeta;
  f[4] = p * p;
  f[5] = p * zeta * zeta;
  float s1, c1;
  sincospif(zeta, &s1, &c1);
  float s = s1, c = c1;
#pragma unroll
  for (int k = 1; k <= 5; k++) {
    f[4 + 2 * k] = s;
    f[5 + 2 * k] = c;
    const float sn = fmaf(s, c1, c * s1);
    c = fmaf(c, c1, -s * s1);
    s = sn;
  }
}

// D (16x8, fp32) += A (16x16, bf16, row) . B (16x8, bf16, col).
__device__ __forceinline__ void mma_bf16_16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Shared-memory image of the network for the warp-level forward pass.
constexpr int MLP_LD_IN = MLP_IN + 8;  // padded row strides (bf16 elements)
constexpr int MLP_LD_H = MLP_H + 8;
struct MlpSmem {
  __nv_bfloat16 w1[MLP_H][MLP_LD_IN];
  __nv_bfloat16 wh[3][MLP_H][MLP_LD_H];  // W2, W3, W4
  __nv_bfloat16 w5[MLP_OUT][MLP_LD_H];
  float b1[MLP_H], bh[3][MLP_H], b5[MLP_OUT];
};

// Copies the BF16 weights and FP32 biases (flat layout above) into shared
// memory; all threads of the block take part.
__device__ inline void mlp_load_smem(MlpSmem& s, const __nv_bfloat16* __restrict__ wb,
                                     const float* __restrict__ pf) {
  for (int e = threadIdx.x; e < MLP_H * MLP_IN; e += blockDim.x) s.w1[e / MLP_IN][e % MLP_IN] = wb[MLP_OFF_W1 + e];
  for (int e = threadIdx.x; e < MLP_H * MLP_H; e += blockDim.x) {
    s.wh[0][e / MLP_H][e % MLP_H] = wb[MLP_OFF_W2 + e];
    s.wh[1][e / MLP_H][e % MLP_H] = wb[MLP_OFF_W3 + e];
    s.wh[2][e / MLP_H][e % MLP_H] = wb[MLP_OFF_W4 + e];
  }
  for (int e = threadIdx.x; e < MLP_OUT * MLP_H; e += blockDim.x) s.w5[e / MLP_H][e % MLP_H] = wb[MLP_OFF_W5 + e];
  for (int e = threadIdx.x; e < MLP_H; e += blockDim.x) {
    s.b1[e] = pf[MLP_OFF_B1 + e];
    s.bh[0][e] = pf[MLP_OFF_B2 + e];
    s.bh[1][e] = pf[MLP_OFF_B3 + e];
    s.bh[2][e] = pf[MLP_OFF_B4 + e];
  }
  for (int e = threadIdx.x; e < MLP_OUT; e += blockDim.x) s.b5[e] = pf[MLP_OFF_B5 + e];
}

// One hidden layer for one 16-row m-tile held in A fragments `a` (K = 128,
// 8 k-blocks): produces the next layer's A fragments after bias + SiLU.
// The C fragment of two adjacent n8 tiles is exactly the A fragment of one
// k16 block, so activations never leave registers.
__device__ __forceinline__ void mlp_hidden_layer(const __nv_bfloat16 (*W)[MLP_LD_H], const float* bias,
                                                 const uint32_t (&a)[8][4], uint32_t (&out)[8][4], int g, int q) {
#pragma unroll
  for (int kb = 0; kb < 8; kb++) {  // output columns 16 kb .. 16 kb + 15
    // two partial sums per n8 tile (even / odd k-blocks): four independent
    // accumulation chains instead of two
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
    float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int ki = 0; ki < 8; ki++) {
      uint32_t b0[2], b1[2];
      int n0 = 16 * kb + g, n1 = 16 * kb + 8 + g;
      b0[0] = *reinterpret_cast<const uint32_t*>(&W[n0][16 * ki + 2 * q]);
      b0[1] = *reinterpret_cast<const uint32_t*>(&W[n0][16 * ki + 8 + 2 * q]);
      b1[0] = *reinterpret_cast<const uint32_t*>(&W[n1][16 * ki + 2 * q]);
      b1[1] = *reinterpret_cast<const uint32_t*>(&W[n1][16 * ki + 8 + 2 * q]);
      if (ki & 1) {
        mma_bf16_16816(d0, a[ki], b0);
        mma_bf16_16816(d1, a[ki], b1);
      } else {
        mma_bf16_16816(c0, a[ki], b0);
        mma_bf16_16816(c1, a[ki], b1);
      }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      c0[c] += d0[c];
      c1[c] += d1[c];
    }
    int col0 = 16 * kb + 2 * q, col1 = 16 * kb + 8 + 2 * q;
    out[kb][0] = silu2_bf16(c0[0] + bias[col0], c0[1] + bias[col0 + 1]);
    out[kb][1] = silu2_bf16(c0[2] + bias[col0], c0[3] + bias[col0 + 1]);
    out[kb][2] = silu2_bf16(c1[0] + bias[col1], c1[1] + bias[col1 + 1]);
    out[kb][3] = silu2_bf16(c1[2] + bias[col1], c1[3] + bias[col1 + 1]);
  }
}

// Forward pass of the network for the 32 points of a warp.  `feat` is the
// warp's [32][MLP_IN] feature block and `out` its [32][MLP_OUT] result block
// in shared memory; every lane writes its row of `feat` before the call and
// reads its row of `out` after it.
__device__ inline void mlp_warp_forward(const MlpSmem& s, const __nv_bfloat16 (*feat)[MLP_LD_IN],
                                        float (*out)[MLP_OUT]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  __syncwarp();
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    const int r0 = 16 * mt + g, r1 = r0 + 8;
    // layer 1: K = 16 (one k-block)
    uint32_t a1[4];
    a1[0] = *reinterpret_cast<const uint32_t*>(&feat[r0][2 * q]);
    a1[1] = *reinterpret_cast<const uint32_t*>(&feat[r1][2 * q]);
    a1[2] = *reinterpret_cast<const uint32_t*>(&feat[r0][8 + 2 * q]);
    a1[3] = *reinterpret_cast<const uint32_t*>(&feat[r1][8 + 2 * q]);
    uint32_t h[8][4], h2[8][4];
#pragma unroll
    for (int kb = 0; kb < 8; kb++) {
      float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t b0[2], b1[2];
      int n0 = 16 * kb + g, n1 = 16 * kb + 8 + g;
      b0[0] = *reinterpret_cast<const uint32_t*>(&s.w1[n0][2 * q]);
      b0[1] = *reinterpret_cast<const uint32_t*>(&s.w1[n0][8 + 2 * q]);
      b1[0] = *reinterpret_cast<const uint32_t*>(&s.w1[n1][2 * q]);
      b1[1] = *reinterpret_cast<const uint32_t*>(&s.w1[n1][8 + 2 * q]);
      mma_bf16_16816(c0, a1, b0);
      mma_bf16_16816(c1, a1, b1);
      int col0 = 16 * kb + 2 * q, col1 = 16 * kb + 8 + 2 * q;
      h[kb][0] = silu2_bf16(c0[0] + s.b1[col0], c0[1] + s.b1[col0 + 1]);
      h[kb][1] = silu2_bf16(c0[2] + s.b1[col0], c0[3] + s.b1[col0 + 1]);
      h[kb][2] = silu2_bf16(c1[0] + s.b1[col1], c1[1] + s.b1[col1 + 1]);
      h[kb][3] = silu2_bf16(c1[2] + s.b1[col1], c1[3] + s.b1[col1 + 1]);
    }
    // the three hidden layers share one copy of the code (smaller kernel:
    // fewer instruction-fetch stalls)
#pragma unroll 1
    for (int l = 0; l < 3; l++) {
      mlp_hidden_layer(s.wh[l], s.bh[l], h, h2, g, q);
#pragma unroll
      for (int kb = 0; kb < 8; kb++)
#pragma unroll
        for (int c = 0; c < 4; c++) h[kb][c] = h2[kb][c];
    }
    // output layer: N = MLP_OUT (MLP_OUT / 8 n8 tiles), FP32 results
    constexpr int NT = MLP_OUT / 8;
    float c[NT][4];
#pragma unroll
    for (int t = 0; t < NT; t++) c[t][0] = c[t][1] = c[t][2] = c[t][3] = 0.f;
#pragma unroll
    for (int ki = 0; ki < 8; ki++) {
#pragma unroll
      for (int t = 0; t < NT; t++) {
        uint32_t b[2];
        b[0] = *reinterpret_cast<const uint32_t*>(&s.w5[8 * t + g][16 * ki + 2 * q]);
        b[1] = *reinterpret_cast<const uint32_t*>(&s.w5[8 * t + g][16 * ki + 8 + 2 * q]);
        mma_bf16_16816(c[t], h2[ki], b);
      }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const int col = 8 * t + 2 * q;
      out[r0][col] = c[t][0] + s.b5[col];
      out[r0][col + 1] = c[t][1] + s.b5[col + 1];
      out[r1][col] = c[t][2] + s.b5[col];
      out[r1][col + 1] = c[t][3] + s.b5[col + 1];
    }
  }
  __syncwarp();
}

}  // namespace tb
