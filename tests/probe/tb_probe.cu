// tb_probe.cu -- measurement and test helpers, built into libtb_probe.so
// beside the tests (not into the product library):
//   * an FP64 pipe throughput probe, the roofline denominator of the
//     FP64-bound kernels (the tracer's field sums, the fill and field
//     kernels): each thread runs 8 independent FMA chains, and the result is
//     written so the work cannot be removed;
//   * the device math of the ring-pair loops (tb_fastmath.cuh) evaluated on
//     arrays, for comparison with the CUDA library functions.
#include "../../traceon_b200/csrc/tb_common.cuh"
#include "../../traceon_b200/csrc/tb_internal.cuh"
#include "../../traceon_b200/csrc/tb_fastmath.cuh"
#include "tb_probe.h"

namespace tb {

__global__ void __launch_bounds__(256) k_fp64_fma(int64_t iters, double seed, double* out) {
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = seed + i + threadIdx.x;
  const double m = 0.9999999, c = 1e-7;
  for (int64_t k = 0; k < iters; k++) {
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = fma(a[i], m, c);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += a[i];
  if (s == 12345.678) out[0] = s;  // practically never taken
}

__global__ void k_probe_math(const double* __restrict__ x, int64_t n, int fn, double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = x[i], r;
  switch (fn) {
    case 0: r = rcp_nr(v); break;
    case 1: r = rsqrt_nr(v); break;
    case 2: r = log_bf(v); break;
    case 10: r = 1.0 / v; break;
    case 11: r = 1.0 / sqrt(v); break;
    default: r = log(v); break;
  }
  out[i] = r;
}

}  // namespace tb

extern "C" int tb_probe_math(const double* x, int64_t n, int fn, double* out, tb_probe_stream_t stream) {
  if (n < 0 || (n > 0 && (!x || !out))) return tb::BAD_ARG;
  if (n == 0) return tb::OK;
  tb::k_probe_math<<<unsigned((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, n, fn, out);
  return tb::launch_status();
}

extern "C" int tb_probe_fp64_fma(int blocks, int64_t iters, double* out, tb_probe_stream_t stream) {
  if (blocks <= 0 || iters <= 0 || !out) return tb::BAD_ARG;
  tb::k_fp64_fma<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0, out);
  return tb::launch_status();
}
