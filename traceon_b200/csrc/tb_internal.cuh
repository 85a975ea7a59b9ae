// tb_internal.cuh -- small device and host helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include "tb_common.cuh"

namespace tb {

// Bounded waits inside kernels (an MMA chain's completion, a pipeline
// stage, a flag another CTA publishes) give up after this many SM clock
// cycles: ~1 s at 1.9 GHz, far beyond any wait of a healthy launch.
constexpr long long DEFAULT_WAIT_CYCLES = 2000000000LL;
// Waits that drain work already in flight before shared or tensor memory
// is given up (after a failure too) always use the default bound.
constexpr long long DRAIN_WAIT_CYCLES = DEFAULT_WAIT_CYCLES;

// The limit of the progress waits, read on the host at every launch and
// passed to the kernel (tb_set_wait_limit sets it; one value per process).
inline std::atomic<long long>& wait_limit_cycles() {
  static std::atomic<long long> v{DEFAULT_WAIT_CYCLES};
  return v;
}
inline long long wait_limit() { return wait_limit_cycles().load(std::memory_order_relaxed); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Status of the last kernel launch on this thread.
inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? OK : CUDA_ERR;
}

// Number of SMs of the current device (cached per device).
inline int num_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

// Axial series (radial.c:312-384): locate the interval of z on the equally
// spaced grid zi and evaluate the derivative polynomials first .. 8 (the
// field needs 1 .. 8, the potential 0, 2, 4, 6, 8).  Returns false outside
// [zi[0], zi[Nz-1]].
__host__ __device__ inline bool axial_eval(double z, const double* zi, const double* coeff, int64_t Nz,
                                           double* d, int first = 0) {
  double z0 = zi[0], zl = zi[Nz - 1];
  if (!(z0 <= z && z <= zl)) return false;
  double dz = zi[1] - zi[0];
  int64_t idx = (int64_t)((z - z0) / dz);
  if (idx < 0) idx = 0;
  if (idx > Nz - 2) idx = Nz - 2;
  double x = z - zi[idx];
  const double* C = coeff + idx * NDERIV * 6;
  for (int i = first; i < NDERIV; i++) {
    const double* c = C + i * 6;
    d[i] = ((((c[0] * x + c[1]) * x + c[2]) * x + c[3]) * x + c[4]) * x + c[5];
  }
  return true;
}

// potential_radial_derivs, radial.c:340-343
__host__ __device__ inline double axial_potential(const double* d, double r2) {
  return d[0] - r2 / 4 * d[2] + r2 * r2 / 64. * d[4] - r2 * r2 * r2 / 2304. * d[6] +
         r2 * r2 * r2 * r2 / 147456. * d[8];
}

// field_radial_derivs, radial.c:376-383
__host__ __device__ inline void axial_field(const double* d, const double* p, double r2, double* f) {
  double fr = 0.5 * (d[2] - r2 / 8 * d[4] + r2 * r2 / 192 * d[6] - r2 * r2 * r2 / 9216 * d[8]);
  double fz = -d[1] + r2 / 4 * d[3] - r2 * r2 / 64 * d[5] + r2 * r2 * r2 / 2304 * d[7];
  f[0] = p[0] * fr;
  f[1] = p[1] * fr;
  f[2] = fz;
}

}  // namespace tb
