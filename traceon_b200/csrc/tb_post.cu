// tb_post.cu -- trajectory post-processing on the device, for traces that
// stay in device memory: the plane crossing of every stored trajectory
// (plane_intersection, traceon/backend/tracing.c:184-223, behind
// traceon/tracing.py:247-335) and the least-squares focus of a beam
// (focus_position, traceon/focus.py:9-42).
#include <cmath>

#include "tb_internal.cuh"
#include "traceon_b200.h"

namespace tb {

// Signed distance of the point s[0..2] from the plane through p0 with normal
// nv, written as tracing.c:195 writes it.
__device__ __forceinline__ double plane_kappa(const double* s, double3 p0, double3 nv, double nn) {
  return (nv.z * p0.z - s[2] * nv.z + nv.y * p0.y - s[1] * nv.y + nv.x * p0.x - s[0] * nv.x) / nn;
}

// One warp per trajectory.  The reference walks from the last row towards
// the first and stops at the first sign change of kappa (sign: kappa > 0 or
// not) between rows i and i + 1; here 32 consecutive pairs are tested per
// pass, from the end, and the lowest lane of the ballot is the largest such
// i.  The crossing interpolates all 7 columns (t, x..vz) linearly with the
// reference's weights.
__global__ void k_plane_rows(const double* __restrict__ rows, const int64_t* __restrict__ nrows, int64_t n,
                             int64_t max_rows, double3 p0, double3 nv, double nn, double* __restrict__ out,
                             int32_t* __restrict__ found) {
  const int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x % 32;
  if (k >= n) return;  // whole warps
  const double* R = rows + k * max_rows * 7;
  int64_t np = nrows[k];
  np = np < 0 ? 0 : (np > max_rows ? max_rows : np);
  for (int64_t base = np - 2; base >= 0; base -= 32) {
    const int64_t i = base - lane;
    double ki = 0.0, ki1 = 0.0;
    bool change = false;
    if (i >= 0) {
      ki = plane_kappa(R + i * 7 + 1, p0, nv, nn);
      ki1 = plane_kappa(R + (i + 1) * 7 + 1, p0, nv, nn);
      change = (ki > 0) != (ki1 > 0);
    }
    const unsigned m = __ballot_sync(0xffffffffu, change);
    if (m) {
      if (lane == __ffs(m) - 1) {
        const double diff = ki - ki1;
        const double factor = -ki1 / diff, prev_factor = ki / diff;
        for (int c = 0; c < 7; c++) out[k * 7 + c] = prev_factor * R[(i + 1) * 7 + c] + factor * R[i * 7 + c];
        found[k] = 1;
      }
      return;
    }
  }
  if (lane == 0) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int c = 0; c < 7; c++) out[k * 7 + c] = nan;
    found[k] = 0;
  }
}

// ---------------------------------------------------------------- focus
// focus.py solves min || A (z, x, y) - b || with, per particle, the rows
// (-ax, 1, 0) . (z, x, y) = x - z_e ax and (-ay, 0, 1) . (z, x, y) = y - z_e ay
// (ax = vx / vz, ay = vy / vz at the final state).  For fixed z the best x,
// y are the means of bx + ax z, by + ay z (bx = x - z_e ax, by = y - z_e ay),
// which leaves a one-dimensional problem in z:
//   z = -sum(dax dbx + day dby) / sum(dax^2 + day^2),  d = deviation from the mean
// -- the same minimiser as the reference's lstsq for a full-rank system,
// computed from centred sums (two passes) so that it does not lose the
// digits the normal equations would.  The system counts as rank deficient
// (lstsq would return its minimum-norm solution; here NaN) when the spread
// of the final directions, sum(dax^2 + day^2), is below 1e-26 of
// sum(ax^2 + ay^2) -- directions equal to about 13 digits.  Sums are per
// block in a fixed grid-stride order, then over blocks in a fixed order:
// deterministic.
constexpr int FOCUS_BLOCKS = 296, FOCUS_THREADS = 256;

__device__ __forceinline__ void focus_terms(const double* s, double& ax, double& ay, double& bx, double& by) {
  ax = s[3] / s[5];
  ay = s[4] / s[5];
  bx = s[0] - s[2] * ax;
  by = s[1] - s[2] * ay;
}

// Sum over the CTA (256 threads) in a fixed order; the result is valid in
// every thread.
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();  // red may still be read by a previous call
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < FOCUS_THREADS / 32; w++) t += red[w];
  return t;
}

// The means of ax, ay, bx, by and of ax^2 + ay^2 from the first pass's
// block sums (part1[b * 5 + q]).
__device__ void focus_means(const double* __restrict__ part1, int64_t n, double* mean, double* red) {
  for (int q = 0; q < 5; q++) {
    double v = 0.0;
    for (int b = threadIdx.x; b < FOCUS_BLOCKS; b += blockDim.x) v += part1[b * 5 + q];
    mean[q] = block_sum(v, red) / double(n);
  }
}

template <int PASS>
__global__ void __launch_bounds__(FOCUS_THREADS) k_focus_sums(const double* __restrict__ S, int64_t n, int64_t ld,
                                                              double* __restrict__ part1, double* __restrict__ part2) {
  __shared__ double red[FOCUS_THREADS / 32];
  double mean[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (PASS == 1) focus_means(part1, n, mean, red);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double ax, ay, bx, by;
    focus_terms(S + i * ld, ax, ay, bx, by);
    if (PASS == 0) {
      acc[0] += ax;
      acc[1] += ay;
      acc[2] += bx;
      acc[3] += by;
      acc[4] += ax * ax + ay * ay;
    } else {
      const double dax = ax - mean[0], day = ay - mean[1], dbx = bx - mean[2], dby = by - mean[3];
      acc[0] += dax * dbx + day * dby;
      acc[1] += dax * dax + day * day;
    }
  }
  if (PASS == 0) {
    for (int q = 0; q < 5; q++) {
      const double t = block_sum(acc[q], red);
      if (threadIdx.x == 0) part1[blockIdx.x * 5 + q] = t;
    }
  } else {
    for (int q = 0; q < 2; q++) {
      const double t = block_sum(acc[q], red);
      if (threadIdx.x == 0) part2[blockIdx.x * 2 + q] = t;
    }
  }
}

// out = (x, y, z) of the focus; NaN when the system is rank deficient
// (final directions equal, or fewer than two particles).
__global__ void __launch_bounds__(FOCUS_THREADS) k_focus_final(const double* __restrict__ part1,
                                                               const double* __restrict__ part2, int64_t n,
                                                               double* __restrict__ out) {
  __shared__ double red[FOCUS_THREADS / 32];
  double mean[5];
  focus_means(part1, n, mean, red);
  double s[2];
  for (int q = 0; q < 2; q++) {
    double v = 0.0;
    for (int b = threadIdx.x; b < FOCUS_BLOCKS; b += blockDim.x) v += part2[b * 2 + q];
    s[q] = block_sum(v, red);
  }
  if (threadIdx.x == 0) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (!(s[1] > 1e-26 * mean[4] * double(n)) || n < 2) {
      out[0] = out[1] = out[2] = nan;
    } else {
      const double z = -s[0] / s[1];
      out[0] = mean[2] + mean[0] * z;
      out[1] = mean[3] + mean[1] * z;
      out[2] = z;
    }
  }
}

}  // namespace tb

using namespace tb;

extern "C" int tb_plane_intersection_rows(const double* rows, const int64_t* nrows, int64_t n, int64_t max_rows,
                                          const double* p0, const double* normal, double* out, int32_t* found,
                                          tb_stream_t stream) {
  if (n < 0 || max_rows < 0 || !p0 || !normal) return BAD_ARG;
  if (n == 0) return OK;
  if (!rows || !nrows || !out || !found || max_rows == 0) return BAD_ARG;
  const double nn = std::sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
  if (!(nn > 0.0) || !std::isfinite(nn)) return BAD_ARG;
  const int64_t threads = n * 32;
  k_plane_rows<<<unsigned((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      rows, nrows, n, max_rows, make_double3(p0[0], p0[1], p0[2]), make_double3(normal[0], normal[1], normal[2]), nn,
      out, found);
  return launch_status();
}

extern "C" int64_t tb_focus_position_workspace(void) { return int64_t(FOCUS_BLOCKS) * 7 * int64_t(sizeof(double)); }

extern "C" int tb_focus_position(const double* states, int64_t n, int64_t ld, double* out, void* work,
                                 int64_t work_bytes, tb_stream_t stream) {
  if (n < 0 || ld < 6 || !out || !work || work_bytes < tb_focus_position_workspace()) return BAD_ARG;
  if (n > 0 && !states) return BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  double* part1 = static_cast<double*>(work);
  double* part2 = part1 + FOCUS_BLOCKS * 5;
  k_focus_sums<0><<<FOCUS_BLOCKS, FOCUS_THREADS, 0, s>>>(states, n, ld, part1, part2);
  k_focus_sums<1><<<FOCUS_BLOCKS, FOCUS_THREADS, 0, s>>>(states, n, ld, part1, part2);
  k_focus_final<<<1, FOCUS_THREADS, 0, s>>>(part1, part2, n, out);
  return launch_status();
}
