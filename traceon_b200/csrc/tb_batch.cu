// tb_batch.cu -- the batching workload's charge solve: the matrices of many
// geometries of uneven N filled, factored and solved in ONE persistent launch.
// The reference fills and solves one geometry at a time (traceon/solver.py:
// 160-180 for the solve, 204-232 for the fill).
//
// Every geometry's matrix is padded to T x T tiles of 64 x 64 (identity on
// the padded diagonal, zeros elsewhere) in a workspace that
// tb_batch_solve_plan lays out; the plan also lists the tile tasks:
//   FILL(g, i, j)  the tile's entries: the 16-point Gauss sums of
//                  radial.c:249-310 off the diagonal and the singular self
//                  terms on it (the device functions of the one-geometry
//                  fill, tb_fill.cuh)
//   FACT(g, i, j)  left-looking LU without pivoting, s = min(i, j):
//                  C = A_ij - sum_{k<s} L_ik U_kj (operands staged through
//                  shared memory by cp.async in a four-stage pipeline), then
//                  on the diagonal the tile's own LU and the inverses of both
//                  of its triangles, below the diagonal L_ij = C U_jj^-1,
//                  right of it U_ij = L_ii^-1 C
//   FWD(g, i)      y_i = L_ii^-1 (F_i - sum_{k<i} L_ik y_k)
//   BWD(g, i)      x_i = U_ii^-1 (y_i - sum_{k>i} U_ik x_k); the block's
//                  charges are written out and packed with their elements'
//                  Gauss rings into the tracer's source layout
// The list is ordered so that a task depends only on tasks before it: all
// FILL tasks; FACT step by step across the geometries with one step of
// lookahead (the two tiles next to the next diagonal tile, then that
// diagonal tile, then the rest of the step); FWD by block row; BWD by block
// row from the bottom.  The CTAs of a persistent grid draw task numbers from
// an atomic ticket and wait (bounded, on per-tile and per-block flags with
// release / acquire ordering) for their task's inputs.  A dependency always
// holds a smaller ticket, drawn by a CTA that is already running, so the
// waits end; one that runs out anyway sets the abort word, after which every
// CTA stops drawing tasks and the unfinished geometries keep status -1.
//
// No pivoting: these single-layer matrices factor stably without row
// exchanges (growth factor 1 on the synthetic lenses, charges within ~1e-13
// of LAPACK's).  A zero or non-finite pivot or charge marks the geometry
// TB_SINGULAR, and the host solves it again with the pivoted LU.
#include <climits>
#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "tb_fill.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

constexpr int BT = 64;      // tile edge
constexpr int BTH = 256;    // threads per CTA: a 16 x 16 grid, 4 x 4 tile entries each
constexpr int KC = 16;      // inner-dimension chunk of a staged GEMM stage
constexpr int NSTAGE = 4;   // cp.async pipeline depth
constexpr int LDT = BT + 1; // padded row of a whole tile in shared memory
constexpr int STAGE_DOUBLES = 2 * BT * KC;
constexpr int SMEM_DOUBLES = 2 * BT * LDT;  // two tiles (or the GEMM stages)
static_assert(NSTAGE * STAGE_DOUBLES <= 2 * BT * LDT, "the pipeline stages fit in the two tile buffers");
constexpr size_t BATCH_SMEM = SMEM_DOUBLES * sizeof(double);

enum BatchTaskType : int { TASK_FILL = 0, TASK_FACT = 1, TASK_FWD = 2, TASK_BWD = 3 };
constexpr int ST_FILLED = 1, ST_FINAL = 2;  // tile states
constexpr int CTL_TICKET = 0, CTL_ABORT = 1, CTL_WORDS = 32;

struct BatchArgs {
  const tb_batch_item_t* items;
  const int4* tasks;
  int64_t n_tasks;
  double* work;
  int* flags;
  double* src;     // (3, rings) packed sources, or null
  int64_t rings;
  int* status;
  long long wait_cycles;
};

__device__ __forceinline__ int b_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void b_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Thread 0's bounded wait for *f >= want.  A wait that runs out sets the
// abort word; an abort set by another CTA ends the wait too.
__device__ __noinline__ bool thread_wait(const BatchArgs& a, const int* f, int want) {
  if (b_ld_acquire(f) >= want) return true;
  int* abort_word = a.flags + CTL_ABORT;
  const long long t0 = clock64();
  unsigned ns = 32;
  for (;;) {
    if (b_ld_acquire(f) >= want) return true;
    if (*(volatile int*)abort_word) return false;
    if (clock64() - t0 > a.wait_cycles) {
      atomicExch(abort_word, 1);
      return false;
    }
    __nanosleep(ns);
    ns = ns < 1024 ? 2 * ns : 1024;
  }
}

// The CTA waits for f0 >= w0 and, when n > 1, f1 >= w1 and f2 >= w2 (thread
// 0 polls; the result and the acquired data reach the CTA through the
// barrier).
__device__ __forceinline__ bool cta_wait(const BatchArgs& a, int n, const int* f0, int w0, const int* f1 = nullptr,
                                         int w1 = 0, const int* f2 = nullptr, int w2 = 0, int* s_ok = nullptr) {
  if (threadIdx.x == 0) {
    bool ok = thread_wait(a, f0, w0);
    if (ok && n > 1) ok = thread_wait(a, f1, w1) && thread_wait(a, f2, w2);
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  const bool ok = *s_ok;
  __syncthreads();
  return ok;
}

__device__ __forceinline__ bool cta_wait1(const BatchArgs& a, const int* f, int want, int* s_ok) {
  return cta_wait(a, 1, f, want, nullptr, 0, nullptr, 0, s_ok);
}

// Every thread's stores of the task are done (barrier), then thread 0
// publishes the flag with release ordering.
__device__ __forceinline__ void publish(int* f, int v) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    b_st_release(f, v);
  }
}

__device__ __forceinline__ int* tile_flags(const BatchArgs& a, const tb_batch_item_t& it) {
  return a.flags + it.flag_off;
}

// ---------------------------------------------------------------- FILL
__device__ void task_fill(const BatchArgs& a, const tb_batch_item_t& it, int i, int j, double* sm) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t N = it.N, T = it.T, Np = T * BT;
  double* s_r = sm;
  double* s_z = sm + BT * (NQ + 1);
  double* s_w = sm + 2 * BT * (NQ + 1);
  // the Gauss rings of the tile's 64 columns (the jacobian buffer's values)
  for (int e = tid; e < BT * NQ; e += BTH) {
    const int c = e / NQ, k = e % NQ;
    const int64_t col = (int64_t)j * BT + c;
    double r = 0, z = 0, w = 0;
    if (col < N) {
      Cubic cu;
      cu.load(it.vertices + col * 12);
      double jj;
      cu.point(gauss_x(k), false, r, z, jj);
      w = gauss_w(k) * jj;
    }
    s_r[c * (NQ + 1) + k] = r;
    s_z[c * (NQ + 1) + k] = z;
    s_w[c * (NQ + 1) + k] = w;
  }
  __syncthreads();
  double* A = a.work + it.a_off;
#pragma unroll 1
  for (int aa = 0; aa < 4; aa++) {
    const int64_t row = (int64_t)i * BT + ty + 16 * aa;
#pragma unroll 1
    for (int bb = 0; bb < 4; bb++) {
      const int c = tx + 16 * bb;
      const int64_t col = (int64_t)j * BT + c;
      if (row == col && row < N) continue;  // self term below
      double v;
      if (row < N && col < N)
        v = fill_entry(it.vertices, it.types, it.values, row, s_r + c * (NQ + 1), s_z + c * (NQ + 1),
                       s_w + c * (NQ + 1));
      else
        v = row == col ? 1.0 : 0.0;
      A[row * Np + col] = v;
    }
  }
  if (i == j) {
    const int warp = tid >> 5, lane = tid & 31;
    for (int e = warp; e < BT; e += BTH / 32) {
      const int64_t el = (int64_t)i * BT + e;
      if (el >= N) break;
      const double v = self_term_warp(it.vertices, it.types, it.values, el, lane);
      if (lane == 0) A[el * Np + el] = v;
    }
  }
  publish(tile_flags(a, it) + (int64_t)i * T + j, ST_FILLED);
}

// ---------------------------------------------------------------- FACT
// C (registers) -= sum_{k<s} L_ik U_kj, the operands streamed through
// NSTAGE shared-memory stages of (64 x KC) and (KC x 64).
__device__ __forceinline__ void fact_gemm(const double* __restrict__ A, int64_t Np, int i, int j, int s,
                                          double* sm, double (&acc)[4][4]) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int nq = s * (BT / KC);
  auto issue = [&](int q) {
    const int k = q / (BT / KC), kc = q % (BT / KC);
    double* Ls = sm + (q % NSTAGE) * STAGE_DOUBLES;  // [64][KC]
    double* Us = Ls + BT * KC;                       // [KC][64]
    const double* Lg = A + (int64_t)i * BT * Np + (int64_t)k * BT + kc * KC;
    const double* Ug = A + ((int64_t)k * BT + kc * KC) * Np + (int64_t)j * BT;
#pragma unroll
    for (int e = tid; e < BT * KC / 2; e += BTH) {
      const int row = e / (KC / 2), part = e % (KC / 2);
      cp_async16(Ls + row * KC + part * 2, Lg + row * Np + part * 2);
    }
#pragma unroll
    for (int e = tid; e < KC * BT / 2; e += BTH) {
      const int row = e / (BT / 2), part = e % (BT / 2);
      cp_async16(Us + row * BT + part * 2, Ug + row * Np + part * 2);
    }
  };
#pragma unroll
  for (int q = 0; q < NSTAGE - 1; q++) {
    if (q < nq) issue(q);
    cp_async_commit();
  }
#pragma unroll 1
  for (int q = 0; q < nq; q++) {
    cp_async_wait<NSTAGE - 2>();
    __syncthreads();
    const double* Ls = sm + (q % NSTAGE) * STAGE_DOUBLES;
    const double* Us = Ls + BT * KC;
#pragma unroll
    for (int kk = 0; kk < KC; kk++) {
      double l[4], u[4];
#pragma unroll
      for (int aa = 0; aa < 4; aa++) l[aa] = Ls[(ty + 16 * aa) * KC + kk];
#pragma unroll
      for (int bb = 0; bb < 4; bb++) u[bb] = Us[kk * BT + tx + 16 * bb];
#pragma unroll
      for (int aa = 0; aa < 4; aa++)
#pragma unroll
        for (int bb = 0; bb < 4; bb++) acc[aa][bb] = fma(-l[aa], u[bb], acc[aa][bb]);
    }
    if (q + NSTAGE - 1 < nq) issue(q + NSTAGE - 1);
    cp_async_commit();
  }
  cp_async_wait<0>();
  __syncthreads();
}

// LU without pivoting of the tile D (shared, [64][LDT]) in place: per step
// the column below the pivot is scaled, then every thread updates its own
// entries (ty + 16 aa, tx + 16 bb) of the trailing block.  Returns false on a
// zero or non-finite pivot.
__device__ __forceinline__ bool diag_lu(double* D) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  bool good = true;
#pragma unroll 1
  for (int p = 0; p < BT; p++) {
    const double piv = D[p * LDT + p];
    good = good && fabs(piv) > 0.0 && isfinite(piv);
    if (tid > p && tid < BT) D[tid * LDT + p] /= piv;
    __syncthreads();
#pragma unroll
    for (int aa = 0; aa < 4; aa++) {
      const int r = ty + 16 * aa;
      if (r <= p) continue;
      const double l = D[r * LDT + p];
#pragma unroll
      for (int bb = 0; bb < 4; bb++) {
        const int c = tx + 16 * bb;
        if (c > p) D[r * LDT + c] = fma(-l, D[p * LDT + c], D[r * LDT + c]);
      }
    }
    __syncthreads();
  }
  return good;
}

// Inverses of the two triangles of the factored tile D (shared, [64][LDT]):
// M gets U^-1 on and above the diagonal and the strict lower part of L^-1
// (whose diagonal is 1).  Thread pairs own one column each (pairs 0-63 of
// U^-1, 64-127 of L^-1) and run the column's substitution, the pair's two
// halves splitting every dot product.
__device__ __forceinline__ void diag_inverses(const double* D, double* M) {
  const int tid = threadIdx.x, half = tid & 1, pair = tid >> 1;
  const bool upper = pair < BT;
  const int c = upper ? pair : pair - BT;
  if (upper && half == 0) M[c * LDT + c] = 1.0 / D[c * LDT + c];
  __syncwarp();
#pragma unroll 1
  for (int t = 0; t < BT - 1; t++) {
    double s = 0.0;
    int r;
    if (upper) {
      r = c - 1 - t;  // X[r][c] = -sum_{q=r+1..c} U[r][q] X[q][c] / U[r][r]
      if (r >= 0)
        for (int q = r + 1 + half; q <= c; q += 2) s = fma(D[r * LDT + q], M[q * LDT + c], s);
    } else {
      r = c + 1 + t;  // X[r][c] = -sum_{q=c..r-1} L[r][q] X[q][c], X[c][c] = 1
      if (r < BT)
        for (int q = c + half; q < r; q += 2) s = fma(D[r * LDT + q], q == c ? 1.0 : M[q * LDT + c], s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (half == 0) {
      if (upper && r >= 0) M[r * LDT + c] = -s / D[r * LDT + r];
      if (!upper && r < BT) M[r * LDT + c] = -s;
    }
    __syncwarp();
  }
}

__device__ bool task_fact(const BatchArgs& a, const tb_batch_item_t& it, int g, int i, int j, double* sm, int* s_ok) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t T = it.T, Np = T * BT;
  double* A = a.work + it.a_off;
  int* fl = tile_flags(a, it);
  const int s = i < j ? i : j;
  // this tile filled; the tiles of step s - 1 in its row and column final
  if (!cta_wait(a, s > 0 ? 3 : 1, fl + (int64_t)i * T + j, ST_FILLED, fl + (int64_t)i * T + (s - 1), ST_FINAL,
                fl + (int64_t)(s - 1) * T + j, ST_FINAL, s_ok))
    return false;
  double acc[4][4];
#pragma unroll
  for (int aa = 0; aa < 4; aa++)
#pragma unroll
    for (int bb = 0; bb < 4; bb++)
      acc[aa][bb] = __ldcg(A + ((int64_t)i * BT + ty + 16 * aa) * Np + (int64_t)j * BT + tx + 16 * bb);
  fact_gemm(A, Np, i, j, s, sm, acc);
  double* D = sm;
  double* M = sm + BT * LDT;
  if (i == j) {
#pragma unroll
    for (int aa = 0; aa < 4; aa++)
#pragma unroll
      for (int bb = 0; bb < 4; bb++) D[(ty + 16 * aa) * LDT + tx + 16 * bb] = acc[aa][bb];
    __syncthreads();
    const bool good = diag_lu(D);
    if (tid == 0 && !good) atomicOr(fl + T * T + 2 * T, 1);
    diag_inverses(D, M);
    __syncthreads();
    double* inv = a.work + it.inv_off + (int64_t)i * BT * BT;
    for (int e = tid; e < BT * BT; e += BTH) inv[e] = M[(e >> 6) * LDT + (e & 63)];
    publish(fl + (int64_t)i * T + j, ST_FINAL);
    return true;
  }
  if (!cta_wait1(a, fl + (int64_t)s * T + s, ST_FINAL, s_ok)) return false;
  const bool lower = i > j;
  const double* inv = a.work + it.inv_off + (int64_t)s * BT * BT;
#pragma unroll
  for (int aa = 0; aa < 4; aa++)
#pragma unroll
    for (int bb = 0; bb < 4; bb++) D[(ty + 16 * aa) * LDT + tx + 16 * bb] = acc[aa][bb];
  // below the diagonal U_ss^-1 (zeros under it), right of it L_ss^-1 (ones on
  // the diagonal, zeros above it)
  for (int e = tid; e < BT * BT; e += BTH) {
    const int r = e >> 6, c = e & 63;
    const double v = __ldcg(inv + e);
    M[r * LDT + c] = lower ? (r <= c ? v : 0.0) : (r > c ? v : (r == c ? 1.0 : 0.0));
  }
  __syncthreads();
  const double* X = lower ? D : M;  // out = X Y
  const double* Y = lower ? M : D;
  double out[4][4] = {};
#pragma unroll 4
  for (int q = 0; q < BT; q++) {
    double x[4], y[4];
#pragma unroll
    for (int aa = 0; aa < 4; aa++) x[aa] = X[(ty + 16 * aa) * LDT + q];
#pragma unroll
    for (int bb = 0; bb < 4; bb++) y[bb] = Y[q * LDT + tx + 16 * bb];
#pragma unroll
    for (int aa = 0; aa < 4; aa++)
#pragma unroll
      for (int bb = 0; bb < 4; bb++) out[aa][bb] = fma(x[aa], y[bb], out[aa][bb]);
  }
#pragma unroll
  for (int aa = 0; aa < 4; aa++)
#pragma unroll
    for (int bb = 0; bb < 4; bb++)
      A[((int64_t)i * BT + ty + 16 * aa) * Np + (int64_t)j * BT + tx + 16 * bb] = out[aa][bb];
  publish(fl + (int64_t)i * T + j, ST_FINAL);
  return true;
}

// ---------------------------------------------------------------- sweeps
// Thread (rr, part) = (tid / 4, tid % 4) owns row rr of a 64 x 64 block and
// its 16 columns part*16 .. part*16 + 15; the quad's partial sums meet by
// shuffles.
__device__ __forceinline__ double quad_sum(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v;
}

__device__ __forceinline__ double row_dot16(const double* __restrict__ m, const double* __restrict__ v) {
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int q = 0; q < 16; q += 2) {
    const double2 mm = __ldcg(reinterpret_cast<const double2*>(m + q));
    const double2 vv = __ldcg(reinterpret_cast<const double2*>(v + q));
    s0 = fma(mm.x, vv.x, s0);
    s1 = fma(mm.y, vv.y, s1);
  }
  return s0 + s1;
}

__device__ bool task_fwd(const BatchArgs& a, const tb_batch_item_t& it, int i, double* sm, int* s_ok) {
  const int tid = threadIdx.x, rr = tid >> 2, part = tid & 3;
  const int64_t T = it.T, Np = T * BT;
  const double* A = a.work + it.a_off;
  double* v = a.work + it.v_off;
  int* fl = tile_flags(a, it);
  int* yd = fl + T * T;
  // the diagonal tile final implies every tile left of it and above it
  if (!cta_wait1(a, fl + (int64_t)i * T + i, ST_FINAL, s_ok)) return false;
  const double* Lrow = A + ((int64_t)i * BT + rr) * Np + part * 16;
  double acc = 0.0;
#pragma unroll 1
  for (int k = 0; k < i; k++) {
    double l[16];
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
      const double2 mm = __ldcg(reinterpret_cast<const double2*>(Lrow + (int64_t)k * BT + q));
      l[q] = mm.x;
      l[q + 1] = mm.y;
    }
    if (!cta_wait1(a, yd + k, 1, s_ok)) return false;
    const double* yk = v + (int64_t)k * BT + part * 16;
#pragma unroll
    for (int q = 0; q < 16; q++) acc = fma(l[q], __ldcg(yk + q), acc);
  }
  acc = quad_sum(acc);
  double* s_r = sm;
  const int64_t row = (int64_t)i * BT + rr;
  if (part == 0) s_r[rr] = (row < it.N ? it.rhs[row] : 0.0) - acc;
  __syncthreads();
  // y = (I + strict lower part of the inverse tile) r
  const double* inv = a.work + it.inv_off + (int64_t)i * BT * BT + rr * BT;
  double y = 0.0;
#pragma unroll
  for (int q0 = 0; q0 < 16; q0++) {
    const int q = part * 16 + q0;
    const double m = q < rr ? __ldcg(inv + q) : (q == rr ? 1.0 : 0.0);
    y = fma(m, s_r[q], y);
  }
  y = quad_sum(y);
  if (part == 0) v[row] = y;
  publish(yd + i, 1);
  return true;
}

__device__ bool task_bwd(const BatchArgs& a, const tb_batch_item_t& it, int g, int i, double* sm, int* s_ok) {
  const int tid = threadIdx.x, rr = tid >> 2, part = tid & 3;
  const int64_t T = it.T, Np = T * BT, N = it.N;
  const double* A = a.work + it.a_off;
  double* v = a.work + it.v_off;
  int* fl = tile_flags(a, it);
  int* yd = fl + T * T;
  int* xd = yd + T;
  // the last forward block implies every factor tile and every y block
  if (!cta_wait1(a, yd + (T - 1), 1, s_ok)) return false;
  const double* Urow = A + ((int64_t)i * BT + rr) * Np + part * 16;
  double acc = 0.0;
#pragma unroll 1
  for (int64_t k = T - 1; k > i; k--) {
    double l[16];
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
      const double2 mm = __ldcg(reinterpret_cast<const double2*>(Urow + k * BT + q));
      l[q] = mm.x;
      l[q + 1] = mm.y;
    }
    if (!cta_wait1(a, xd + k, 1, s_ok)) return false;
    const double* xk = v + k * BT + part * 16;
#pragma unroll
    for (int q = 0; q < 16; q++) acc = fma(l[q], __ldcg(xk + q), acc);
  }
  acc = quad_sum(acc);
  double* s_r = sm;
  double* s_x = sm + BT;
  const int64_t row = (int64_t)i * BT + rr;
  if (part == 0) s_r[rr] = __ldcg(v + row) - acc;
  __syncthreads();
  // x = (upper part of the inverse tile, diagonal included) r
  const double* inv = a.work + it.inv_off + (int64_t)i * BT * BT + rr * BT;
  double x = 0.0;
#pragma unroll
  for (int q0 = 0; q0 < 16; q0++) {
    const int q = part * 16 + q0;
    const double m = q >= rr ? __ldcg(inv + q) : 0.0;
    x = fma(m, s_r[q], x);
  }
  x = quad_sum(x);
  if (part == 0) {
    v[row] = x;
    s_x[rr] = x;
    if (row < N) {
      it.charges[row] = x;
      if (!isfinite(x)) atomicOr(fl + T * T + 2 * T, 1);
    }
  }
  __syncthreads();
  if (a.src) {  // tb_pack_sources of the block's elements: r | z | charge x jacobian
    for (int e = tid; e < BT * NQ; e += BTH) {
      const int el = e / NQ, k = e % NQ;
      const int64_t elem = (int64_t)i * BT + el;
      if (elem >= N) continue;
      Cubic cu;
      cu.load(it.vertices + elem * 12);
      double r, z, jj;
      cu.point(gauss_x(k), false, r, z, jj);
      const int64_t ring = it.ring_off + elem * NQ + k;
      a.src[ring] = r;
      a.src[a.rings + ring] = z;
      a.src[2 * a.rings + ring] = s_x[el] * (gauss_w(k) * jj);
    }
  }
  publish(xd + i, 1);
  if (i == 0 && tid == 0) a.status[g] = *(volatile int*)(fl + T * T + 2 * T) ? SINGULAR : OK;
  return true;
}

__global__ void __launch_bounds__(BTH, 2) k_batch_solve(BatchArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_task, s_ok;
  int* ctl = a.flags;
  for (;;) {
    if (threadIdx.x == 0) {
      int t = atomicAdd(ctl + CTL_TICKET, 1);
      if (*(volatile int*)(ctl + CTL_ABORT)) t = INT_MAX;
      s_task = t;
    }
    __syncthreads();
    const int64_t t = s_task;
    if (t >= a.n_tasks) break;
    const int4 task = a.tasks[t];
    const tb_batch_item_t& it = a.items[task.y];
    switch (task.x) {
      case TASK_FILL:
        task_fill(a, it, task.z, task.w, sm);
        break;
      case TASK_FACT:
        task_fact(a, it, task.y, task.z, task.w, sm, &s_ok);
        break;
      case TASK_FWD:
        task_fwd(a, it, task.z, sm, &s_ok);
        break;
      default:
        task_bwd(a, it, task.y, task.z, sm, &s_ok);
        break;
    }
    __syncthreads();  // shared buffers and s_task are reused by the next task
  }
}

}  // namespace tb

using namespace tb;

extern "C" int64_t tb_batch_solve_plan(tb_batch_item_t* items, int n_items, int32_t* tasks, int64_t* sizes) {
  if (!items || n_items <= 0 || !sizes) return -1;
  int64_t wd = 0, fw = CTL_WORDS, rings = 0, tmax = 0;
  for (int g = 0; g < n_items; g++) {
    tb_batch_item_t& it = items[g];
    if (it.N <= 0 || it.N > (int64_t)1 << 20) return -1;
    const int64_t T = (it.N + BT - 1) / BT, Np = T * BT;
    it.T = T;
    it.a_off = wd;
    wd += Np * Np;
    it.inv_off = wd;
    wd += T * BT * BT;
    it.v_off = wd;
    wd += Np;
    it.flag_off = fw;
    fw += T * T + 2 * T + 1;
    it.ring_off = rings;
    rings += it.N * NQ;
    if (T > tmax) tmax = T;
  }
  if (fw > INT_MAX) return -1;
  sizes[0] = wd;
  sizes[1] = fw;
  sizes[2] = rings;
  int64_t n = 0;
  auto put = [&](int type, int g, int64_t i, int64_t j) {
    if (tasks) {
      tasks[4 * n] = type;
      tasks[4 * n + 1] = g;
      tasks[4 * n + 2] = int32_t(i);
      tasks[4 * n + 3] = int32_t(j);
    }
    n++;
  };
  for (int g = 0; g < n_items; g++)
    for (int64_t i = 0; i < items[g].T; i++)
      for (int64_t j = 0; j < items[g].T; j++) put(TASK_FILL, g, i, j);
  for (int g = 0; g < n_items; g++) put(TASK_FACT, g, 0, 0);
  for (int64_t s = 0; s < tmax; s++) {
    for (int g = 0; g < n_items; g++)
      if (items[g].T > s + 1) {
        put(TASK_FACT, g, s + 1, s);
        put(TASK_FACT, g, s, s + 1);
      }
    for (int g = 0; g < n_items; g++)
      if (items[g].T > s + 1) put(TASK_FACT, g, s + 1, s + 1);
    for (int g = 0; g < n_items; g++)
      for (int64_t t = 2; s + t < items[g].T; t++) {
        put(TASK_FACT, g, s + t, s);
        put(TASK_FACT, g, s, s + t);
      }
  }
  for (int64_t i = 0; i < tmax; i++)
    for (int g = 0; g < n_items; g++)
      if (items[g].T > i) put(TASK_FWD, g, i, 0);
  for (int64_t m = 0; m < tmax; m++)
    for (int g = 0; g < n_items; g++)
      if (items[g].T > m) put(TASK_BWD, g, items[g].T - 1 - m, 0);
  return n;
}

extern "C" int tb_batch_solve(const tb_batch_item_t* items, int n_items, const int32_t* tasks, int64_t n_tasks,
                              double* work, int32_t* flags, int64_t n_flags, double* sources, int64_t total_rings,
                              int32_t* status, int blocks_per_sm, tb_stream_t stream) {
  if (!items || n_items <= 0 || !tasks || n_tasks <= 0 || n_tasks > INT_MAX / 2 || !work || !flags ||
      n_flags < CTL_WORDS || !status || (sources && total_rings <= 0) || blocks_per_sm < 0)
    return BAD_ARG;
  if ((reinterpret_cast<uintptr_t>(work) & 15) != 0) return BAD_ARG;  // 16-byte cp.async sources
  cudaStream_t s = (cudaStream_t)stream;
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CUDA_ERR;
  if (dev < 0 || dev >= 64) return BAD_ARG;
  if (!attr[dev]) {
    if (cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, int(BATCH_SMEM)) !=
        cudaSuccess)
      return CUDA_ERR;
    attr[dev] = true;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve, BTH, BATCH_SMEM) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
  int64_t blocks = (int64_t)num_sms() * per_sm;
  if (blocks > n_tasks) blocks = n_tasks;
  if (cudaMemsetAsync(flags, 0, size_t(n_flags) * sizeof(int32_t), s) != cudaSuccess) return CUDA_ERR;
  if (cudaMemsetAsync(status, 0xff, size_t(n_items) * sizeof(int32_t), s) != cudaSuccess) return CUDA_ERR;
  BatchArgs a;
  a.items = items;
  a.tasks = reinterpret_cast<const int4*>(tasks);
  a.n_tasks = n_tasks;
  a.work = work;
  a.flags = flags;
  a.src = sources;
  a.rings = total_rings;
  a.status = status;
  a.wait_cycles = wait_limit();
  k_batch_solve<<<unsigned(blocks), BTH, BATCH_SMEM, s>>>(a);
  return launch_status();
}
