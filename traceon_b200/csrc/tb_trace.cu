// tb_trace.cu -- persistent adaptive RKF45 tracer (tracing.c:60-123) for many
// particles at once.
//
// Particles are pulled from a device work queue by teams.  For BEM fields a
// team is 1-8 warps that split the ring sums of every field evaluation
// (field_radial_traceable, tracing.c:125-165) and reduce them with shuffles
// (and a named barrier across warps); every lane of a team then holds the
// same field bits, so the step control runs redundantly and uniformly in all
// lanes.  For axial-interpolated fields (field_radial_derivs_traceable,
// tracing.c:168-174) a team is one thread.
//
// Step control is the reference's: Fehlberg 4(5) tableau, error = max|pos
// err| + h max|vel err|, accept if error <= atol, h <- min(0.9 h
// (atol/error)^(1/5), hmax) after every attempt, hmax = 0.01 / |v0|, stop
// when the state leaves the inclusive bounds.  Unlike the reference, every
// particle has a cap on step attempts and a non-finite check, so a trapped or
// broken particle ends with a status instead of looping forever.
#include <cstddef>
#include <cstring>

#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "tb_mlp.cuh"
#include "tb_tc.cuh"
#include "../../include/traceon_b200.h"

namespace tb {

struct TraceParams {
  const double* esrc;
  int64_t ne;
  const double* msrc;
  int64_t nm;
  const double* csrc;
  int64_t nc;
  const double* fb;
  const double* az;
  const double* aec;
  const double* amc;
  int64_t anz;
  double bounds[6];
  double atol;
  double plane_z;
  int record_plane;
  int64_t max_attempts;
  int64_t max_rows;
  const double* start;
  const double* t0;
  const double* qm;
  int64_t n;
  double* rows;
  int64_t* nrows;
  int32_t* status;
  double* final_state;
  double* plane;
  int64_t* counters;
  int32_t* work;
  // many geometries in one launch (BEM tracer): particle i sums the rings
  // eoff[geom[i]] .. eoff[geom[i] + 1] - 1 of esrc; geom == nullptr: all of them
  const int32_t* geom = nullptr;
  const int64_t* eoff = nullptr;
  int64_t ngeom = 0;
  const double* gbounds = nullptr;  // (ngeom, 6) per-geometry bounds, or null: bounds
  long long wait_cycles = DEFAULT_WAIT_CYCLES;  // bound of the engine's progress waits
};

// Fehlberg 4(5) tableau, tracing.c:9-16
__constant__ double RK_B[6][5] = {{0, 0, 0, 0, 0},
                                  {2. / 9., 0, 0, 0, 0},
                                  {1. / 12., 1. / 4., 0, 0, 0},
                                  {69. / 128., -243. / 128., 135. / 64., 0, 0},
                                  {-17. / 12., 27. / 4., -27. / 5., 16. / 15., 0},
                                  {65. / 432., -5. / 16., 13. / 16., 4. / 27., 5. / 144.}};
__constant__ double RK_CH[6] = {47. / 450., 0., 12. / 25., 32. / 225., 1. / 30., 6. / 25.};
__constant__ double RK_CT[6] = {-1. / 150., 0., 3. / 100., -16. / 75., -1. / 20., 6. / 25.};

__device__ __forceinline__ bool in_bounds(const double* b, const double* y) {
  return b[0] <= y[0] && y[0] <= b[1] && b[2] <= y[1] && y[1] <= b[3] && b[4] <= y[2] && y[2] <= b[5];
}

// Cubic Hermite crossing of z = zp between accepted states s0 (time t0) and
// s1 (time t0 + h): Newton iteration safeguarded by bisection from the
// linear estimate.  Position from the Hermite cubic, velocity linear.
__device__ void hermite_crossing(double h, const double* s0, const double* s1, double zp, double t0, double* out) {
  auto pos = [&](double u, int c) {
    double u2 = u * u, u3 = u2 * u;
    return (2 * u3 - 3 * u2 + 1) * s0[c] + (u3 - 2 * u2 + u) * h * s0[3 + c] + (-2 * u3 + 3 * u2) * s1[c] +
           (u3 - u2) * h * s1[3 + c];
  };
  auto dpos = [&](double u, int c) {
    double u2 = u * u;
    return (6 * u2 - 6 * u) * s0[c] + (3 * u2 - 4 * u + 1) * h * s0[3 + c] + (-6 * u2 + 6 * u) * s1[c] +
           (3 * u2 - 2 * u) * h * s1[3 + c];
  };
  double u = (zp - s0[2]) / (s1[2] - s0[2]);
  double lo = 0.0, hi = 1.0;
  bool s0_above = s0[2] - zp > 0;
  for (int it = 0; it < 60; it++) {
    double f = pos(u, 2) - zp;
    if ((f > 0) == s0_above)
      lo = u;
    else
      hi = u;
    double d = dpos(u, 2);
    double un = d != 0 ? u - f / d : 0.5 * (lo + hi);
    if (!(lo < un && un < hi)) un = 0.5 * (lo + hi);
    if (fabs(un - u) < 1e-16) {
      u = un;
      break;
    }
    u = un;
  }
  out[0] = t0 + u * h;
  out[1] = pos(u, 0);
  out[2] = pos(u, 1);
  out[3] = zp;
  for (int c = 0; c < 3; c++) out[4 + c] = (1 - u) * s0[3 + c] + u * s1[3 + c];
}

// The integrator.  `field(p, E, H)` must return identical bits in every
// thread that shares a particle; `ks` is per-team scratch for the 6 stages,
// or, with REGS, unused: the stage loop is unrolled and the stage vectors
// live in registers of the one thread that owns the particle.
template <class FieldFn, bool REGS = false>
__device__ void rk45_particle(const TraceParams& P, int64_t idx, FieldFn& field, double (*ks_shared)[6],
                              bool writer) {
  double ks_regs[REGS ? 6 : 1][6];
  double (*ks)[6] = REGS ? ks_regs : ks_shared;
  double y[6];
  for (int c = 0; c < 6; c++) y[c] = P.start[idx * 6 + c];
  const double qm = P.qm[idx];
  double t = P.t0 ? P.t0[idx] : 0.0;
  const double V = sqrt(y[3] * y[3] + y[4] * y[4] + y[5] * y[5]);
  const double hmax = STEP_MAX / V;
  double h = hmax;
  int64_t nrow = 1, accepted = 0, attempts = 0;
  int status = TRACE_EXITED;
  const double atol = P.atol;
  if (writer && P.rows) {
    double* r = P.rows + idx * P.max_rows * 7;
    r[0] = t;
    for (int c = 0; c < 6; c++) r[1 + c] = y[c];
  }
  if (writer && P.plane)
    for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = __longlong_as_double(0x7ff8000000000000LL);

  while (in_bounds(P.bounds, y)) {
    if (attempts >= P.max_attempts) {
      status = TRACE_MAX_ATTEMPTS;
      break;
    }
    attempts++;
#pragma unroll(REGS ? 6 : 1)
    for (int s = 0; s < 6; s++) {
      double ys[6];
#pragma unroll
      for (int c = 0; c < 6; c++) {
        double v = y[c];
        for (int j = 0; j < s; j++) v += RK_B[s][j] * ks[j][c];
        ys[c] = v;
      }
      double E[3], H[3];
      field(ys, E, H);
      double cx = ys[4] * H[2] - ys[5] * H[1];
      double cy = ys[5] * H[0] - ys[3] * H[2];
      double cz = ys[3] * H[1] - ys[4] * H[0];
      double k0 = h * ys[3], k1 = h * ys[4], k2 = h * ys[5];
      double k3 = h * qm * (E[0] + MU0 * cx);
      double k4 = h * qm * (E[1] + MU0 * cy);
      double k5 = h * qm * (E[2] + MU0 * cz);
      ks[s][0] = k0;
      ks[s][1] = k1;
      ks[s][2] = k2;
      ks[s][3] = k3;
      ks[s][4] = k4;
      ks[s][5] = k5;
    }
    double ep = 0.0, ev = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double a = 0.0, b = 0.0;
      for (int j = 0; j < 6; j++) {
        a += RK_CT[j] * ks[j][c];
        b += RK_CT[j] * ks[j][c + 3];
      }
      ep = fmax(ep, fabs(a));
      ev = fmax(ev, fabs(b));
    }
    double err = ep + h * ev;
    if (!(err == err)) {
      status = TRACE_NONFINITE;
      break;
    }
    if (err <= atol) {
      double yn[6];
#pragma unroll
      for (int c = 0; c < 6; c++)
        yn[c] = y[c] + (RK_CH[0] * ks[0][c] + RK_CH[1] * ks[1][c] + RK_CH[2] * ks[2][c] + RK_CH[3] * ks[3][c] +
                        RK_CH[4] * ks[4][c] + RK_CH[5] * ks[5][c]);
      double tn = t + h;
      if (P.record_plane && ((y[2] - P.plane_z > 0) != (yn[2] - P.plane_z > 0))) {
        double cr[7];
        hermite_crossing(h, y, yn, P.plane_z, t, cr);
        if (writer && P.plane)
          for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = cr[c];
      }
#pragma unroll
      for (int c = 0; c < 6; c++) y[c] = yn[c];
      t = tn;
      accepted++;
      bool finite = true;
      for (int c = 0; c < 6; c++) finite = finite && isfinite(y[c]);
      if (P.rows) {
        if (writer) {
          double* r = P.rows + (idx * P.max_rows + nrow) * 7;
          r[0] = t;
          for (int c = 0; c < 6; c++) r[1 + c] = y[c];
        }
        nrow++;
      }
      if (!finite) {
        status = TRACE_NONFINITE;
        break;
      }
      if (P.rows && nrow >= P.max_rows) {
        status = TRACE_ROWS_FULL;
        break;
      }
    }
    h = fmin(0.9 * h * pow(atol / err, 0.2), hmax);
  }
  if (writer) {
    if (P.nrows) P.nrows[idx] = P.rows ? nrow : 1;
    if (P.status) P.status[idx] = status;
    if (P.final_state) {
      P.final_state[idx * 7] = t;
      for (int c = 0; c < 6; c++) P.final_state[idx * 7 + 1 + c] = y[c];
    }
    if (P.counters) {
      P.counters[idx * 2] = accepted;
      P.counters[idx * 2 + 1] = attempts;
    }
  }
}

__device__ __forceinline__ void team_barrier(int team, int nthreads) {
  if (nthreads <= 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(nthreads) : "memory");
}

// BEM field of a team: the elec and mag ring sums split over the team's
// threads, then a butterfly reduction (identical bits in every lane) and,
// for teams of several warps, a fixed-order sum of the warp partials.
template <int TW, bool GEOM>
struct BemTeamField {
  const TraceParams& P;
  int team, lt;
  double (*red)[6];  // [TW][6] per team
  int64_t e0 = 0, e1 = 0;  // GEOM: the electrostatic rings of the current particle's geometry
  const double* bnd = nullptr;  // GEOM: its bounding box (null: P.bounds)

  __device__ void operator()(const double* p, double* E, double* H) {
    constexpr int T = 32 * TW;
    const double* fb = P.fb;
    bool inside = fb == nullptr || (fb[0] < p[0] && p[0] < fb[1] && fb[2] < p[1] && p[1] < fb[3] &&
                                    fb[4] < p[2] && p[2] < fb[5]);
    double r0 = sqrt(p[0] * p[0] + p[1] * p[1]), z0 = p[2];
    // s: elec (Sr, Sz), mag (Sr, Sz), currents (Br, Bz)
    double s[6] = {0, 0, 0, 0, 0, 0};
    double dummy = 0;
    if (inside) {
      const double* er = P.esrc;
#pragma unroll 2
      for (int64_t j = (GEOM ? e0 : 0) + lt; j < (GEOM ? e1 : P.ne); j += T)
        ring_field_acc<false>(r0, z0, er[j], er[P.ne + j], er[2 * P.ne + j], s[0], s[1], dummy);
      const double* mr = P.msrc;
      for (int64_t j = lt; j < P.nm; j += T)
        ring_field_acc<false>(r0, z0, mr[j], mr[P.nm + j], mr[2 * P.nm + j], s[2], s[3], dummy);
      const double* cr = P.csrc;
      for (int64_t j = lt; j < P.nc; j += T) {
        double hr, hz;
        current_field_ring(r0, z0, cr[j], cr[P.nc + j], hr, hz);
        s[4] = fma(cr[2 * P.nc + j], hr, s[4]);
        s[5] = fma(cr[2 * P.nc + j], hz, s[5]);
      }
    }
    const int nsum = P.nc > 0 ? 6 : 4;
    for (int c = 0; c < nsum; c++) s[c] = warp_sum(s[c]);
    if (TW > 1) {
      int w = lt / 32;
      if ((lt & 31) == 0)
        for (int c = 0; c < nsum; c++) red[w][c] = s[c];
      team_barrier(team, T);
      for (int c = 0; c < nsum; c++) {
        double a = 0;
        for (int k = 0; k < TW; k++) a += red[k][c];
        s[c] = a;
      }
      team_barrier(team, T);
    }
    if (!inside) {
      for (int c = 0; c < 3; c++) E[c] = H[c] = 0.0;
      return;
    }
    if (r0 >= MIN_AXIS) {
      double er = s[0] / (2 * PI * r0), mr = s[2] / (2 * PI * r0);
      E[0] = p[0] / r0 * er;
      E[1] = p[1] / r0 * er;
      H[0] = p[0] / r0 * mr;
      H[1] = p[1] / r0 * mr;
    } else {
      E[0] = E[1] = H[0] = H[1] = 0.0;
    }
    E[2] = -s[1] * INV_PI;
    H[2] = -s[3] * INV_PI;
    if (P.nc > 0) {
      if (r0 >= MIN_AXIS) {
        H[0] += p[0] / r0 * s[4];
        H[1] += p[1] / r0 * s[4];
      }
      H[2] += s[5];
    }
  }
};

constexpr int TRACE_THREADS = 256;

// Integrator state of one warp, kept in shared memory rather than registers
// so that the only values live across a field evaluation are the evaluation
// point and the loop's own (every lane would otherwise hold its own copy of
// the whole state).  Each warp of a team keeps its own copy: all lanes of a
// warp store identical values in the same instruction, while warps of a team
// only meet at the barriers of the field reduction, so a warp never reads a
// value that another warp has already advanced.
struct TeamState {
  double y[6];
  double k[6][6];
  double t, h, hmax, qm;
  double bnd[6];  // many geometries: the particle's bounding box
  int64_t nrow, accepted, attempts;
  int status;
};

// rk45_particle (above) with its state in shared memory, for the BEM teams.
template <int TW, bool GEOM>
__device__ void rk45_team(const TraceParams& P, int64_t idx, BemTeamField<TW, GEOM>& field, volatile TeamState* S,
                          bool writer) {
  for (int c = 0; c < 6; c++) S->y[c] = P.start[idx * 6 + c];
  S->qm = P.qm[idx];
  S->t = P.t0 ? P.t0[idx] : 0.0;
  {
    const double V = sqrt(S->y[3] * S->y[3] + S->y[4] * S->y[4] + S->y[5] * S->y[5]);
    S->hmax = STEP_MAX / V;
    S->h = S->hmax;
  }
  S->nrow = 1;
  S->accepted = 0;
  S->attempts = 0;
  S->status = TRACE_EXITED;
  if (writer && P.rows) {
    double* r = P.rows + idx * P.max_rows * 7;
    r[0] = S->t;
    for (int c = 0; c < 6; c++) r[1 + c] = S->y[c];
  }
  if (writer && P.plane)
    for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = __longlong_as_double(0x7ff8000000000000LL);
  const double atol = P.atol;

  if (GEOM)  // the box in the team's shared state (no pointer held in registers)
    for (int c = 0; c < 6; c++) S->bnd[c] = field.bnd ? field.bnd[c] : P.bounds[c];
  for (;;) {
    {
      double y[6];
      for (int c = 0; c < 6; c++) y[c] = S->y[c];
      if (GEOM) {
        double b[6];
        for (int c = 0; c < 6; c++) b[c] = S->bnd[c];
        if (!in_bounds(b, y)) break;
      } else if (!in_bounds(P.bounds, y)) {
        break;
      }
    }
    if (S->attempts >= P.max_attempts) {
      S->status = TRACE_MAX_ATTEMPTS;
      break;
    }
    S->attempts = S->attempts + 1;
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
      double p[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        double v = S->y[c];
        for (int j = 0; j < s; j++) v += RK_B[s][j] * S->k[j][c];
        p[c] = v;
      }
      double E[3], H[3];
      field(p, E, H);
      double u[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        double v = S->y[3 + c];
        for (int j = 0; j < s; j++) v += RK_B[s][j] * S->k[j][3 + c];
        u[c] = v;
      }
      const double h = S->h, qm = S->qm;
      double cx = u[1] * H[2] - u[2] * H[1];
      double cy = u[2] * H[0] - u[0] * H[2];
      double cz = u[0] * H[1] - u[1] * H[0];
      S->k[s][0] = h * u[0];
      S->k[s][1] = h * u[1];
      S->k[s][2] = h * u[2];
      S->k[s][3] = h * qm * (E[0] + MU0 * cx);
      S->k[s][4] = h * qm * (E[1] + MU0 * cy);
      S->k[s][5] = h * qm * (E[2] + MU0 * cz);
    }
    const double h = S->h;
    double ep = 0.0, ev = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double a = 0.0, b = 0.0;
      for (int j = 0; j < 6; j++) {
        a += RK_CT[j] * S->k[j][c];
        b += RK_CT[j] * S->k[j][c + 3];
      }
      ep = fmax(ep, fabs(a));
      ev = fmax(ev, fabs(b));
    }
    const double err = ep + h * ev;
    if (!(err == err)) {
      S->status = TRACE_NONFINITE;
      break;
    }
    if (err <= atol) {
      double y[6], yn[6];
#pragma unroll
      for (int c = 0; c < 6; c++) {
        y[c] = S->y[c];
        yn[c] = y[c] + (RK_CH[0] * S->k[0][c] + RK_CH[1] * S->k[1][c] + RK_CH[2] * S->k[2][c] +
                        RK_CH[3] * S->k[3][c] + RK_CH[4] * S->k[4][c] + RK_CH[5] * S->k[5][c]);
      }
      const double t = S->t;
      if (P.record_plane && ((y[2] - P.plane_z > 0) != (yn[2] - P.plane_z > 0))) {
        double cr[7];
        hermite_crossing(h, y, yn, P.plane_z, t, cr);
        if (writer && P.plane)
          for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = cr[c];
      }
      bool finite = true;
#pragma unroll
      for (int c = 0; c < 6; c++) {
        S->y[c] = yn[c];
        finite = finite && isfinite(yn[c]);
      }
      S->t = t + h;
      S->accepted = S->accepted + 1;
      if (P.rows) {
        const int64_t nrow = S->nrow;
        if (writer) {
          double* r = P.rows + (idx * P.max_rows + nrow) * 7;
          r[0] = t + h;
          for (int c = 0; c < 6; c++) r[1 + c] = yn[c];
        }
        S->nrow = nrow + 1;
      }
      if (!finite) {
        S->status = TRACE_NONFINITE;
        break;
      }
      if (P.rows && S->nrow >= P.max_rows) {
        S->status = TRACE_ROWS_FULL;
        break;
      }
    }
    S->h = fmin(0.9 * h * pow(atol / err, 0.2), S->hmax);
  }
  if (writer) {
    if (P.nrows) P.nrows[idx] = P.rows ? S->nrow : 1;
    if (P.status) P.status[idx] = S->status;
    if (P.final_state) {
      P.final_state[idx * 7] = S->t;
      for (int c = 0; c < 6; c++) P.final_state[idx * 7 + 1 + c] = S->y[c];
    }
    if (P.counters) {
      P.counters[idx * 2] = S->accepted;
      P.counters[idx * 2 + 1] = S->attempts;
    }
  }
}

template <int TW, bool GEOM>
__global__ void __launch_bounds__(TRACE_THREADS, 2) k_trace_bem(TraceParams P) {
  constexpr int T = 32 * TW;
  constexpr int TEAMS = TRACE_THREADS / T;
  __shared__ TeamState s_state[TEAMS][TW];
  __shared__ double s_red[TEAMS][TW][6];
  __shared__ int64_t s_idx[TEAMS];
  const int team = threadIdx.x / T, lt = threadIdx.x % T;
  BemTeamField<TW, GEOM> field{P, team, lt, s_red[team]};
  for (;;) {
    int64_t idx;
    if (TW == 1) {
      int v = 0;
      if (lt == 0) v = atomicAdd(P.work, 1);
      idx = __shfl_sync(0xffffffffu, v, 0);
    } else {
      if (lt == 0) s_idx[team] = atomicAdd(P.work, 1);
      team_barrier(team, T);
      idx = s_idx[team];
      team_barrier(team, T);
    }
    if (idx >= P.n) break;
    if (GEOM) {  // an id outside [0, ngeom) sums no rings (the host checks ids)
      const int g = P.geom[idx];
      const bool ok = g >= 0 && g < P.ngeom;
      field.e0 = ok ? P.eoff[g] : 0;
      field.e1 = ok ? P.eoff[g + 1] : 0;
      field.bnd = ok && P.gbounds ? P.gbounds + 6 * g : nullptr;
    }
    rk45_team(P, idx, field, &s_state[team][lt / 32], lt == 0);
    __syncwarp();
  }
}

// Axial-interpolated field (field_radial_derivs_traceable): per thread.
struct AxialField {
  const TraceParams& P;
  __device__ void operator()(const double* p, double* E, double* H) {
    double d[NDERIV];
    double r2 = p[0] * p[0] + p[1] * p[1];
    if (axial_eval(p[2], P.az, P.aec, P.anz, d, 1))
      axial_field(d, p, r2, E);
    else
      E[0] = E[1] = E[2] = 0.0;
    if (P.amc && axial_eval(p[2], P.az, P.amc, P.anz, d, 1))
      axial_field(d, p, r2, H);
    else
      H[0] = H[1] = H[2] = 0.0;
  }
};

// One thread per particle: the stage loop fully unrolled, so the six stage
// vectors stay in registers (the team tracers share theirs in shared memory).
__global__ void __launch_bounds__(128) k_trace_axial(TraceParams P) {
  AxialField field{P};
  for (;;) {
    int64_t idx = atomicAdd(P.work, 1);
    if (idx >= P.n) break;
    rk45_particle<AxialField, true>(P, idx, field, nullptr, true);
  }
}

template <int TW, bool GEOM>
static int launch_bem(const TraceParams& P, cudaStream_t s) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_bem<TW, GEOM>, TRACE_THREADS, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int64_t teams_needed = P.n;
  int64_t blocks = (int64_t)num_sms() * per_sm;
  int64_t by_work = (teams_needed + (TRACE_THREADS / (32 * TW)) - 1) / (TRACE_THREADS / (32 * TW));
  if (blocks > by_work) blocks = by_work;
  if (blocks < 1) blocks = 1;
  k_trace_bem<TW, GEOM><<<unsigned(blocks), TRACE_THREADS, 0, s>>>(P);
  return launch_status();
}

// ============================================================================
// Surrogate-field tracer.  The field at a point is the axial-series field
// (radial.c:347-384) of coefficient tables for the actual excitation plus a
// learned correction: a small MLP predicts, per field source at unit
// strength (an electrode at 1 V, a current coil at 1 A-turn), the
// difference between the BEM field and the axial series, scaled by rho^p
// (rho = r / r_max) so that the correction vanishes toward the axis where the
// series is already exact; the per-source outputs are contracted with the
// source strengths (the fields are linear in them, the magnetizable
// material having a constant permeability).  Points within `fallback_dist`
// of an electrode segment, or outside the network's domain, fall back to the
// exact BEM sums.  MAG kernels add the magnetic field H (axial series of the
// magnetostatic table + the coils' learned corrections; magnetostatic
// charges and current rings in the fallback) and the Lorentz force
// q/m (E + mu0 v x H) of tracing.c:20-57.
// ============================================================================
struct SurrogateParams {
  const __nv_bfloat16* wb;
  const float* pf;
  MlpDomain dom;
  double z_lo, z_hi;
  // the network outputs contracted with the source strengths: before the
  // envelope, the learned corrections are sum_j w[j] y[j] with
  // wr[3 s + 1] = V_s scale[3 s + 1] and wz[3 s + 2] = V_s scale[3 s + 2] for
  // electrode s (E_r, E_z), hr / hz the same with the currents of the coils
  // (H_r, H_z), zero elsewhere
  float wr[MLP_OUT], wz[MLP_OUT], hr[MLP_OUT], hz[MLP_OUT];
  int env_p;
  const double* segs;  // (nseg, 4): r0, z0, r1, z1
  int nseg;
  double fb_dist2;
};

constexpr int SG_THREADS = 512;
constexpr int SG_WARPS = SG_THREADS / 32;
constexpr int SG_MAX_SEGS = 64;

// Electrode segment of the fallback test, staged in shared memory in FP32
// as (r0, z0, dr, dz, 1 / |d|^2), so the distance test takes no division.
// FP32 places the 50 um fallback boundary to within ~1e-10 m, far below
// anything that matters for the choice between network and exact field.
struct Seg {
  float ar, az, ur, uz, il2;
  float rmin;  // the smallest radius of all segments (the same in every entry)
};

struct SurrogateSmem {
  MlpSmem mlp;
  __nv_bfloat16 feat[SG_WARPS][32][MLP_LD_IN];
  float out[SG_WARPS][32][MLP_OUT];
  Seg segs[SG_MAX_SEGS];
};

__device__ inline void load_segments(Seg* seg, const double* __restrict__ segs, int nseg) {
  float rmin = 3.0e38f;
  for (int i = 0; i < nseg; i++) rmin = fminf(rmin, fminf(float(segs[4 * i]), float(segs[4 * i + 2])));
  for (int i = threadIdx.x; i < nseg; i += blockDim.x) {
    const double ar = segs[4 * i], az = segs[4 * i + 1];
    const double ur = segs[4 * i + 2] - ar, uz = segs[4 * i + 3] - az;
    const double L2 = ur * ur + uz * uz;
    seg[i] = Seg{float(ar), float(az), float(ur), float(uz), L2 > 0 ? float(1.0 / L2) : 0.f, rmin};
  }
}

__device__ __forceinline__ bool near_segments(const Seg* seg, int nseg, double r_d, double z_d, float d2) {
  const float r = float(r_d), z = float(z_d);
  if (nseg > 0) {  // inside the innermost radius of all segments, by more than the distance: none is near
    const float gap = seg[0].rmin - r;
    if (gap > 0.f && gap * gap > d2) return false;
  }
  bool nearby = false;
  for (int i = 0; i < nseg; i++) {
    const Seg g = seg[i];
    float tt = fmaf(r - g.ar, g.ur, (z - g.az) * g.uz) * g.il2;
    tt = fminf(fmaxf(tt, 0.f), 1.f);
    const float dr = r - fmaf(tt, g.ur, g.ar), dz = z - fmaf(tt, g.uz, g.az);
    nearby = nearby || (fmaf(dr, dr, dz * dz) < d2);
  }
  return nearby;
}

// Raw ring sums of the exact BEM field at (r0, z) over the rings first,
// first + stride, ...: s[0], s[1] the electrostatic (S_r, S_z) and, with MAG,
// s[2], s[3] the magnetostatic charges' and s[4], s[5] the current rings'
// (H_r, H_z) (field_radial_traceable, tracing.c:141-163).  Out of line: it
// is the rare path of the surrogate tracer, and inlined its ring kernels'
// registers would count against the whole tracer.
struct BemSums {
  double s[6];
};

template <bool MAG>
__device__ __noinline__ BemSums bem_sums(const TraceParams& P, double r0, double z, int first, int stride) {
  BemSums out;
  double* s = out.s;
  double Sr = 0, Sz = 0, dummy = 0;
  const double* er = P.esrc;
  // The magnetic variant (the combined workload's fallback, two systems of
  // rings per point) unrolls four rings per iteration: more independent
  // work for the few warps that run it (the accumulation order is
  // unchanged).  The electrostatic variant stays rolled, which keeps its
  // callers' registers (the headline tracer) free of the extra spills.
  if (MAG) {
#pragma unroll 4
    for (int64_t j = first; j < P.ne; j += stride)
      ring_field_acc<false>(r0, z, er[j], er[P.ne + j], er[2 * P.ne + j], Sr, Sz, dummy);
  } else {
    for (int64_t j = first; j < P.ne; j += stride)
      ring_field_acc<false>(r0, z, er[j], er[P.ne + j], er[2 * P.ne + j], Sr, Sz, dummy);
  }
  s[0] = Sr;
  s[1] = Sz;
  if (MAG) {
    double Mr = 0, Mz = 0, Cr = 0, Cz = 0;
    const double* mr = P.msrc;
#pragma unroll 4
    for (int64_t j = first; j < P.nm; j += stride)
      ring_field_acc<false>(r0, z, mr[j], mr[P.nm + j], mr[2 * P.nm + j], Mr, Mz, dummy);
    const double* cr = P.csrc;
    for (int64_t j = first; j < P.nc; j += stride) {
      double hr, hz;
      current_field_ring(r0, z, cr[j], cr[P.nc + j], hr, hz);
      Cr = fma(cr[2 * P.nc + j], hr, Cr);
      Cz = fma(cr[2 * P.nc + j], hz, Cz);
    }
    s[2] = Mr;
    s[3] = Mz;
    s[4] = Cr;
    s[5] = Cz;
  } else {
    s[2] = s[3] = s[4] = s[5] = 0.0;
  }
  return out;
}

// E (and with MAG H) at p from the raw sums of bem_sums.
template <bool MAG>
__device__ __forceinline__ void bem_finish(const double* p, double r0, const double* s, double* E, double* H) {
  if (r0 >= MIN_AXIS) {
    double e = s[0] / (2 * PI * r0);
    E[0] = p[0] / r0 * e;
    E[1] = p[1] / r0 * e;
  } else {
    E[0] = E[1] = 0.0;
  }
  E[2] = -s[1] * INV_PI;
  if (MAG) {
    if (r0 >= MIN_AXIS) {
      const double h = s[2] / (2 * PI * r0) + s[4];
      H[0] = p[0] / r0 * h;
      H[1] = p[1] / r0 * h;
    } else {
      H[0] = H[1] = 0.0;
    }
    H[2] = -s[3] * INV_PI + s[5];
  }
}

// Exact BEM field at one point, by one lane.
template <bool MAG>
__device__ __forceinline__ void bem_point_field(const TraceParams& P, const double* p, double* E, double* H) {
  const double r0 = sqrt(p[0] * p[0] + p[1] * p[1]);
  const BemSums s = bem_sums<MAG>(P, r0, p[2], 0, 1);
  bem_finish<MAG>(p, r0, s.s, E, H);
}

// Axial series of one coefficient table plus the learned correction
// (cr, cz) times the envelope env: the radial part (cr rho^(p+1)) applied
// as x * (F_r / r).
__device__ __forceinline__ void axial_plus_correction(const TraceParams& P, const double* table, const double* p,
                                                      double r2, double env_r, double env, float cr, float cz,
                                                      double* F) {
  double d[NDERIV];
  if (table && axial_eval(p[2], P.az, table, P.anz, d, 1))
    axial_field(d, p, r2, F);
  else
    F[0] = F[1] = F[2] = 0.0;
  const double fr = double(cr) * env_r, fz = double(cz) * env;
  F[0] += p[0] * fr;
  F[1] += p[1] * fr;
  F[2] += fz;
}

// The field at point p from the contracted network outputs c (the learned
// E_r, E_z and, with MAG, H_r, H_z corrections before the envelope): zero
// outside the field bounds, exact BEM near electrodes and outside the
// network's domain, else axial series + learned correction.
constexpr int FIELD_ZERO = 0, FIELD_BEM = 1, FIELD_SURROGATE = 2;

// Which field applies at p: none (not live, or outside the field bounds),
// the exact BEM sums (near an electrode or outside the network's domain), or
// the surrogate.
__device__ __forceinline__ int surrogate_kind(const TraceParams& P, const SurrogateParams& S, const Seg* segs,
                                              const double* p, double r, bool live) {
  const double* fb = P.fb;
  if (!live ||
      (fb && !(fb[0] < p[0] && p[0] < fb[1] && fb[2] < p[1] && p[1] < fb[3] && fb[4] < p[2] && p[2] < fb[5])))
    return FIELD_ZERO;
  const bool out_of_domain = r > S.dom.r_max || p[2] < S.z_lo || p[2] > S.z_hi;
  if (out_of_domain || near_segments(segs, S.nseg, r, p[2], float(S.fb_dist2))) return FIELD_BEM;
  return FIELD_SURROGATE;
}

template <bool MAG>
__device__ __forceinline__ void surrogate_apply(const TraceParams& P, const SurrogateParams& S, const double* p,
                                                double r2, double r, const float* c, double* E, double* H);

template <bool MAG>
__device__ __forceinline__ void surrogate_combine(const TraceParams& P, const SurrogateParams& S,
                                                 const Seg* segs, const double* p, double r2, double r,
                                                 bool live, const float* c, double* E, double* H, bool& used_bem) {
  const int kind = surrogate_kind(P, S, segs, p, r, live);
  used_bem = kind == FIELD_BEM;
  if (kind == FIELD_SURROGATE) {
    surrogate_apply<MAG>(P, S, p, r2, r, c, E, H);
  } else if (kind == FIELD_BEM) {
    bem_point_field<MAG>(P, p, E, H);
  } else {
    E[0] = E[1] = E[2] = 0.0;
    if (MAG) H[0] = H[1] = H[2] = 0.0;
  }
}

// Axial series + learned correction at p, inside the network's domain.
template <bool MAG>
__device__ __forceinline__ void surrogate_apply(const TraceParams& P, const SurrogateParams& S, const double* p,
                                                double r2, double r, const float* c, double* E, double* H) {
  const double rho = r / S.dom.r_max;
  double env = 1.0;
  for (int i = 0; i < S.env_p; i++) env *= rho;
  const double env_r = env / S.dom.r_max;
  axial_plus_correction(P, P.aec, p, r2, env_r, env, c[0], c[1], E);
  if (MAG) axial_plus_correction(P, P.amc, p, r2, env_r, env, c[2], c[3], H);
}

// The network's outputs y at a point contracted with the source strengths
// into c (the learned E_r, E_z and, with MAG, H_r, H_z corrections).
template <bool MAG>
__device__ __forceinline__ void contract_outputs(const SurrogateParams& S, const float* y, float* c) {
  c[0] = c[1] = 0.f;
  if (MAG) c[2] = c[3] = 0.f;
#pragma unroll
  for (int j = 0; j < MLP_OUT; j++) {
    c[0] = fmaf(S.wr[j], y[j], c[0]);
    c[1] = fmaf(S.wz[j], y[j], c[1]);
    if (MAG) {
      c[2] = fmaf(S.hr[j], y[j], c[2]);
      c[3] = fmaf(S.hz[j], y[j], c[3]);
    }
  }
}

// Field at this lane's point; every lane of the warp must call it.
template <bool MAG>
__device__ void surrogate_field(const TraceParams& P, const SurrogateParams& S, SurrogateSmem& sm, int warp, int lane,
                                const double* p, bool live, double* E, double* H, bool& used_bem) {
  const double r2 = p[0] * p[0] + p[1] * p[1], r = sqrt(r2);
  float f[MLP_IN];
  mlp_features(r, p[2], S.dom, f);
#pragma unroll
  for (int c = 0; c < MLP_IN; c++) sm.feat[warp][lane][c] = __float2bfloat16(f[c]);
  mlp_warp_forward(sm.mlp, sm.feat[warp], sm.out[warp]);
  float c[4];
  contract_outputs<MAG>(S, sm.out[warp][lane], c);
  surrogate_combine<MAG>(P, S, sm.segs, p, r2, r, live, c, E, H, used_bem);
}

// The RKF45 particle loop of the surrogate tracer, shared by both network
// engines.  `eng.any(b)` is true if b holds on any thread that evaluates the
// network together with this one; `eng.field(p, live, E, H, used_bem)` is
// the field at p (all those threads call it together; H only with MAG) and
// returns false if the engine failed (uniformly across them).
template <bool MAG, class Engine>
__device__ void surrogate_trace_loop(const TraceParams& P, const SurrogateParams& S, Engine& eng) {
  bool engine_failed = false;
  double y[6];
  double t = 0, h = 0, hmax = 0, qm = 0;
  int accepted = 0, attempts = 0, fallbacks = 0;  // the launch caps max_attempts below 2^31
  int status = TRACE_EXITED;
  int64_t idx = atomicAdd(P.work, 1);
  bool active = idx < P.n;

  auto start = [&]() {
    for (int c = 0; c < 6; c++) y[c] = P.start[idx * 6 + c];
    qm = P.qm[idx];
    t = P.t0 ? P.t0[idx] : 0.0;
    hmax = STEP_MAX / sqrt(y[3] * y[3] + y[4] * y[4] + y[5] * y[5]);
    h = hmax;
    accepted = attempts = fallbacks = 0;
    status = TRACE_EXITED;
    if (P.plane)
      for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = __longlong_as_double(0x7ff8000000000000LL);
  };
  auto finish = [&]() {
    if (P.status) P.status[idx] = status;
    if (P.nrows) P.nrows[idx] = 1;
    if (P.final_state) {
      P.final_state[idx * 7] = t;
      for (int c = 0; c < 6; c++) P.final_state[idx * 7 + 1 + c] = y[c];
    }
    if (P.counters) {
      P.counters[idx * 3] = accepted;
      P.counters[idx * 3 + 1] = attempts;
      P.counters[idx * 3 + 2] = fallbacks;
    }
    idx = atomicAdd(P.work, 1);
    active = idx < P.n;
  };
  if (active) start();

  while (eng.any(active)) {
    bool go = false;
    if (active) {
      if (!in_bounds(P.bounds, y)) {
        finish();
        if (active) start();
      } else if (attempts >= P.max_attempts) {
        status = TRACE_MAX_ATTEMPTS;
        finish();
        if (active) start();
      }
      go = active && in_bounds(P.bounds, y) && attempts < P.max_attempts;
    }
    if (go) attempts++;
    // Stage sums kept as running accumulators with static indices (no
    // dynamically indexed array, so nothing goes to local memory):
    // off[i] = sum_j B[i+1][j] k_j (input of stage i + 1), k5 = sum_j CH[j] k_j
    // (fifth-order increment), ke = sum_j CT[j] k_j (error estimate).
    double off[5][6], k5[6], ke[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
      k5[c] = ke[c] = 0.0;
#pragma unroll
      for (int i = 0; i < 5; i++) off[i][c] = 0.0;
    }
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
      double ys[6];
#pragma unroll
      for (int c = 0; c < 6; c++) {
        double o = 0.0;
#pragma unroll
        for (int i = 0; i < 5; i++) o = (s == i + 1) ? off[i][c] : o;
        ys[c] = y[c] + o;
      }
      if (!go) {
        ys[0] = 0.5 * S.dom.r_max;
        ys[1] = 0.0;
        ys[2] = S.dom.z_c;
      }
      double E[3], H[MAG ? 3 : 1];
      bool used_bem;
      if (!eng.field(ys, go, E, H, used_bem)) {
        engine_failed = true;
        break;
      }
      if (go) {
        fallbacks += used_bem ? 1 : 0;
        if (MAG) {  // Lorentz force: E + mu0 v x H (tracing.c:20-57)
          const double cx = ys[4] * H[2] - ys[5] * H[1];
          const double cy = ys[5] * H[0] - ys[3] * H[2];
          const double cz = ys[3] * H[1] - ys[4] * H[0];
          E[0] += MU0 * cx;
          E[1] += MU0 * cy;
          E[2] += MU0 * cz;
        }
        const double k[6] = {h * ys[3], h * ys[4], h * ys[5], h * qm * E[0], h * qm * E[1], h * qm * E[2]};
        const double ch = RK_CH[s], ct = RK_CT[s];
#pragma unroll
        for (int c = 0; c < 6; c++) {
          k5[c] = fma(ch, k[c], k5[c]);
          ke[c] = fma(ct, k[c], ke[c]);
        }
        if (s < 5) {
#pragma unroll
          for (int i = 0; i < 5; i++) {
            const double b = RK_B[i + 1][s];  // zero for s >= i + 1
#pragma unroll
            for (int c = 0; c < 6; c++) off[i][c] = fma(b, k[c], off[i][c]);
          }
        }
      }
    }
    if (engine_failed) {
      // the tensor-core engine gave up waiting for its MMAs (group-uniform):
      // the particles in hand end with TRACE_ENGINE_TIMEOUT at their last
      // accepted state, and so does every particle this group still draws
      // from the queue (untraced: start state, zero counters), so that each
      // particle of the launch leaves with a defined status
      while (active) {
        status = TRACE_ENGINE_TIMEOUT;
        finish();
        if (active) start();
      }
      return;
    }
    if (!go) continue;
    double ep = 0.0, ev = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      ep = fmax(ep, fabs(ke[c]));
      ev = fmax(ev, fabs(ke[c + 3]));
    }
    double err = ep + h * ev;
    if (!(err == err)) {
      status = TRACE_NONFINITE;
      finish();
      if (active) start();
      continue;
    }
    if (err <= P.atol) {
      double yn[6];
#pragma unroll
      for (int c = 0; c < 6; c++) yn[c] = y[c] + k5[c];
      if (P.record_plane && ((y[2] - P.plane_z > 0) != (yn[2] - P.plane_z > 0))) {
        double cr[7];
        hermite_crossing(h, y, yn, P.plane_z, t, cr);
        if (P.plane)
          for (int c = 0; c < 7; c++) P.plane[idx * 7 + c] = cr[c];
      }
      bool finite = true;
#pragma unroll
      for (int c = 0; c < 6; c++) {
        y[c] = yn[c];
        finite = finite && isfinite(yn[c]);
      }
      t += h;
      accepted++;
      if (!finite) {
        status = TRACE_NONFINITE;
        finish();
        if (active) start();
        continue;
      }
    }
    h = fmin(0.9 * h * pow(P.atol / err, 0.2), hmax);
  }
}


// Network engine of the warp-level kernel: the 32 lanes of a warp evaluate
// the network together with mma.sync.
template <bool MAG>
struct WarpEngine {
  const TraceParams& P;
  const SurrogateParams& S;
  SurrogateSmem& sm;
  int warp, lane;
  __device__ bool any(bool b) const { return __any_sync(0xffffffffu, b); }
  __device__ bool field(const double* p, bool live, double* E, double* H, bool& used_bem) {
    surrogate_field<MAG>(P, S, sm, warp, lane, p, live, E, H, used_bem);
    return true;
  }
};

template <bool MAG>
__global__ void __launch_bounds__(SG_THREADS, 1) k_trace_surrogate(TraceParams P, SurrogateParams S) {
  extern __shared__ __align__(16) unsigned char sg_raw[];
  SurrogateSmem& sm = *reinterpret_cast<SurrogateSmem*>(sg_raw);
  mlp_load_smem(sm.mlp, S.wb, S.pf);
  load_segments(sm.segs, S.segs, S.nseg);
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;

  WarpEngine<MAG> eng{P, S, sm, warp, lane};
  surrogate_trace_loop<MAG>(P, S, eng);
}

// Surrogate field E (and with MAG the magnetic field H) at M points (one
// point per lane), for tests.
template <bool MAG>
__global__ void __launch_bounds__(SG_THREADS, 1)
    k_surrogate_points(TraceParams P, SurrogateParams S, const double* __restrict__ pts, int64_t M,
                       double* __restrict__ field, double* __restrict__ hfield, int32_t* __restrict__ used_bem) {
  extern __shared__ __align__(16) unsigned char sg_raw[];
  SurrogateSmem& sm = *reinterpret_cast<SurrogateSmem*>(sg_raw);
  mlp_load_smem(sm.mlp, S.wb, S.pf);
  load_segments(sm.segs, S.segs, S.nseg);
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * SG_THREADS + warp * 32; base < M; base += (int64_t)gridDim.x * SG_THREADS) {
    int64_t i = base + lane;
    bool live = i < M;
    double p[3] = {0.5 * S.dom.r_max, 0.0, S.dom.z_c};
    if (live)
      for (int c = 0; c < 3; c++) p[c] = pts[3 * i + c];
    double E[3], H[3] = {0.0, 0.0, 0.0};
    bool ub;
    surrogate_field<MAG>(P, S, sm, warp, lane, p, live, E, H, ub);
    if (live) {
      for (int c = 0; c < 3; c++) field[3 * i + c] = E[c];
      if (hfield)
        for (int c = 0; c < 3; c++) hfield[3 * i + c] = H[c];
      if (used_bem) used_bem[i] = ub ? 1 : 0;
    }
  }
}

// ============================================================================
// Tensor-memory engine of the surrogate tracer (tcgen05).  The CTA's threads
// form TC_GROUPS groups of 128 (one warpgroup each); a group's 128 particles
// are the 128 rows of one MMA tile.  At every RK stage the threads write
// their input features (BF16) into the group's activation tile in shared
// memory; one elected thread issues the layer's tcgen05.mma chain (A: the
// activation tile, B: the layer's weights, both K-major SWIZZLE_128B in
// shared memory; D: the group's 128 FP32 columns of tensor memory) and
// commits it to the group's mbarrier; the threads read their own row back
// (tcgen05.ld: thread row = TMEM lane), add the bias, apply SiLU and write
// the next layer's BF16 activations into the same tile.  The weights are
// staged once per CTA; one CTA per SM (shared memory ~218 KB).
// ============================================================================
#ifndef TB_TC_GROUPS
#define TB_TC_GROUPS 3
#endif
constexpr int TC_GROUPS = TB_TC_GROUPS;
constexpr int TC_THREADS = 128 * TC_GROUPS;
constexpr uint32_t TC_TMEM_COLS = 512;              // 3 x 128 used
constexpr uint32_t TC_ATOM = 128 * 128;             // bytes of a 128-row SWIZZLE_128B atom

struct TcSmem {
  uint8_t w1[TC_ATOM];                    // W1: 128 rows x K = 16 (chunks 0, 1 of each row)
  uint8_t wh[3][2][TC_ATOM];              // W2..W4: 128 rows x K = 128 (two atoms)
  uint8_t w5[2][MLP_OUT * 128];           // W5: MLP_OUT rows x K = 128
  uint8_t act[TC_GROUPS][2][TC_ATOM];     // per group: activations, 128 rows x K <= 128
  float b1[MLP_H], bh[3][MLP_H], b5[MLP_OUT];
  Seg segs[SG_MAX_SEGS];
  uint64_t mbar[TC_GROUPS];
  uint32_t tmem_base;
};
static_assert(offsetof(TcSmem, wh) % 1024 == 0 && offsetof(TcSmem, w5) % 1024 == 0 &&
                  offsetof(TcSmem, act) % 1024 == 0,
              "operand tiles must be 1024-byte aligned");
constexpr int TC_SMEM_BYTES = int(sizeof(TcSmem)) + 1024;  // + alignment slack of the dynamic window

__device__ __forceinline__ void st_bf16(uint8_t* dst, __nv_bfloat16 v) { *reinterpret_cast<__nv_bfloat16*>(dst) = v; }

// x / 2 of a BF16 value (exact: a power-of-two scale).
__device__ __forceinline__ __nv_bfloat16 half_bf16(__nv_bfloat16 x) {
  return __float2bfloat16(0.5f * __bfloat162float(x));
}

// Stages the network in the swizzled operand layout (all threads take part).
// The four SiLU layers' weights and biases are stored scaled by 1/2 (exact),
// so their accumulators hold h = z / 2 directly (silu(z) = h + h tanh(h)).
__device__ void tc_load_network(TcSmem& s, const __nv_bfloat16* __restrict__ wb, const float* __restrict__ pf) {
  const int nt = blockDim.x;
  for (int e = threadIdx.x; e < MLP_H * MLP_IN; e += nt) {
    const int n = e / MLP_IN, k = e % MLP_IN;
    st_bf16(s.w1 + tc::sw128(n, k >> 3) + (k & 7) * 2, half_bf16(wb[MLP_OFF_W1 + e]));
  }
  const int64_t off[3] = {MLP_OFF_W2, MLP_OFF_W3, MLP_OFF_W4};
  for (int l = 0; l < 3; l++)
    for (int e = threadIdx.x; e < MLP_H * MLP_H; e += nt) {
      const int n = e / MLP_H, k = e % MLP_H;
      st_bf16(s.wh[l][k >> 6] + tc::sw128(n, (k & 63) >> 3) + (k & 7) * 2, half_bf16(wb[off[l] + e]));
    }
  for (int e = threadIdx.x; e < MLP_OUT * MLP_H; e += nt) {
    const int n = e / MLP_H, k = e % MLP_H;
    st_bf16(s.w5[k >> 6] + tc::sw128(n, (k & 63) >> 3) + (k & 7) * 2, wb[MLP_OFF_W5 + e]);
  }
  for (int e = threadIdx.x; e < MLP_H; e += nt) {
    s.b1[e] = 0.5f * pf[MLP_OFF_B1 + e];
    s.bh[0][e] = 0.5f * pf[MLP_OFF_B2 + e];
    s.bh[1][e] = 0.5f * pf[MLP_OFF_B3 + e];
    s.bh[2][e] = 0.5f * pf[MLP_OFF_B4 + e];
  }
  for (int e = threadIdx.x; e < MLP_OUT; e += nt) s.b5[e] = pf[MLP_OFF_B5 + e];
}

// Issues layer `layer` (0: K = 16 -> 128, 1-3: 128 -> 128, 4: 128 -> MLP_OUT)
// of one group: A = the group's activation tile, D = its TMEM columns.
__device__ __forceinline__ void tc_issue_layer(const TcSmem& s, uint32_t act, uint32_t dtm, int layer) {
  constexpr uint32_t ID128 = tc::idesc_bf16_f32(128, 128);
  constexpr uint32_t IDOUT = tc::idesc_bf16_f32(128, MLP_OUT);
  if (layer == 0) {
    tc::mma_bf16(dtm, tc::desc_sw128(act), tc::desc_sw128(tc::smem_u32(s.w1)), ID128, 0u);
    return;
  }
  const uint32_t wbase = layer < 4 ? tc::smem_u32(s.wh[layer - 1][0]) : tc::smem_u32(s.w5[0]);
  const uint32_t watom = layer < 4 ? TC_ATOM : uint32_t(MLP_OUT) * 128u;
  const uint32_t id = layer < 4 ? ID128 : IDOUT;
#pragma unroll
  for (int kk = 0; kk < 8; kk++) {
    const uint32_t ka = (kk >> 2) * TC_ATOM + (kk & 3) * 32;
    const uint32_t kb = (kk >> 2) * watom + (kk & 3) * 32;
    tc::mma_bf16(dtm, tc::desc_sw128(act + ka), tc::desc_sw128(wbase + kb), id, kk > 0 ? 1u : 0u);
  }
}

// One group's view of the engine.
template <bool MAG>
struct TcEngine {
  const TraceParams& P;
  const SurrogateParams& S;
  TcSmem& s;
  int g;           // group index
  int row;         // this thread's row of the group's tile = its TMEM lane
  uint32_t act;    // shared address of the group's activation tile
  uint32_t dtm;    // TMEM address of the group's accumulator (lane 0)
  uint32_t tld;    // the same with this warp's lane quarter, for tcgen05.ld
  uint32_t phase;  // parity of the group's next mbarrier phase

  __device__ bool any(bool b) const { return tc::bar_any(1 + g, 128, b); }

  // Network outputs for this thread's features, contracted with the source
  // strengths into c (contract_outputs); all 128 threads of the group call
  // it together.  False (group-uniform) if an MMA wait ran out.
  __device__ __forceinline__ bool forward(const float* feat, float* c) {
    tc::st_shared_v4(act + tc::sw128(row, 0), pack_bf16(feat[0], feat[1]), pack_bf16(feat[2], feat[3]),
                     pack_bf16(feat[4], feat[5]), pack_bf16(feat[6], feat[7]));
    tc::st_shared_v4(act + tc::sw128(row, 1), pack_bf16(feat[8], feat[9]), pack_bf16(feat[10], feat[11]),
                     pack_bf16(feat[12], feat[13]), pack_bf16(feat[14], feat[15]));
#pragma unroll 1
    for (int layer = 0; layer < 5; layer++) {
      // the A tile is complete and every earlier TMEM read of the group done
      tc::fence_async_smem();
      tc::fence_before_sync();
      asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
      if (row == 0) {
        tc::fence_after_sync();
        tc_issue_layer(s, act, dtm, layer);
        tc::mma_commit(&s.mbar[g]);
      }
      const bool ok = tc::mbar_wait_warp(&s.mbar[g], phase, P.wait_cycles);
      if (tc::bar_any(1 + g, 128, !ok)) {
        // the chain committed above must finish before the group gives up
        // its tile and its tensor memory
        tc::mbar_wait_warp(&s.mbar[g], phase, DRAIN_WAIT_CYCLES);
        phase ^= 1u;
        return false;
      }
      phase ^= 1u;
      tc::fence_after_sync();
      if (layer < 4) {
        const float* bias = layer == 0 ? s.b1 : s.bh[layer - 1];
        // 16 columns at a time, the TMEM load of the next chunk in flight
        // while this one is processed.  The staged weights and biases of
        // these layers are pre-scaled by 1/2 (exact), so acc + bias is
        // h = z / 2 and silu(z) = h + h tanh(h).
        uint32_t va[16], vb[16];
        tc::tmem_ld16(tld, va);
        tc::tmem_wait_ld16(va);
#pragma unroll
        for (int c = 0; c < 8; c++) {  // columns 16c .. 16c + 15
          uint32_t* cur = (c & 1) ? vb : va;
          uint32_t* nxt = (c & 1) ? va : vb;
          if (c < 7) tc::tmem_ld16(tld + 16 * (c + 1), nxt);
          uint32_t q[8];
#pragma unroll
          for (int j = 0; j < 8; j++)
            q[j] = silu2_bf16_half_bias(__uint_as_float(cur[2 * j]), __uint_as_float(cur[2 * j + 1]),
                                        bias[16 * c + 2 * j], bias[16 * c + 2 * j + 1]);
          // next layer's K = 16c .. 16c + 15: atom c / 4, chunks 2 (c % 4), 2 (c % 4) + 1
          const uint32_t base = act + (c >> 2) * TC_ATOM;
          tc::st_shared_v4(base + tc::sw128(row, 2 * (c & 3)), q[0], q[1], q[2], q[3]);
          tc::st_shared_v4(base + tc::sw128(row, 2 * (c & 3) + 1), q[4], q[5], q[6], q[7]);
          if (c < 7) tc::tmem_wait_ld16(nxt);
        }
      } else {
        // the MLP_OUT outputs 16 columns at a time, contracted as they come
        c[0] = c[1] = 0.f;
        if (MAG) c[2] = c[3] = 0.f;
#pragma unroll
        for (int hc = 0; hc < MLP_OUT / 16; hc++) {
          uint32_t v[16];
          tc::tmem_ld16(tld + 16 * hc, v);
          tc::tmem_wait_ld16(v);
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const int o = 16 * hc + j;
            const float y = __uint_as_float(v[j]) + s.b5[o];
            c[0] = fmaf(S.wr[o], y, c[0]);
            c[1] = fmaf(S.wz[o], y, c[1]);
            if (MAG) {
              c[2] = fmaf(S.hr[o], y, c[2]);
              c[3] = fmaf(S.hz[o], y, c[3]);
            }
          }
        }
      }
    }
    return true;
  }

  __device__ __forceinline__ bool field(const double* p, bool live, double* E, double* H, bool& used_bem) {
    const double r2 = p[0] * p[0] + p[1] * p[1], r = sqrt(r2);
    float f[MLP_IN], c[4];
    mlp_features(r, p[2], S.dom, f);
    if (!forward(f, c)) {
      E[0] = E[1] = E[2] = 0.0;
      if (MAG) H[0] = H[1] = H[2] = 0.0;
      used_bem = false;
      return false;
    }
    const int kind = surrogate_kind(P, S, s.segs, p, r, live);
    used_bem = kind == FIELD_BEM;
    if (kind == FIELD_SURROGATE) {
      surrogate_apply<MAG>(P, S, p, r2, r, c, E, H);
    } else {
      E[0] = E[1] = E[2] = 0.0;
      if (MAG) H[0] = H[1] = H[2] = 0.0;
    }
    if (any(used_bem)) group_bem(p, used_bem, E, H);
    return true;
  }

  // The exact field at the points of the group's threads that need it,
  // summed by all 128 threads together, one point at a time (the rings
  // strided over the group, warp sums, then the four warps' partials in a
  // fixed order).  Scratch: the group's activation tile, free between
  // network evaluations (the last MMA that read it has completed).
  __device__ __forceinline__ void group_bem(const double* p, bool need, double* E, double* H) {
    double* sc = reinterpret_cast<double*>(&s.act[g][0][0]);  // [0..2] point, [4..27] partials
    int* owner = reinterpret_cast<int*>(sc + 3);
    double* part = sc + 4;
    const int w = row >> 5, lane = row & 31;
    bool pending = need;
    while (any(pending)) {
      if (row == 0) *owner = 128;
      asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
      if (pending) atomicMin(owner, row);
      asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
      const int o = *owner;
      if (row == o) {
        sc[0] = p[0];
        sc[1] = p[1];
        sc[2] = p[2];
      }
      asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
      const double q[3] = {sc[0], sc[1], sc[2]};
      const double r0 = sqrt(q[0] * q[0] + q[1] * q[1]);
      const BemSums sums = bem_sums<MAG>(P, r0, q[2], row, 128);
#pragma unroll
      for (int k = 0; k < (MAG ? 6 : 2); k++) {
        const double v = warp_sum(sums.s[k]);
        if (lane == 0) part[w * 6 + k] = v;
      }
      asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
      if (row == o) {
        double tot[6];
#pragma unroll
        for (int k = 0; k < 6; k++) tot[k] = ((part[k] + part[6 + k]) + part[12 + k]) + part[18 + k];
        bem_finish<MAG>(q, r0, tot, E, H);
        pending = false;
      }
    }
  }
};

// Shared set-up of the tcgen05 kernels: network and segments staged,
// mbarriers initialised, TMEM allocated (warp 0).  Returns the aligned
// shared-memory image.
__device__ TcSmem& tc_setup(unsigned char* raw, const SurrogateParams& S) {
  const uint32_t a = tc::smem_u32(raw);
  TcSmem& s = *reinterpret_cast<TcSmem*>(raw + (((a + 1023u) & ~1023u) - a));
  tc_load_network(s, S.wb, S.pf);
  load_segments(s.segs, S.segs, S.nseg);
  if (threadIdx.x < TC_GROUPS) tc::mbar_init(&s.mbar[threadIdx.x], 1);
  if (threadIdx.x == 0) tc::fence_mbar_init();
  if (threadIdx.x / 32 == 0) {
    tc::tmem_alloc(&s.tmem_base, TC_TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  return s;
}

__device__ void tc_teardown(TcSmem& s) {
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x / 32 == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(s.tmem_base, TC_TMEM_COLS);
  }
}

template <bool MAG>
__device__ __forceinline__ TcEngine<MAG> tc_engine(const TraceParams& P, const SurrogateParams& S, TcSmem& s) {
  const int g = threadIdx.x / 128, row = threadIdx.x % 128;
  const uint32_t dtm = s.tmem_base + uint32_t(128 * g);
  const uint32_t tld = dtm + (uint32_t((threadIdx.x / 32) % 4 * 32) << 16);
  return TcEngine<MAG>{P, S, s, g, row, tc::smem_u32(s.act[g][0]), dtm, tld, 0u};
}

template <bool MAG>
__global__ void __launch_bounds__(TC_THREADS, 1) k_trace_surrogate_tc(TraceParams P, SurrogateParams S) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& s = tc_setup(tc_raw, S);
  TcEngine<MAG> eng = tc_engine<MAG>(P, S, s);
  surrogate_trace_loop<MAG>(P, S, eng);
  tc_teardown(s);
}

// Surrogate field E (and with MAG the magnetic field H) at M points (one
// point per thread, 128 per group), for tests; used_bem = -1 marks points
// whose MMA wait ran out.
template <bool MAG>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_surrogate_points_tc(TraceParams P, SurrogateParams S, const double* __restrict__ pts, int64_t M,
                          double* __restrict__ field, double* __restrict__ hfield, int32_t* __restrict__ used_bem) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& s = tc_setup(tc_raw, S);
  TcEngine<MAG> eng = tc_engine<MAG>(P, S, s);
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  for (int64_t base = ((int64_t)blockIdx.x * TC_GROUPS + eng.g) * 128; base < M;
       base += (int64_t)gridDim.x * TC_THREADS) {
    const int64_t i = base + eng.row;
    const bool live = i < M;
    double p[3] = {0.5 * S.dom.r_max, 0.0, S.dom.z_c};
    if (live)
      for (int c = 0; c < 3; c++) p[c] = pts[3 * i + c];
    double E[3], H[3] = {0.0, 0.0, 0.0};
    bool ub;
    const bool ok = eng.field(p, live, E, H, ub);
    if (live) {
      for (int c = 0; c < 3; c++) field[3 * i + c] = ok ? E[c] : nan;
      if (hfield)
        for (int c = 0; c < 3; c++) hfield[3 * i + c] = ok ? H[c] : nan;
      if (used_bem) used_bem[i] = ok ? (ub ? 1 : 0) : -1;
    }
    if (!ok) break;
  }
  tc_teardown(s);
}

}  // namespace tb

using namespace tb;

// cudaFuncSetAttribute once per device and kernel (a later call, e.g. inside
// a stream capture, then only launches).
template <class K>
static int set_smem_once(K* kernel, int bytes, bool (&done)[64]) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CUDA_ERR;
  if (dev >= 0 && dev < 64 && done[dev]) return OK;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    return CUDA_ERR;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return OK;
}
static bool g_attr_trace_tc[2][64], g_attr_points_tc[2][64], g_attr_trace_warp[2][64], g_attr_points_warp[2][64];

// Kernel parameters of a surrogate launch; `mag` is set when the field has a
// magnetic part (coils in the network, a magnetostatic axial table, or
// magnetostatic charges / current rings for the fallback).
static int fill_surrogate_params(const tb_field_t* field, const tb_surrogate_t* sur, TraceParams& P,
                                 SurrogateParams& S, bool& mag) {
  if (!field->axial_z || field->axial_nz < 2 || !field->axial_elec) return BAD_ARG;
  if ((field->n_elec > 0 && !field->elec_sources) || (field->n_mag > 0 && !field->mag_sources) ||
      (field->n_cur > 0 && !field->cur_sources) || field->n_elec < 0 || field->n_mag < 0 || field->n_cur < 0)
    return BAD_ARG;
  const int nsrc = sur->n_electrodes + sur->n_coils;
  if (!sur->weights_bf16 || !sur->params_f32 || sur->n_electrodes < 0 || sur->n_coils < 0 || nsrc < 1 ||
      nsrc > MLP_MAX_SOURCES)
    return BAD_ARG;
  if (sur->n_segments < 0 || sur->n_segments > SG_MAX_SEGS || (sur->n_segments > 0 && !sur->segments)) return BAD_ARG;
  if (!(sur->r_max > 0) || !(sur->z_half > 0) || sur->env_power < 0 || sur->env_power > 32) return BAD_ARG;
  if (sur->engine != 0 && sur->engine != 1) return BAD_ARG;
  mag = sur->n_coils > 0 || field->axial_mag != nullptr || field->n_mag > 0 || field->n_cur > 0;
  memset(&P, 0, sizeof(P));
  P.wait_cycles = wait_limit();
  P.esrc = field->elec_sources;
  P.ne = field->n_elec;
  P.msrc = field->mag_sources;
  P.nm = field->n_mag;
  P.csrc = field->cur_sources;
  P.nc = field->n_cur;
  P.fb = field->field_bounds;
  P.az = field->axial_z;
  P.aec = field->axial_elec;
  P.amc = field->axial_mag;
  P.anz = field->axial_nz;
  memset(&S, 0, sizeof(S));
  S.wb = static_cast<const __nv_bfloat16*>(sur->weights_bf16);
  S.pf = sur->params_f32;
  S.dom = MlpDomain{sur->r_max, sur->z_c, sur->z_half};
  S.z_lo = sur->z_lo;
  S.z_hi = sur->z_hi;
  for (int src = 0; src < nsrc; src++) {
    const double v = sur->strengths[src];
    float* wr = src < sur->n_electrodes ? S.wr : S.hr;
    float* wz = src < sur->n_electrodes ? S.wz : S.hz;
    wr[3 * src + 1] = float(v * double(sur->scale[3 * src + 1]));
    wz[3 * src + 2] = float(v * double(sur->scale[3 * src + 2]));
  }
  S.env_p = sur->env_power;
  S.segs = sur->segments;
  S.nseg = sur->n_segments;
  S.fb_dist2 = sur->fallback_dist * sur->fallback_dist;
  return OK;
}

template <bool MAG>
static int launch_points(const TraceParams& P, const SurrogateParams& S, int engine, const double* points, int64_t M,
                         double* out, double* out_h, int32_t* used_bem, cudaStream_t stream) {
  if (engine == 0) {
    if (set_smem_once(k_surrogate_points_tc<MAG>, TC_SMEM_BYTES, g_attr_points_tc[MAG]) != OK) return CUDA_ERR;
    int64_t blocks = (M + TC_THREADS - 1) / TC_THREADS;
    if (blocks > num_sms()) blocks = num_sms();
    k_surrogate_points_tc<MAG><<<unsigned(blocks), TC_THREADS, TC_SMEM_BYTES, stream>>>(P, S, points, M, out, out_h,
                                                                                      used_bem);
    return launch_status();
  }
  const int smem = int(sizeof(SurrogateSmem));
  if (set_smem_once(k_surrogate_points<MAG>, smem, g_attr_points_warp[MAG]) != OK) return CUDA_ERR;
  int64_t blocks = (M + SG_THREADS - 1) / SG_THREADS;
  if (blocks > 4 * num_sms()) blocks = 4 * num_sms();
  k_surrogate_points<MAG><<<unsigned(blocks), SG_THREADS, smem, stream>>>(P, S, points, M, out, out_h, used_bem);
  return launch_status();
}

extern "C" int tb_surrogate_field_points(const double* points, int64_t M, const tb_field_t* field,
                                         const tb_surrogate_t* sur, double* out, double* out_h, int32_t* used_bem,
                                         tb_stream_t stream) {
  if (!field || !sur || M < 0 || (M > 0 && (!points || !out))) return BAD_ARG;
  if (M == 0) return OK;
  TraceParams P;
  SurrogateParams S;
  bool mag = false;
  int st = fill_surrogate_params(field, sur, P, S, mag);
  if (st != OK) return st;
  if (out_h && !mag) {
    if (cudaMemsetAsync(out_h, 0, sizeof(double) * 3 * M, (cudaStream_t)stream) != cudaSuccess) return CUDA_ERR;
    out_h = nullptr;
  }
  return mag ? launch_points<true>(P, S, sur->engine, points, M, out, out_h, used_bem, (cudaStream_t)stream)
             : launch_points<false>(P, S, sur->engine, points, M, out, out_h, used_bem, (cudaStream_t)stream);
}

template <bool MAG>
static int launch_trace(const TraceParams& P, const SurrogateParams& S, int engine, int64_t n, cudaStream_t s) {
  if (engine == 0) {
    // one CTA (3 groups of 128 particles) per SM; fewer only when there are
    // fewer particles than that
    if (set_smem_once(k_trace_surrogate_tc<MAG>, TC_SMEM_BYTES, g_attr_trace_tc[MAG]) != OK) return CUDA_ERR;
    int64_t blocks = num_sms();
    const int64_t by_work = (n + TC_THREADS - 1) / TC_THREADS;
    if (blocks > by_work) blocks = by_work;
    k_trace_surrogate_tc<MAG><<<unsigned(blocks), TC_THREADS, TC_SMEM_BYTES, s>>>(P, S);
    return launch_status();
  }
  const int smem = int(sizeof(SurrogateSmem));
  if (set_smem_once(k_trace_surrogate<MAG>, smem, g_attr_trace_warp[MAG]) != OK) return CUDA_ERR;
  // one block per SM; fewer only when there is not a warp of particles per SM
  int64_t blocks = num_sms();
  int64_t by_work = (n + 31) / 32;
  if (blocks > by_work) blocks = by_work;
  k_trace_surrogate<MAG><<<unsigned(blocks), SG_THREADS, smem, s>>>(P, S);
  return launch_status();
}

extern "C" int tb_trace_surrogate(const double* start, const double* t0, const double* qm, int64_t n,
                                  const tb_field_t* field, const tb_surrogate_t* sur, const tb_trace_opts_t* opts,
                                  int32_t* status, double* final_state, double* plane, int64_t* counters,
                                  int32_t* work, tb_stream_t stream) {
  if (!field || !sur || !opts || n < 0 || !work) return BAD_ARG;
  if (n == 0) return OK;
  if (n > 0x3fffffff || !start || !qm) return BAD_ARG;
  if (opts->max_attempts <= 0 || !(opts->atol > 0)) return BAD_ARG;
  TraceParams P;
  SurrogateParams S;
  bool mag = false;
  int st = fill_surrogate_params(field, sur, P, S, mag);
  if (st != OK) return st;
  for (int i = 0; i < 6; i++) P.bounds[i] = opts->bounds[i];
  P.atol = opts->atol;
  P.plane_z = opts->plane_z;
  P.record_plane = opts->record_plane;
  P.max_attempts = opts->max_attempts < 0x7fffffff ? opts->max_attempts : 0x7fffffff;
  P.start = start;
  P.t0 = t0;
  P.qm = qm;
  P.n = n;
  P.status = status;
  P.final_state = final_state;
  P.plane = plane;
  P.counters = counters;
  P.work = work;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(work, 0, sizeof(int32_t), s) != cudaSuccess) return CUDA_ERR;
  return mag ? launch_trace<true>(P, S, sur->engine, n, s) : launch_trace<false>(P, S, sur->engine, n, s);
}

static int trace_rk45(const double* start, const double* t0, const double* qm, const int32_t* geom, int64_t n,
                      const tb_field_t* field, const int64_t* src_offsets, int64_t n_geoms,
                      const double* geom_bounds, const tb_trace_opts_t* opts,
                      double* rows, int64_t* nrows, int32_t* status, double* final_state, double* plane,
                      int64_t* counters, int32_t* work, tb_stream_t stream) {
  if (!field || !opts || n < 0 || !work) return BAD_ARG;
  if (n == 0) return OK;
  if (n > 0x7fffffff || !start || !qm) return BAD_ARG;
  if (opts->max_attempts <= 0 || !(opts->atol > 0)) return BAD_ARG;
  if (rows && opts->max_rows < 2) return BAD_ARG;
  bool axial = field->axial_z != nullptr;
  if (axial && (field->axial_nz < 2 || !field->axial_elec)) return BAD_ARG;
  if (!axial && ((field->n_elec > 0 && !field->elec_sources) || (field->n_mag > 0 && !field->mag_sources)))
    return BAD_ARG;
  if (field->n_elec < 0 || field->n_mag < 0 || field->n_cur < 0) return BAD_ARG;
  if (!axial && field->n_cur > 0 && !field->cur_sources) return BAD_ARG;
  TraceParams P;
  P.esrc = field->elec_sources;
  P.ne = field->n_elec;
  P.msrc = field->mag_sources;
  P.nm = field->n_mag;
  P.csrc = field->cur_sources;
  P.nc = field->n_cur;
  P.fb = field->field_bounds;
  P.az = field->axial_z;
  P.aec = field->axial_elec;
  P.amc = field->axial_mag;
  P.anz = field->axial_nz;
  for (int i = 0; i < 6; i++) P.bounds[i] = opts->bounds[i];
  P.atol = opts->atol;
  P.plane_z = opts->plane_z;
  P.record_plane = opts->record_plane;
  P.max_attempts = opts->max_attempts;
  P.max_rows = rows ? opts->max_rows : 0;
  P.start = start;
  P.t0 = t0;
  P.qm = qm;
  P.n = n;
  P.rows = rows;
  P.nrows = nrows;
  P.status = status;
  P.final_state = final_state;
  P.plane = plane;
  P.counters = counters;
  P.work = work;
  if (geom) {  // many geometries: BEM electrostatic sources only
    if (axial || field->n_mag > 0 || field->n_cur > 0 || !src_offsets || n_geoms <= 0) return BAD_ARG;
    P.geom = geom;
    P.eoff = src_offsets;
    P.ngeom = n_geoms;
    P.gbounds = geom_bounds;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(work, 0, sizeof(int32_t), s) != cudaSuccess) return CUDA_ERR;
  if (axial) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_axial, 128, 0) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    int64_t blocks = (int64_t)num_sms() * per_sm;
    int64_t by_work = (n + 127) / 128;
    if (blocks > by_work) blocks = by_work;
    k_trace_axial<<<unsigned(blocks), 128, 0, s>>>(P);
    return launch_status();
  }
  int tw = opts->team_warps;
  if (tw == 0) {
    // Fill the GPU: about 32 resident warps per SM.
    int64_t want = (int64_t)num_sms() * 32;
    tw = 1;
    while (tw < 8 && n * tw * 2 <= want) tw *= 2;
  }
  switch (tw) {
    case 1: return P.geom ? launch_bem<1, true>(P, s) : launch_bem<1, false>(P, s);
    case 2: return P.geom ? launch_bem<2, true>(P, s) : launch_bem<2, false>(P, s);
    case 4: return P.geom ? launch_bem<4, true>(P, s) : launch_bem<4, false>(P, s);
    case 8: return P.geom ? launch_bem<8, true>(P, s) : launch_bem<8, false>(P, s);
    default: return BAD_ARG;
  }
}

extern "C" int tb_trace_rk45(const double* start, const double* t0, const double* qm, int64_t n,
                             const tb_field_t* field, const tb_trace_opts_t* opts, double* rows, int64_t* nrows,
                             int32_t* status, double* final_state, double* plane, int64_t* counters, int32_t* work,
                             tb_stream_t stream) {
  return trace_rk45(start, t0, qm, nullptr, n, field, nullptr, 0, nullptr, opts, rows, nrows, status, final_state, plane,
                    counters, work, stream);
}

extern "C" int tb_trace_rk45_geometries(const double* start, const double* t0, const double* qm, const int32_t* geom,
                                        int64_t n, const tb_field_t* field, const int64_t* src_offsets,
                                        int64_t n_geoms, const double* geom_bounds, const tb_trace_opts_t* opts,
                                        double* rows, int64_t* nrows,
                                        int32_t* status, double* final_state, double* plane, int64_t* counters,
                                        int32_t* work, tb_stream_t stream) {
  if (n > 0 && !geom) return BAD_ARG;
  if (n == 0) return OK;
  return trace_rk45(start, t0, qm, geom, n, field, src_offsets, n_geoms, geom_bounds, opts, rows, nrows, status,
                    final_state,
                    plane, counters, work, stream);
}

extern "C" int tb_num_sms(void) { return num_sms(); }

extern "C" int64_t tb_set_wait_limit(int64_t cycles) {
  return wait_limit_cycles().exchange(cycles >= 1 ? (long long)cycles : DEFAULT_WAIT_CYCLES);
}
