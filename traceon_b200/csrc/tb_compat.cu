// tb_compat.cu -- the reference-compatible C ABI (host pointers).
//
// Same names, argument order and meaning as the reference C backend's
// exported functions (traceon/backend/*.c, bound by
// traceon/backend/__init__.py:287-353), so that the reference's ctypes shim
// can load this library instead.  Array work is copied to the device and
// run by the CUDA kernels of tb_bem.cu / tb_trace.cu; scalar helpers run on
// the host through the same __host__ __device__ functions.
#include <cmath>
#include <cstring>
#include <vector>

#include "tb_common.cuh"
#include "tb_internal.cuh"
#include "../../include/traceon_b200.h"

using namespace tb;

extern "C" {
extern const size_t TRACING_BLOCK_SIZE = 100000;  // tracing.c:7
extern const int DERIV_2D_MAX_SYM = NDERIV;
extern const int N_QUAD_2D_SYM = NQ;
extern const int N_TRIANGLE_QUAD_SYM = NTRI;
extern const int NU_MAX_SYM = 4;
extern const int M_MAX_SYM = 8;
}

namespace {

thread_local int g_status = OK;

inline void set_status(int s) { g_status = s; }

// Device buffer owned for the duration of one compat call.
struct DevBuf {
  void* p = nullptr;
  bool ok = true;
  explicit DevBuf(size_t bytes) {
    if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) {
      p = nullptr;
      ok = false;
    }
  }
  DevBuf(const void* host, size_t bytes) : DevBuf(bytes) {
    if (ok && bytes && cudaMemcpy(p, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

inline bool all_ok(std::initializer_list<const DevBuf*> bs) {
  for (auto b : bs)
    if (!b->ok) return false;
  return true;
}

inline int sync_status(int st) {
  if (st != OK) return st;
  return cudaDeviceSynchronize() == cudaSuccess ? OK : CUDA_ERR;
}

// struct effective_point_charges_2d / _3d, radial.c:10-15 / three_d.c:18-23
struct EffCharges {
  double* charges;
  double* jacobians;
  double* positions;
  size_t N;
};
// struct field_evaluation_args, radial.c:175-180
struct FieldEvalArgs {
  void* elec_charges;
  void* mag_charges;
  void* currents;
  double* bounds;
};
// struct field_derivs_args, three_d.c:26-31
struct FieldDerivsArgs {
  double* z;
  double* elec_coeffs;
  double* mag_coeffs;
  size_t N_z;
};
// struct self_field_dot_normal_radial_args, radial.c:198-201
struct SelfFluxArgs {
  double* line_points;
  double K;
};

// Charges of one effective_point_charges_2d uploaded and packed as sources.
struct DevSources {
  DevBuf src;
  int64_t n = 0;
  bool ok = true;
  DevSources(const double* q, const double* jac, const double* pos, size_t N, bool current)
      : src(size_t(3) * N * (current ? NTRI : NQ) * sizeof(double)) {
    const int nq = current ? NTRI : NQ;
    n = int64_t(N) * nq;
    if (N == 0) return;
    DevBuf dq(q, N * sizeof(double)), dj(jac, N * nq * sizeof(double)),
        dp(pos, N * nq * (current ? 3 : 2) * sizeof(double));
    ok = src.ok && all_ok({&dq, &dj, &dp});
    if (!ok) return;
    int st = current ? tb_pack_current_sources(dq.as<double>(), dj.as<double>(), dp.as<double>(), src.as<double>(),
                                               int64_t(N), nullptr)
                     : tb_pack_sources(dq.as<double>(), dj.as<double>(), dp.as<double>(), src.as<double>(),
                                       int64_t(N), nullptr);
    ok = sync_status(st) == OK;
  }
};

}  // namespace

extern "C" {

int tb_last_status(void) { return g_status; }

// ------------------------------------------------------------ host scalars
double ellipkm1(double p) { return tb::ellipkm1(p); }
double ellipk(double k) { return tb::ellipk(k); }
double ellipem1(double p) { return tb::ellipem1(p); }
double ellipe(double k) { return tb::ellipe(k); }

void normal_2d(const double* p1, const double* p2, double* normal) {
  double tx = p2[0] - p1[0], ty = p2[1] - p1[1];
  double nx = ty, ny = -tx, l = std::sqrt(nx * nx + ny * ny);
  normal[0] = nx / l;
  normal[1] = ny / l;
}

void higher_order_normal_radial(double alpha, const double* v1, const double* v2, const double* v3, const double* v4,
                                double* normal) {
  Cubic c;
  c.load4(v1, v2, v3, v4);
  c.normal(alpha, normal[0], normal[1]);
}

void position_and_jacobian_radial(double alpha, const double* v1, const double* v2, const double* v3,
                                  const double* v4, double* pos, double* jac) {
  Cubic c;
  c.load4(v1, v2, v3, v4);
  c.point(alpha, false, pos[0], pos[1], *jac);
}

void delta_position_and_jacobian_radial(double alpha, const double* v1, const double* v2, const double* v3,
                                        const double* v4, double* pos, double* jac) {
  Cubic c;
  c.load4(v1, v2, v3, v4);
  c.point(alpha, true, pos[0], pos[1], *jac);
}

double potential_radial_ring(double r0, double z0, double dr, double dz, void*) {
  return tb::potential_radial_ring(r0, z0, dr, dz);
}
double dr1_potential_radial_ring(double r0, double z0, double dr, double dz, void*) {
  return tb::dr1_potential_radial_ring(r0, z0, dr, dz);
}
double dz1_potential_radial_ring(double r0, double z0, double dr, double dz, void*) {
  return tb::dz1_potential_radial_ring(r0, z0, dr, dz);
}
double flux_density_to_charge_factor(double K) { return flux_factor(K); }

double charge_radial(const double* vertices, double charge) {
  Cubic c;
  c.load(vertices);
  double s = 0;
  for (int k = 0; k < NQ; k++) {
    double r, z, j;
    c.point(gauss_x(k), false, r, z, j);
    s += 2 * PI * r * gauss_w(k) * j * charge;
  }
  return s;
}

void current_field_radial_ring(double x0, double y0, double x, double y, double* result) {
  current_field_ring(x0, y0, x, y, result[0], result[1]);
}

double current_potential_axial_radial_ring(double z0, double r, double z) {
  double dz = z0 - z;
  return -dz / (2 * std::sqrt(dz * dz + r * r));
}

double self_potential_radial(double alpha, void* line_points) {
  Cubic c;
  c.load(static_cast<const double*>(line_points));
  double tr, tz, tj, dr, dz, j;
  c.point(0.0, false, tr, tz, tj);
  c.point(alpha, true, dr, dz, j);
  return j * tb::potential_radial_ring(tr, tz, dr, dz);
}

double self_field_dot_normal_radial(double alpha, void* args) {
  const SelfFluxArgs* a = static_cast<const SelfFluxArgs*>(args);
  Cubic c;
  c.load(a->line_points);
  double tr, tz, tj, dr, dz, j, nr, nz;
  c.point(0.0, false, tr, tz, tj);
  c.point(alpha, true, dr, dz, j);
  c.normal(0.0, nr, nz);
  return j * field_dot_normal_ring(tr, tz, dr, dz, nr, nz, flux_factor(a->K));
}

double potential_radial_derivs(const double* point, const double* z, const double* coeffs, size_t N_z) {
  double d[NDERIV];
  if (N_z < 2 || !axial_eval(point[2], z, coeffs, int64_t(N_z), d)) return 0.0;
  return axial_potential(d, point[0] * point[0] + point[1] * point[1]);
}

void field_radial_derivs(const double* point, double* field, const double* z, const double* coeffs, size_t N_z) {
  double d[NDERIV];
  if (N_z < 2 || !axial_eval(point[2], z, coeffs, int64_t(N_z), d)) {
    field[0] = field[1] = field[2] = 0.0;
    return;
  }
  axial_field(d, point, point[0] * point[0] + point[1] * point[1], field);
}

bool plane_intersection(const double* p0, const double* n, const double* pos, size_t N_p, double* result) {
  if (N_p < 2) return false;
  double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  auto kappa = [&](size_t i) {
    const double* s = pos + 6 * i;
    return (n[2] * p0[2] - s[2] * n[2] + n[1] * p0[1] - s[1] * n[1] + n[0] * p0[0] - s[0] * n[0]) / nn;
  };
  double prev = kappa(N_p - 1);
  for (size_t ii = N_p - 1; ii-- > 0;) {
    double k = kappa(ii);
    if ((k > 0) != (prev > 0)) {
      double diff = k - prev, f = -prev / diff, pf = k / diff;
      for (int c = 0; c < 6; c++) result[c] = pf * pos[6 * (ii + 1) + c] + f * pos[6 * ii + c];
      return true;
    }
    prev = k;
  }
  return false;
}

// ------------------------------------------------------------ GPU arrays
void fill_jacobian_buffer_radial(double* jac, double* pos, const double* vertices, size_t N) {
  set_status(OK);
  if (N == 0) return;
  DevBuf dv(vertices, N * 12 * sizeof(double)), dj(N * NQ * sizeof(double)), dp(N * NQ * 2 * sizeof(double));
  if (!all_ok({&dv, &dj, &dp})) return set_status(CUDA_ERR);
  int st = sync_status(tb_jacobian_buffer_radial(dv.as<double>(), dj.as<double>(), dp.as<double>(), int64_t(N), nullptr));
  if (st == OK && cudaMemcpy(jac, dj.p, N * NQ * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) st = CUDA_ERR;
  if (st == OK && cudaMemcpy(pos, dp.p, N * NQ * 2 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = CUDA_ERR;
  set_status(st);
}

void fill_matrix_radial(double* matrix, const double* lines, const uint8_t* types, const double* values,
                        const double* jac, const double* pos, size_t N_lines, size_t N_matrix, int start, int end) {
  set_status(OK);
  if (start < 0 || end < start || size_t(end) >= N_lines || N_matrix < N_lines) return set_status(BAD_ARG);
  for (int i = start; i <= end; i++) {
    int t = types[i];
    if (!(t == VOLTAGE_FIXED || t == VOLTAGE_FUN || t == MAGNETOSTATIC_POT || t == DIELECTRIC || t == MAGNETIZABLE))
      return set_status(BAD_ARG);  // the reference prints and exit(1)s, radial.c:305-308
  }
  const size_t N = N_lines, rows = size_t(end - start + 1);
  DevBuf dA(rows * N_matrix * sizeof(double)), dv(lines, N * 12 * sizeof(double)), dt(types, N),
      dval(values, N * sizeof(double)), dj(jac, N * NQ * sizeof(double)), dp(pos, N * NQ * 2 * sizeof(double));
  if (!all_ok({&dA, &dv, &dt, &dval, &dj, &dp})) return set_status(CUDA_ERR);
  double* hrow = matrix + size_t(start) * N_matrix;
  if (cudaMemcpy(dA.p, hrow, rows * N_matrix * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_status(CUDA_ERR);
  // the device block holds rows [start, end]; shift the matrix origin so
  // row `start` lands on its first row
  double* origin = dA.as<double>() - int64_t(start) * int64_t(N_matrix);
  int st = sync_status(tb_fill_matrix_radial(origin, int64_t(N_matrix), dv.as<double>(), dt.as<uint8_t>(),
                                             dval.as<double>(), dj.as<double>(), dp.as<double>(), int64_t(N), start,
                                             int64_t(end) + 1, 1, 1, nullptr));
  if (st == OK && cudaMemcpy(hrow, dA.p, rows * N_matrix * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = CUDA_ERR;
  set_status(st);
}

static void field_or_potential(const double* point, const double* q, const double* jac, const double* pos, size_t N,
                               double* pot, double* field) {
  set_status(OK);
  if (pot) *pot = 0.0;
  if (field) field[0] = field[1] = field[2] = 0.0;
  DevSources s(q, jac, pos, N, false);
  DevBuf dp(point, 3 * sizeof(double)), dout(4 * sizeof(double));
  if (!s.ok || !all_ok({&dp, &dout})) return set_status(CUDA_ERR);
  double* d = dout.as<double>();
  int st = sync_status(tb_field_radial_points(dp.as<double>(), 1, s.src.as<double>(), s.n, pot ? d : nullptr,
                                              field ? d + 1 : nullptr, nullptr));
  double h[4] = {0, 0, 0, 0};
  if (st == OK && cudaMemcpy(h, d, 4 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) st = CUDA_ERR;
  if (st == OK) {
    if (pot) *pot = h[0];
    if (field) std::memcpy(field, h + 1, 3 * sizeof(double));
  }
  set_status(st);
}

double potential_radial(const double* point, const double* charges, const double* jac, const double* pos, size_t N) {
  double p = 0.0;
  field_or_potential(point, charges, jac, pos, N, &p, nullptr);
  return p;
}

void field_radial(const double* point, double* result, const double* charges, const double* jac, const double* pos,
                  size_t N) {
  field_or_potential(point, charges, jac, pos, N, nullptr, result);
}

static void axial_common(double* derivs, const double* q, const double* jac, const double* pos, size_t N,
                         const double* z, size_t Nz, bool current) {
  set_status(OK);
  if (Nz == 0) return;
  DevSources s(q, jac, pos, N, current);
  DevBuf dz(z, Nz * sizeof(double)), dd(Nz * NDERIV * sizeof(double));
  if (!s.ok || !all_ok({&dz, &dd})) return set_status(CUDA_ERR);
  int st = current ? tb_current_axial_derivatives(dz.as<double>(), int64_t(Nz), s.src.as<double>(), s.n,
                                                  dd.as<double>(), nullptr)
                   : tb_axial_derivatives_radial(dz.as<double>(), int64_t(Nz), s.src.as<double>(), s.n,
                                                 dd.as<double>(), nullptr);
  st = sync_status(st);
  std::vector<double> h(Nz * NDERIV);
  if (st == OK && cudaMemcpy(h.data(), dd.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = CUDA_ERR;
  if (st == OK)
    for (size_t i = 0; i < h.size(); i++) derivs[i] += h[i];  // the reference accumulates
  set_status(st);
}

void axial_derivatives_radial(double* derivs, const double* charges, const double* jac, const double* pos, size_t N,
                              const double* z, size_t N_z) {
  axial_common(derivs, charges, jac, pos, N, z, N_z, false);
}

void current_axial_derivatives_radial(double* derivs, const double* currents, const double* jac, const double* pos,
                                      size_t N, const double* z, size_t N_z) {
  axial_common(derivs, currents, jac, pos, N, z, N_z, true);
}

double current_potential_axial(double z0, const double* currents, const double* jac, const double* pos, size_t N) {
  double d[NDERIV] = {0};
  axial_common(d, currents, jac, pos, N, &z0, 1, true);
  return d[0];
}

void current_field_radial(const double* point, double* result, const double* currents, const double* jac,
                          const double* pos, size_t N) {
  set_status(OK);
  result[0] = result[1] = result[2] = 0.0;
  DevSources s(currents, jac, pos, N, true);
  DevBuf dp(point, 3 * sizeof(double)), dout(3 * sizeof(double));
  if (!s.ok || !all_ok({&dp, &dout})) return set_status(CUDA_ERR);
  int st = sync_status(tb_current_field_points(dp.as<double>(), 1, s.src.as<double>(), s.n, dout.as<double>(), nullptr));
  if (st == OK && cudaMemcpy(result, dout.p, 3 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = CUDA_ERR;
  set_status(st);
}

// ------------------------------------------------------------ tracing
void field_radial_derivs_traceable(const double* position, const double*, void* args_p, double* elec_out,
                                   double* mag_out) {
  const FieldDerivsArgs* a = static_cast<const FieldDerivsArgs*>(args_p);
  field_radial_derivs(position, elec_out, a->z, a->elec_coeffs, a->N_z);
  field_radial_derivs(position, mag_out, a->z, a->mag_coeffs, a->N_z);
}

// One evaluation of the BEM field for the tracer callback, on the GPU
// through the tracer's own field code (a zero-length trace is not possible,
// so this evaluates the sums with the point kernels).
void field_radial_traceable(const double* position, const double*, void* args_p, double* elec_out,
                            double* mag_out) {
  const FieldEvalArgs* a = static_cast<const FieldEvalArgs*>(args_p);
  const double* b = a->bounds;
  bool inside = b == nullptr || (b[0] < position[0] && position[0] < b[1] && b[2] < position[1] &&
                                 position[1] < b[3] && b[4] < position[2] && position[2] < b[5]);
  for (int c = 0; c < 3; c++) elec_out[c] = mag_out[c] = 0.0;
  if (!inside) return;
  const EffCharges* e = static_cast<const EffCharges*>(a->elec_charges);
  const EffCharges* m = static_cast<const EffCharges*>(a->mag_charges);
  const EffCharges* c = static_cast<const EffCharges*>(a->currents);
  field_radial(position, elec_out, e->charges, e->jacobians, e->positions, e->N);
  int st = g_status;
  field_radial(position, mag_out, m->charges, m->jacobians, m->positions, m->N);
  st = st != OK ? st : g_status;
  double cur[3] = {0, 0, 0};
  current_field_radial(position, cur, c->charges, c->jacobians, c->positions, c->N);
  st = st != OK ? st : g_status;
  for (int k = 0; k < 3; k++) mag_out[k] += cur[k];
  set_status(st);
}

size_t trace_particle(double* times, double* positions, double qm, void* field, const double* bounds, double atol,
                      void* args) {
  set_status(OK);
  const bool bem = field == reinterpret_cast<void*>(&field_radial_traceable);
  const bool axial = field == reinterpret_cast<void*>(&field_radial_derivs_traceable);
  if (!bem && !axial) {
    // A host callback (e.g. a Python field) cannot run inside the GPU
    // integrator; report it instead of integrating on the CPU.
    set_status(UNSUPPORTED);
    return 1;
  }
  const size_t max_rows = TRACING_BLOCK_SIZE;
  tb_trace_opts_t o;
  for (int i = 0; i < 6; i++) o.bounds[i] = bounds[i];
  o.atol = atol;
  o.plane_z = 0.0;
  o.record_plane = 0;
  o.max_attempts = int64_t(20) * int64_t(max_rows);
  o.max_rows = int64_t(max_rows);
  o.team_warps = 8;
  tb_field_t f;
  std::memset(&f, 0, sizeof(f));
  double st6[6];
  std::memcpy(st6, positions, sizeof(st6));
  DevBuf dstart(st6, sizeof(st6)), dt0(times, sizeof(double)), dqm(&qm, sizeof(double));
  DevBuf drows(max_rows * 7 * sizeof(double)), dn(sizeof(int64_t)), dstat(sizeof(int32_t)), dwork(sizeof(int32_t));
  if (!all_ok({&dstart, &dt0, &dqm, &drows, &dn, &dstat, &dwork})) {
    set_status(CUDA_ERR);
    return 1;
  }
  int st;
  if (bem) {
    const FieldEvalArgs* a = static_cast<const FieldEvalArgs*>(args);
    const EffCharges* e = static_cast<const EffCharges*>(a->elec_charges);
    const EffCharges* m = static_cast<const EffCharges*>(a->mag_charges);
    const EffCharges* c = static_cast<const EffCharges*>(a->currents);
    DevSources se(e->charges, e->jacobians, e->positions, e->N, false);
    DevSources sm(m->charges, m->jacobians, m->positions, m->N, false);
    DevSources sc(c->charges, c->jacobians, c->positions, c->N, true);
    DevBuf dfb(a->bounds, a->bounds ? 6 * sizeof(double) : 0);
    if (!se.ok || !sm.ok || !sc.ok || !dfb.ok) {
      set_status(CUDA_ERR);
      return 1;
    }
    f.elec_sources = se.src.as<double>();
    f.n_elec = se.n;
    f.mag_sources = sm.src.as<double>();
    f.n_mag = sm.n;
    f.cur_sources = sc.src.as<double>();
    f.n_cur = sc.n;
    f.field_bounds = a->bounds ? dfb.as<double>() : nullptr;
    st = sync_status(tb_trace_rk45(dstart.as<double>(), dt0.as<double>(), dqm.as<double>(), 1, &f, &o,
                                   drows.as<double>(), dn.as<int64_t>(), dstat.as<int32_t>(), nullptr, nullptr, nullptr,
                                   dwork.as<int32_t>(), nullptr));
  } else {
    const FieldDerivsArgs* a = static_cast<const FieldDerivsArgs*>(args);
    size_t nz = a->N_z;
    size_t nc = (nz - 1) * NDERIV * 6;
    DevBuf dz(a->z, nz * sizeof(double)), de(a->elec_coeffs, nc * sizeof(double)),
        dm(a->mag_coeffs, nc * sizeof(double));
    if (!all_ok({&dz, &de, &dm}) || nz < 2) {
      set_status(nz < 2 ? BAD_ARG : CUDA_ERR);
      return 1;
    }
    f.axial_z = dz.as<double>();
    f.axial_elec = de.as<double>();
    f.axial_mag = dm.as<double>();
    f.axial_nz = int64_t(nz);
    st = sync_status(tb_trace_rk45(dstart.as<double>(), dt0.as<double>(), dqm.as<double>(), 1, &f, &o,
                                   drows.as<double>(), dn.as<int64_t>(), dstat.as<int32_t>(), nullptr, nullptr, nullptr,
                                   dwork.as<int32_t>(), nullptr));
  }
  if (st != OK) {
    set_status(st);
    return 1;
  }
  int64_t n = 1;
  if (cudaMemcpy(&n, dn.p, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess || n < 1 || size_t(n) > max_rows) {
    set_status(CUDA_ERR);
    return 1;
  }
  std::vector<double> rows(size_t(n) * 7);
  if (cudaMemcpy(rows.data(), drows.p, rows.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_status(CUDA_ERR);
    return 1;
  }
  for (int64_t i = 0; i < n; i++) {
    times[i] = rows[i * 7];
    for (int c = 0; c < 6; c++) positions[i * 6 + c] = rows[i * 7 + 1 + c];
  }
  return size_t(n);
}

// ------------------------------------------------------------ outside the path
double kronrod_adaptive(void*, double, double, void*, double, double) {
  set_status(UNSUPPORTED);
  return std::nan("");
}
void normal_3d(const double*, double*) { set_status(UNSUPPORTED); }
void position_and_jacobian_3d(double, double, const double*, double*, double*) { set_status(UNSUPPORTED); }
void axial_coefficients_3d(const double*, const double*, const double*, double*, double*, size_t, const double*,
                           double*, size_t) {
  set_status(UNSUPPORTED);
}
void fill_jacobian_buffer_current_three_d(const double*, double*, double*, double*, size_t) { set_status(UNSUPPORTED); }
double potential_3d_derivs(const double*, const double*, const double*, size_t) {
  set_status(UNSUPPORTED);
  return std::nan("");
}
void field_3d_derivs(const double*, double*, const double*, const double*, size_t) { set_status(UNSUPPORTED); }
void fill_jacobian_buffer_3d(double*, double*, const double*, size_t) { set_status(UNSUPPORTED); }
void triangle_areas(const double*, double*, size_t) { set_status(UNSUPPORTED); }

}  // extern "C"
