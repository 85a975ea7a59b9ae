"""ctypes shim over libtraceon_b200.so: the ``traceon.backend`` call surface.

Mirrors traceon/backend/__init__.py of the reference: the library is located
next to this file and loaded with ``ctypes.CDLL`` (reference :23-55), the
compile-time constants are read with ``in_dll`` (:58-66), and the wrapper
functions keep the reference's names, argument order, shape checks and return
values (:355-780).  All array work runs on the GPU inside the library.

Two differences, both by design:

* the singular self terms ``self_potential_radial`` /
  ``self_field_dot_normal_radial`` are integrated on the GPU (composite
  Gauss-Legendre graded toward the singularity) instead of by SciPy QUADPACK
  over a C callback (reference :688-708);
* ``trace_particle`` integrates on the GPU and therefore accepts only this
  library's own field callbacks (``field_radial_traceable`` /
  ``field_radial_derivs_traceable``); a Python field callback raises
  ``NotImplementedError`` instead of running a CPU integrator.

The ``dev_*`` functions are the batched device API (torch tensors in, torch
tensors out, on the current CUDA stream).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

DEBUG = False

_LIB_PATH = _build.LIB
if not os.path.isfile(_LIB_PATH):
    raise RuntimeError(
        f'Cannot find the traceon_b200 CUDA library ({_LIB_PATH}). Build it with '
        '`python -m traceon_b200.build` (nvcc, sm_100a).')

backend_lib = C.CDLL(_LIB_PATH)

TRACING_BLOCK_SIZE = C.c_size_t.in_dll(backend_lib, 'TRACING_BLOCK_SIZE').value
DERIV_2D_MAX = C.c_int.in_dll(backend_lib, 'DERIV_2D_MAX_SYM').value
N_QUAD_2D = C.c_int.in_dll(backend_lib, 'N_QUAD_2D_SYM').value
N_TRIANGLE_QUAD = C.c_int.in_dll(backend_lib, 'N_TRIANGLE_QUAD_SYM').value
NU_MAX = C.c_int.in_dll(backend_lib, 'NU_MAX_SYM').value
M_MAX = C.c_int.in_dll(backend_lib, 'M_MAX_SYM').value

TB_OK, TB_BAD_ARG, TB_CUDA_ERR, TB_NONFINITE, TB_UNSUPPORTED, TB_SINGULAR, TB_TIMEOUT = range(7)
TRACE_EXITED, TRACE_MAX_ATTEMPTS, TRACE_ROWS_FULL, TRACE_NONFINITE, TRACE_ENGINE_TIMEOUT = range(5)

dbl = C.c_double
dbl_p = C.POINTER(dbl)
vp = C.c_void_p
sz = C.c_size_t
i64 = C.c_int64


class BackendError(RuntimeError):
    pass


def _arr(ndim=None, shape=None, dtype=np.float64):
    return np.ctypeslib.ndpointer(ndim=ndim, shape=shape, dtype=dtype, flags=('C_CONTIGUOUS', 'ALIGNED'))


v2 = _arr(shape=(2,))
v3 = _arr(shape=(3,))

# field_fun, traceon/backend/__init__.py:89
field_fun = C.CFUNCTYPE(None, dbl_p, dbl_p, vp, dbl_p, dbl_p)
integration_cb_1d = C.CFUNCTYPE(dbl, dbl, vp)


class EffectivePointCharges2D(C.Structure):
    """struct effective_point_charges_2d (reference radial.c:10-15)"""
    _fields_ = [("charges", dbl_p), ("jacobians", dbl_p), ("positions", dbl_p), ("N", C.c_size_t)]

    def __init__(self, eff, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.charges_arr = ensure_contiguous_aligned(np.asarray(eff.charges, dtype=np.float64))
        self.jacobians_arr = ensure_contiguous_aligned(np.asarray(eff.jacobians, dtype=np.float64))
        self.positions_arr = ensure_contiguous_aligned(np.asarray(eff.positions, dtype=np.float64))
        self.charges = self.charges_arr.ctypes.data_as(dbl_p)
        self.jacobians = self.jacobians_arr.ctypes.data_as(dbl_p)
        self.positions = self.positions_arr.ctypes.data_as(dbl_p)
        self.N = len(self.charges_arr)


EffectivePointCharges3D = EffectivePointCharges2D  # same layout (three_d.c:18-23)


class FieldEvaluationArgsRadial(C.Structure):
    """struct field_evaluation_args (reference radial.c:175-180)"""
    _fields_ = [("elec_charges", C.c_void_p), ("mag_charges", C.c_void_p), ("current_charges", C.c_void_p),
                ("bounds", dbl_p)]

    def __init__(self, elec, mag, current, bounds, *args, **kwargs):
        super().__init__(*args, **kwargs)
        assert bounds is None or np.shape(bounds) == (3, 2)
        self.eff_elec = EffectivePointCharges2D(elec)
        self.eff_mag = EffectivePointCharges2D(mag)
        self.eff_current = EffectivePointCharges3D(current)
        self.elec_charges = C.cast(C.pointer(self.eff_elec), C.c_void_p)
        self.mag_charges = C.cast(C.pointer(self.eff_mag), C.c_void_p)
        self.current_charges = C.cast(C.pointer(self.eff_current), C.c_void_p)
        if bounds is None:
            self.bounds = None
        else:
            self.bounds_arr = ensure_contiguous_aligned(np.asarray(bounds, dtype=np.float64))
            self.bounds = self.bounds_arr.ctypes.data_as(dbl_p)


class FieldDerivsArgs(C.Structure):
    """struct field_derivs_args (reference three_d.c:26-31)"""
    _fields_ = [("z_interpolation", dbl_p), ("electrostatic_axial_coeffs", dbl_p),
                ("magnetostatic_axial_coeffs", dbl_p), ("N_z", C.c_size_t)]

    def __init__(self, z, elec, mag, *args, **kwargs):
        super().__init__(*args, **kwargs)
        assert z.shape == (len(z),) and elec.shape[0] == len(z) - 1 and mag.shape[0] == len(z) - 1
        self.z_arr = ensure_contiguous_aligned(z)
        self.elec_arr = ensure_contiguous_aligned(elec)
        self.mag_arr = ensure_contiguous_aligned(mag)
        self.z_interpolation = self.z_arr.ctypes.data_as(dbl_p)
        self.electrostatic_axial_coeffs = self.elec_arr.ctypes.data_as(dbl_p)
        self.magnetostatic_axial_coeffs = self.mag_arr.ctypes.data_as(dbl_p)
        self.N_z = len(z)


class SelfFieldDotNormalRadialArgs(C.Structure):
    _fields_ = [("line_points", dbl_p), ("K", C.c_double)]


class TbField(C.Structure):
    """tb_field_t of include/traceon_b200.h"""
    _fields_ = [("elec_sources", vp), ("n_elec", i64), ("mag_sources", vp), ("n_mag", i64),
                ("cur_sources", vp), ("n_cur", i64), ("field_bounds", vp), ("axial_z", vp),
                ("axial_elec", vp), ("axial_mag", vp), ("axial_nz", i64)]


class TbGeometry(C.Structure):
    """tb_geometry_t of include/traceon_b200.h"""
    _fields_ = [("vertices", vp), ("types", vp), ("values", vp), ("jac", vp), ("pos", vp), ("A", vp),
                ("lda", i64), ("N", i64), ("tile0", i64), ("elem0", i64)]


class TbBatchItem(C.Structure):
    """tb_batch_item_t of include/traceon_b200.h"""
    _fields_ = [("vertices", vp), ("types", vp), ("values", vp), ("rhs", vp), ("charges", vp), ("N", i64),
                ("T", i64), ("a_off", i64), ("inv_off", i64), ("v_off", i64), ("flag_off", i64), ("ring_off", i64)]


class TbTraceOpts(C.Structure):
    """tb_trace_opts_t of include/traceon_b200.h"""
    _fields_ = [("bounds", dbl * 6), ("atol", dbl), ("plane_z", dbl), ("record_plane", C.c_int),
                ("max_attempts", i64), ("max_rows", i64), ("team_warps", C.c_int)]


def ensure_contiguous_aligned(arr):
    assert isinstance(arr, np.ndarray)
    return np.require(arr, requirements=('C_CONTIGUOUS', 'ALIGNED'))


# Reference-compatible signature table (traceon/backend/__init__.py:287-328).
backend_functions = {
    'ellipkm1': (dbl, dbl),
    'ellipk': (dbl, dbl),
    'ellipem1': (dbl, dbl),
    'ellipe': (dbl, dbl),
    'normal_2d': (None, v2, v2, v2),
    'higher_order_normal_radial': (None, dbl, v3, v3, v3, v3, v2),
    'position_and_jacobian_radial': (None, dbl, v3, v3, v3, v3, v2, dbl_p),
    'delta_position_and_jacobian_radial': (None, dbl, v3, v3, v3, v3, v2, dbl_p),
    'trace_particle': (sz, _arr(shape=(TRACING_BLOCK_SIZE,)), _arr(shape=(TRACING_BLOCK_SIZE, 6)), dbl, vp,
                       _arr(shape=(3, 2)), dbl, vp),
    'potential_radial_ring': (dbl, dbl, dbl, dbl, dbl, vp),
    'dr1_potential_radial_ring': (dbl, dbl, dbl, dbl, dbl, vp),
    'dz1_potential_radial_ring': (dbl, dbl, dbl, dbl, dbl, vp),
    'axial_derivatives_radial': (None, _arr(ndim=2), _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz, _arr(ndim=1), sz),
    'potential_radial': (dbl, v3, _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz),
    'potential_radial_derivs': (dbl, v3, _arr(ndim=1), _arr(ndim=3), sz),
    'flux_density_to_charge_factor': (dbl, dbl),
    'charge_radial': (dbl, _arr(ndim=2), dbl),
    'field_radial': (None, v3, v3, _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz),
    'field_radial_derivs': (None, v3, v3, _arr(ndim=1), _arr(ndim=3), sz),
    'current_potential_axial_radial_ring': (dbl, dbl, dbl, dbl),
    'current_potential_axial': (dbl, dbl, _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz),
    'current_field_radial_ring': (None, dbl, dbl, dbl, dbl, v2),
    'current_field_radial': (None, v3, v3, _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz),
    'current_axial_derivatives_radial': (None, _arr(ndim=2), _arr(ndim=1), _arr(ndim=2), _arr(ndim=3), sz,
                                         _arr(ndim=1), sz),
    'fill_jacobian_buffer_radial': (None, _arr(ndim=2), _arr(ndim=3), _arr(ndim=3), sz),
    'self_potential_radial': (dbl, dbl, vp),
    'self_field_dot_normal_radial': (dbl, dbl, vp),
    'fill_matrix_radial': (None, _arr(ndim=2), _arr(ndim=3), _arr(dtype=np.uint8, ndim=1), _arr(ndim=1),
                           _arr(ndim=2), _arr(ndim=3), sz, sz, C.c_int, C.c_int),
    'plane_intersection': (C.c_bool, v3, v3, _arr(ndim=2), sz, _arr(shape=(6,))),
    'tb_last_status': (C.c_int,),
}

for _name, (_res, *_args) in backend_functions.items():
    _f = getattr(backend_lib, _name)
    _f.restype = _res
    _f.argtypes = _args

_DEV = {
    'tb_jacobian_buffer_radial': (vp, vp, vp, i64, vp),
    'tb_mesh_segments': (vp, vp, i64, vp, i64, vp),
    'tb_element_targets': (vp, vp, vp, i64, vp),
    'tb_fill_matrix_radial': (vp, i64, vp, vp, vp, vp, vp, i64, i64, i64, C.c_int, C.c_int, vp),
    'tb_self_integrals': (vp, vp, vp, vp, vp, i64, i64, vp),
    'tb_rhs_radial': (vp, vp, vp, i64, vp),
    'tb_rhs_radial_field': (vp, vp, vp, vp, vp, i64, vp),
    'tb_lu_factor_perm': (vp, i64, vp, vp, i64, vp),
    'tb_lu_solve_perm': (vp, i64, vp, i64, vp, i64, vp, i64, i64, vp),
    'tb_pack_sources': (vp, vp, vp, vp, i64, vp),
    'tb_pack_current_sources': (vp, vp, vp, vp, i64, vp),
    'tb_field_radial_points': (vp, i64, vp, i64, vp, vp, vp),
    'tb_current_field_points': (vp, i64, vp, i64, vp, vp),
    'tb_axial_derivatives_radial': (vp, i64, vp, i64, vp, vp),
    'tb_current_axial_derivatives': (vp, i64, vp, i64, vp, vp),
    'tb_axial_coefficients': (vp, i64, dbl, vp, vp),
    'tb_axial_field_points': (vp, i64, vp, i64, vp, vp, vp, vp),
    'tb_trace_rk45': (vp, vp, vp, i64, C.POINTER(TbField), C.POINTER(TbTraceOpts), vp, vp, vp, vp, vp, vp, vp, vp),
    'tb_trace_rk45_geometries': (vp, vp, vp, vp, i64, C.POINTER(TbField), vp, i64, vp, C.POINTER(TbTraceOpts), vp, vp,
                                 vp, vp, vp, vp, vp, vp),
    'tb_batch_solve': (vp, C.c_int, vp, i64, vp, vp, i64, vp, i64, vp, C.c_int, vp),
    'tb_num_sms': (),
    'tb_lu_nopiv_f64': (vp, i64, i64, vp),
    'tb_lu_nopiv_f32': (vp, i64, i64, vp),
    'tb_lu_nopiv_f32_tc': (vp, i64, i64, vp, i64, vp, vp),
    'tb_fill_matrix_radial_batched': (vp, C.c_int, i64, vp),
    'tb_self_integrals_batched': (vp, C.c_int, i64, vp),
    'tb_gemm_sub_tf32x3': (vp, i64, vp, i64, vp, i64, i64, i64, i64, vp, i64, vp, vp),
    'tb_solve_mixed': (vp, i64, i64, vp, vp, i64, vp, i64, C.c_int, dbl, C.POINTER(C.c_int), C.POINTER(dbl), vp),
    'tb_plane_intersection_rows': (vp, vp, i64, i64, C.POINTER(dbl), C.POINTER(dbl), vp, vp, vp),
    'tb_focus_position': (vp, i64, i64, vp, vp, i64, vp),
}
for _name, _args in _DEV.items():
    _f = getattr(backend_lib, _name)
    _f.restype = C.c_int
    _f.argtypes = list(_args)
backend_lib.tb_batch_solve_plan.restype = i64
backend_lib.tb_batch_solve_plan.argtypes = [vp, C.c_int, vp, C.POINTER(i64)]
backend_lib.tb_set_solve_lookahead.restype = C.c_int
backend_lib.tb_set_solve_lookahead.argtypes = [C.c_int]
backend_lib.tb_set_wait_limit.restype = i64
backend_lib.tb_set_wait_limit.argtypes = [i64]


def set_solve_lookahead(reserve_sms):
    """SMs the mixed solve leaves to the next panel's factorisation while a
    second stream runs the rest of each trailing update (0: no lookahead, a
    negative value: the default, one SM in five); returns the previous value
    (tb_set_solve_lookahead)."""
    return int(backend_lib.tb_set_solve_lookahead(int(reserve_sms)))


def set_wait_limit(cycles):
    """Bound (SM clock cycles) of the progress waits inside the library's
    kernels, for launches made after the call; cycles <= 0 restores the
    default (about 1 s).  Returns the previous bound (tb_set_wait_limit)."""
    return int(backend_lib.tb_set_wait_limit(int(cycles)))


def _check_status():
    s = backend_lib.tb_last_status()
    if s != TB_OK:
        raise BackendError(f'traceon_b200 backend error status {s}')


# ====================================================================== scalars
ellipkm1 = np.vectorize(backend_lib.ellipkm1)
ellipk = np.vectorize(backend_lib.ellipk)
ellipem1 = np.vectorize(backend_lib.ellipem1)
ellipe = np.vectorize(backend_lib.ellipe)


def _v3(v):
    v = np.zeros(3) if v is None else np.asarray(v, dtype=np.float64)
    if v.shape == (2,):
        v = np.array([v[0], 0.0, v[1]])
    return np.ascontiguousarray(v)


def higher_order_normal_radial(alpha, vertices):
    """traceon/backend/__init__.py:373-377"""
    vertices = np.asarray(vertices, dtype=np.float64)
    assert vertices.shape == (4, 3)
    normal = np.zeros(2)
    backend_lib.higher_order_normal_radial(alpha, _v3(vertices[0]), _v3(vertices[2]), _v3(vertices[3]),
                                           _v3(vertices[1]), normal)
    assert np.isclose(np.linalg.norm(normal), 1.0)
    return normal


def normal_2d(p1, p2):
    normal = np.zeros(2)
    backend_lib.normal_2d(np.ascontiguousarray(p1, dtype=np.float64)[:2].copy(),
                          np.ascontiguousarray(p2, dtype=np.float64)[:2].copy(), normal)
    return normal


def position_and_jacobian_radial(alpha, v1, v2, v3, v4):
    """Returns (jac, pos) like traceon/backend/__init__.py:435-452; the four
    vertices are given in parametric order (alpha = -1, -1/3, 1/3, 1)."""
    pos = np.zeros(2)
    jac = C.c_double(0.0)
    backend_lib.position_and_jacobian_radial(alpha, _v3(v1), _v3(v2), _v3(v3), _v3(v4), pos, C.pointer(jac))
    return jac.value, pos


def delta_position_and_jacobian_radial(alpha, v1, v2, v3, v4):
    pos = np.zeros(2)
    jac = C.c_double(0.0)
    backend_lib.delta_position_and_jacobian_radial(alpha, _v3(v1), _v3(v2), _v3(v3), _v3(v4), pos, C.pointer(jac))
    return jac.value, pos


def potential_radial_ring(r0, z0, delta_r, delta_z):
    return backend_lib.potential_radial_ring(r0, z0, delta_r, delta_z, None)


def dr1_potential_radial_ring(r0, z0, delta_r, delta_z):
    return backend_lib.dr1_potential_radial_ring(r0, z0, delta_r, delta_z, None)


def dz1_potential_radial_ring(r0, z0, delta_r, delta_z):
    return backend_lib.dz1_potential_radial_ring(r0, z0, delta_r, delta_z, None)


def flux_density_to_charge_factor(K):
    return backend_lib.flux_density_to_charge_factor(K)


def charge_radial(vertices, charge):
    vertices = ensure_contiguous_aligned(np.asarray(vertices, dtype=np.float64))
    assert vertices.shape == (len(vertices), 3)
    return backend_lib.charge_radial(vertices, charge)


def current_potential_axial_radial_ring(z0, r, z):
    return backend_lib.current_potential_axial_radial_ring(z0, r, z)


def current_field_radial_ring(x0, y0, x, y):
    res = np.zeros(2)
    backend_lib.current_field_radial_ring(x0, y0, x, y, res)
    return res


def potential_radial_derivs(point, z, coeffs):
    assert coeffs.shape == (len(z) - 1, DERIV_2D_MAX, 6)
    return backend_lib.potential_radial_derivs(_v3(point), ensure_contiguous_aligned(z),
                                               ensure_contiguous_aligned(coeffs), len(z))


def field_radial_derivs(point, z, coeffs):
    assert coeffs.shape == (len(z) - 1, DERIV_2D_MAX, 6)
    field = np.zeros(3)
    backend_lib.field_radial_derivs(_v3(point), field, ensure_contiguous_aligned(z),
                                    ensure_contiguous_aligned(coeffs), len(z))
    return field


def plane_intersection(positions, p0, normal):
    """traceon/backend/__init__.py:763-773"""
    p0, normal = _v3(p0), _v3(normal)
    positions = ensure_contiguous_aligned(np.asarray(positions, dtype=np.float64))
    assert positions.shape == (len(positions), 6)
    result = np.zeros(6)
    found = backend_lib.plane_intersection(p0, normal, positions, len(positions), result)
    if not found:
        raise ValueError("Plane intersection not found. Does the trajectory actually cross the plane?")
    return result


# ====================================================================== arrays (GPU)
def _f64(a):
    return ensure_contiguous_aligned(np.asarray(a, dtype=np.float64))


def fill_jacobian_buffer_radial(vertices):
    vertices = _f64(vertices)
    assert vertices.shape == (len(vertices), 4, 3)
    assert np.all(vertices[:, :, 1] == 0.)
    N = len(vertices)
    jac = np.zeros((N, N_QUAD_2D))
    pos = np.zeros((N, N_QUAD_2D, 2))
    if N:
        backend_lib.fill_jacobian_buffer_radial(jac, pos, vertices, N)
        _check_status()
    return jac, pos


def fill_matrix_radial(matrix, lines, excitation_types, excitation_values, jac_buffer, pos_buffer, start_index,
                       end_index):
    """traceon/backend/__init__.py:712-730 (accumulates rows start..end)."""
    N = len(lines)
    assert np.all(lines[:, :, 1] == 0.0)
    assert matrix.shape == (N, N) and lines.shape == (N, 4, 3)
    assert excitation_types.shape == (N,) and excitation_values.shape == (N,)
    assert jac_buffer.shape == (N, N_QUAD_2D) and pos_buffer.shape == (N, N_QUAD_2D, 2)
    assert 0 <= start_index < N and 0 <= end_index < N and start_index <= end_index
    assert matrix.flags['C_CONTIGUOUS']
    backend_lib.fill_matrix_radial(matrix, _f64(lines), ensure_contiguous_aligned(excitation_types.astype(np.uint8)),
                                   _f64(excitation_values), _f64(jac_buffer), _f64(pos_buffer), N, matrix.shape[0],
                                   int(start_index), int(end_index))
    _check_status()


def potential_radial(point, charges, jac_buffer, pos_buffer):
    point = np.asarray(point)
    assert point.shape == (3,)
    assert jac_buffer.shape == (len(charges), N_QUAD_2D) and pos_buffer.shape == (len(charges), N_QUAD_2D, 2)
    r = backend_lib.potential_radial(_v3(point), _f64(charges), _f64(jac_buffer), _f64(pos_buffer), len(charges))
    _check_status()
    return r


def field_radial(point, charges, jac_buffer, pos_buffer):
    point = np.asarray(point)
    assert point.shape == (3,)
    assert jac_buffer.shape == (len(charges), N_QUAD_2D) and pos_buffer.shape == (len(charges), N_QUAD_2D, 2)
    field = np.zeros(3)
    backend_lib.field_radial(_v3(point), field, _f64(charges), _f64(jac_buffer), _f64(pos_buffer), len(charges))
    _check_status()
    return field


def axial_derivatives_radial(z, charges, jac_buffer, pos_buffer):
    z = _f64(z)
    derivs = np.zeros((z.size, DERIV_2D_MAX))
    assert jac_buffer.shape == (len(charges), N_QUAD_2D) and pos_buffer.shape == (len(charges), N_QUAD_2D, 2)
    if z.size:
        backend_lib.axial_derivatives_radial(derivs, _f64(charges), _f64(jac_buffer), _f64(pos_buffer), len(charges),
                                             z, len(z))
        _check_status()
    return derivs


def current_field_radial(p0, currents, jac_buffer, pos_buffer):
    N = len(currents)
    assert jac_buffer.shape == (N, N_TRIANGLE_QUAD) and pos_buffer.shape == (N, N_TRIANGLE_QUAD, 3)
    result = np.zeros(3)
    backend_lib.current_field_radial(_v3(p0), result, _f64(currents), _f64(jac_buffer), _f64(pos_buffer), N)
    _check_status()
    return result


def current_axial_derivatives_radial(z, currents, jac_buffer, pos_buffer):
    z = _f64(z)
    N = len(currents)
    derivs = np.zeros((z.size, DERIV_2D_MAX))
    if z.size:
        backend_lib.current_axial_derivatives_radial(derivs, _f64(currents), _f64(jac_buffer), _f64(pos_buffer), N,
                                                     z, len(z))
        _check_status()
    return derivs


def current_potential_axial(z, currents, jac_buffer, pos_buffer):
    N = len(currents)
    r = backend_lib.current_potential_axial(float(z), _f64(currents), _f64(jac_buffer), _f64(pos_buffer), N)
    _check_status()
    return r


def self_potential_radial(vertices):
    """Diagonal entry of a voltage row (reference :688-692), integrated on the GPU."""
    vertices = _f64(vertices)
    assert vertices.shape == (4, 3)
    return float(dev_self_integrals_np(vertices[None], np.array([1], np.uint8), np.zeros(1))[0])


def self_field_dot_normal_radial(vertices, K):
    """Self flux term of a dielectric / magnetizable row (reference :697-708),
    integrated on the GPU (without the -1 the solver adds)."""
    vertices = _f64(vertices)
    assert vertices.shape == (4, 3)
    return float(dev_self_integrals_np(vertices[None], np.array([3], np.uint8), np.array([float(K)]))[0]) + 1.0


def wrap_field_fun(ff):
    """Python field callbacks (reference :472-485) are accepted for API
    compatibility, but the GPU tracer cannot call them."""
    def field_fun_wrapper(pos, vel, _, elec_out, mag_out):
        elec, mag = ff(np.array([pos[0], pos[1], pos[2]]), np.array([vel[0], vel[1], vel[2]]))
        for i in range(3):
            elec_out[i] = elec[i]
            mag_out[i] = mag[i]
    return field_fun(field_fun_wrapper)


FIELD_RADIAL_TRACEABLE = C.cast(backend_lib.field_radial_traceable, C.c_void_p).value
FIELD_RADIAL_DERIVS_TRACEABLE = C.cast(backend_lib.field_radial_derivs_traceable, C.c_void_p).value


def trace_particle_wrapper(position_, velocity_, fill_positions_fun):
    """Block-continued tracing, traceon/backend/__init__.py:382-420."""
    position = np.array(position_)
    velocity = np.array(velocity_)
    assert position.shape == (3,) and velocity.shape == (3,)
    pos_blocks, times_blocks = [], []
    times = np.zeros(TRACING_BLOCK_SIZE)
    positions = np.zeros((TRACING_BLOCK_SIZE, 6))
    positions[0] = np.concatenate((position, velocity))
    while True:
        N = fill_positions_fun(times, positions)
        pos_blocks.append(positions[1:N] if len(pos_blocks) > 0 else positions[:N])
        times_blocks.append(times[1:N] if len(times_blocks) > 0 else times[:N])
        if N != TRACING_BLOCK_SIZE:
            break
        times = np.zeros(TRACING_BLOCK_SIZE)
        positions = np.zeros((TRACING_BLOCK_SIZE, 6))
        positions[0] = pos_blocks[-1][-1]
        times[0] = times_blocks[-1][-1]
    if len(pos_blocks) == 1:
        return times_blocks[0], pos_blocks[0]
    return np.concatenate(times_blocks), np.concatenate(pos_blocks)


def _field_address(field):
    if isinstance(field, int):
        return field
    return C.cast(field, C.c_void_p).value


def trace_particle(position, velocity, charge_over_mass, field, bounds, atol, args=None):
    """traceon/backend/__init__.py:487-497; integrated on the GPU."""
    bounds = ensure_contiguous_aligned(np.array(bounds, dtype=np.float64))
    addr = _field_address(field)
    if addr not in (FIELD_RADIAL_TRACEABLE, FIELD_RADIAL_DERIVS_TRACEABLE):
        raise NotImplementedError('the GPU tracer integrates only BEM and axial-interpolated fields of this '
                                  'library; Python field callbacks are not traced')

    def fill(T, P):
        n = backend_lib.trace_particle(T, P, charge_over_mass, addr, bounds, atol, args)
        _check_status()
        return n

    return trace_particle_wrapper(position, velocity, fill)


# ====================================================================== device API
def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream():
    torch = _torch()
    return torch.cuda.current_stream().cuda_stream


def _call(name, *args):
    r = getattr(backend_lib, name)(*args)
    if r != TB_OK:
        raise BackendError(f'{name} failed with status {r}')


def device():
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError('traceon_b200 needs a CUDA device (sm_100a); none is available')
    return torch.device('cuda', torch.cuda.current_device())


def to_dev(a, dtype=None):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.to(device=device())
        if dtype is not None:
            t = t.to(dtype)
        return t.contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device=device(), dtype=dtype).contiguous()


def dev_jacobian_buffer(vertices_t):
    torch = _torch()
    N = vertices_t.shape[0]
    jac = torch.empty((N, N_QUAD_2D), dtype=torch.float64, device=vertices_t.device)
    pos = torch.empty((N, N_QUAD_2D, 2), dtype=torch.float64, device=vertices_t.device)
    _call('tb_jacobian_buffer_radial', _ptr(vertices_t), _ptr(jac), _ptr(pos), N, _stream())
    return jac, pos


def dev_element_targets(vertices_t):
    torch = _torch()
    N = vertices_t.shape[0]
    tgt = torch.empty((N, 2), dtype=torch.float64, device=vertices_t.device)
    nrm = torch.empty((N, 2), dtype=torch.float64, device=vertices_t.device)
    _call('tb_element_targets', _ptr(vertices_t), _ptr(tgt), _ptr(nrm), N, _stream())
    return tgt, nrm


def dev_fill_matrix(A, vertices_t, types_t, values_t, jac, pos, row0=0, row1=None, accumulate=False,
                    gauss_diagonal=False):
    N = vertices_t.shape[0]
    row1 = N if row1 is None else row1
    _call('tb_fill_matrix_radial', _ptr(A), A.stride(0), _ptr(vertices_t), _ptr(types_t), _ptr(values_t), _ptr(jac),
          _ptr(pos), N, row0, row1, int(accumulate), int(gauss_diagonal), _stream())


def dev_self_integrals(vertices_t, types_t, values_t, A=None):
    torch = _torch()
    N = vertices_t.shape[0]
    diag = torch.empty(N, dtype=torch.float64, device=vertices_t.device)
    _call('tb_self_integrals', _ptr(vertices_t), _ptr(types_t), _ptr(values_t), _ptr(diag), _ptr(A),
          A.stride(0) if A is not None else N, N, _stream())
    return diag


backend_lib.tb_batch_plan.restype = i64
backend_lib.tb_batch_plan.argtypes = [vp, C.c_int, C.POINTER(i64)]


def dev_fill_batched(items):
    """Fills the matrices of many geometries (off-diagonal entries in one
    persistent launch, self terms in one more).  items: list of (vertices,
    types, values, jac, pos, A) device tensors, A (N, N) FP64."""
    torch = _torch()
    n = len(items)
    if n == 0:
        return
    arr = (TbGeometry * n)()
    for k, (v, t, val, jac, pos, A) in enumerate(items):
        arr[k] = TbGeometry(v.data_ptr(), t.data_ptr(), val.data_ptr(), jac.data_ptr(), pos.data_ptr(), A.data_ptr(),
                            A.stride(0), v.shape[0], 0, 0)
    total = i64(0)
    tiles = backend_lib.tb_batch_plan(arr, n, C.byref(total))
    if tiles < 0:
        raise BackendError('tb_batch_plan: bad geometry sizes')
    dev = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(items[0][0].device)
    _call('tb_fill_matrix_radial_batched', _ptr(dev), n, tiles, _stream())
    _call('tb_self_integrals_batched', _ptr(dev), n, total.value, _stream())


def dev_self_integrals_np(vertices, types, values):
    torch = _torch()
    d = dev_self_integrals(to_dev(vertices, torch.float64), to_dev(types, torch.uint8), to_dev(values, torch.float64))
    return d.cpu().numpy()


def dev_lu_factor(A):
    """In-place FP64 LU with partial pivoting; returns (ipiv, perm)."""
    torch = _torch()
    N = A.shape[0]
    ipiv = torch.empty(N, dtype=torch.int32, device=A.device)
    perm = torch.empty(N, dtype=torch.int32, device=A.device)
    _call('tb_lu_factor_perm', _ptr(A), A.stride(0), _ptr(ipiv), _ptr(perm), N, _stream())
    return ipiv, perm


def dev_lu_solve(LU, perm, F):
    """Solves A x = f for each row f of F (nrhs, N)."""
    torch = _torch()
    N = LU.shape[0]
    F = F.reshape(-1, N).clone(memory_format=torch.contiguous_format)
    X = torch.empty((F.shape[0], N), dtype=torch.float64, device=F.device)
    # a (1, N) tensor may report stride 0 for its size-1 dimension
    _call('tb_lu_solve_perm', _ptr(LU), LU.stride(0), _ptr(perm), N, _ptr(F), N, _ptr(X), N, F.shape[0], _stream())
    return X


backend_lib.tb_focus_position_workspace.restype = i64
backend_lib.tb_focus_position_workspace.argtypes = []


def dev_plane_intersection_rows(rows, nrows, p0, normal):
    """Plane crossing nearest the end of each stored trajectory (rows
    (n, max_rows, 7), nrows (n) as written by the tracer), linear
    interpolation as traceon/backend/tracing.c:184-223.  Returns device
    tensors (out (n, 7) t, x..vz, NaN where none; found (n) bool)."""
    torch = _torch()
    n, max_rows = rows.shape[0], rows.shape[1]
    assert rows.shape[2:] == (7,) and rows.dtype == torch.float64 and rows.is_contiguous()
    assert nrows.shape == (n,) and nrows.dtype == torch.int64
    out = torch.empty((n, 7), dtype=torch.float64, device=rows.device)
    found = torch.empty(n, dtype=torch.int32, device=rows.device)
    a = (dbl * 3)(*[float(v) for v in np.asarray(p0, dtype=np.float64).reshape(3)])
    b = (dbl * 3)(*[float(v) for v in np.asarray(normal, dtype=np.float64).reshape(3)])
    _call('tb_plane_intersection_rows', _ptr(rows), _ptr(nrows), n, max_rows, a, b, _ptr(out), _ptr(found), _stream())
    return out, found.bool()


def dev_focus_position(states):
    """Least-squares beam focus (traceon/focus.py:9-42) from final states on
    the device: states (n, 6) x..vz, or (n, 7) t, x..vz.  Returns a device
    tensor (3,) = (x, y, z); NaN when rank deficient."""
    torch = _torch()
    assert states.dim() == 2 and states.shape[1] in (6, 7) and states.dtype == torch.float64
    states = states.contiguous()
    off = states.shape[1] - 6
    out = torch.empty(3, dtype=torch.float64, device=states.device)
    nbytes = backend_lib.tb_focus_position_workspace()
    work = torch.empty(nbytes, dtype=torch.uint8, device=states.device)
    _call('tb_focus_position', states.data_ptr() + 8 * off, states.shape[0], states.stride(0), _ptr(out), _ptr(work),
          nbytes, _stream())
    return out


backend_lib.tb_solve_mixed_workspace.restype = i64
backend_lib.tb_solve_mixed_workspace.argtypes = [i64, i64]


def dev_lu_nopiv(A):
    """In-place LU without pivoting of a square FP64 or FP32 device matrix."""
    torch = _torch()
    name = 'tb_lu_nopiv_f64' if A.dtype == torch.float64 else 'tb_lu_nopiv_f32'
    _call(name, _ptr(A), A.stride(0), A.shape[0], _stream())


backend_lib.tb_lu_nopiv_f32_tc_workspace.restype = i64
backend_lib.tb_lu_nopiv_f32_tc_workspace.argtypes = [i64]
backend_lib.tb_gemm_tf32x3_workspace.restype = i64
backend_lib.tb_gemm_tf32x3_workspace.argtypes = [i64, i64, i64]


def dev_lu_nopiv_tc(A):
    """In-place FP32 LU without pivoting of a square FP32 device matrix:
    256-column panels, trailing updates on the tensor cores (3xTF32)."""
    torch = _torch()
    N = A.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    nbytes = backend_lib.tb_lu_nopiv_f32_tc_workspace(N)
    work = torch.empty(nbytes, dtype=torch.uint8, device=A.device) if nbytes else None
    _call('tb_lu_nopiv_f32_tc', _ptr(A), A.stride(0), N, _ptr(work), nbytes, _ptr(err), _stream())
    if int(err.item()):
        raise BackendError('tb_lu_nopiv_f32_tc: a bounded wait in a tensor-core kernel ran out')


def dev_gemm_sub_tf32x3(C, A, B, presplit=False):
    """C -= A @ B (FP32 device matrices, unit column stride) on the tensor
    cores with 3xTF32; presplit: the bulk-copy GEMM on pre-split operands."""
    torch = _torch()
    M, K = A.shape
    N = B.shape[1]
    err = torch.zeros(1, dtype=torch.int32, device=C.device)
    nbytes = backend_lib.tb_gemm_tf32x3_workspace(M, N, K) if presplit else 0
    work = torch.empty(nbytes, dtype=torch.uint8, device=C.device) if nbytes else None
    _call('tb_gemm_sub_tf32x3', _ptr(C), C.stride(0), _ptr(A), A.stride(0), _ptr(B), B.stride(0), M, N, K, _ptr(work),
          nbytes, _ptr(err), _stream())
    if int(err.item()):
        raise BackendError('tb_gemm_sub_tf32x3: a bounded wait in the tensor-core kernel ran out')


def dev_solve_mixed(A, F, max_iter=12, tol=1e-12):
    """Mixed-precision solve (FP32 factors, FP64 refinement) of A x = f for
    each row f of F (nrhs <= 16).  Returns (X, iterations, last relative
    correction); raises BackendError(status) when refinement fails."""
    torch = _torch()
    N = A.shape[0]
    F = F.reshape(-1, N).contiguous()
    nrhs = F.shape[0]
    X = torch.empty((nrhs, N), dtype=torch.float64, device=A.device)
    nbytes = backend_lib.tb_solve_mixed_workspace(N, nrhs)
    work = torch.empty(nbytes, dtype=torch.uint8, device=A.device)
    it = C.c_int(0)
    rel = dbl(0.0)
    r = backend_lib.tb_solve_mixed(_ptr(A), A.stride(0), N, _ptr(F), _ptr(X), nrhs, _ptr(work), nbytes, max_iter, tol,
                                   C.byref(it), C.byref(rel), _stream())
    if r != TB_OK:
        err = BackendError(f'tb_solve_mixed failed with status {r}')
        err.status = r
        raise err
    return X, it.value, rel.value


def dev_pack_sources(charges_t, jac_t, pos_t):
    torch = _torch()
    N = charges_t.shape[0]
    src = torch.empty((3, N * N_QUAD_2D), dtype=torch.float64, device=charges_t.device)
    if N:
        _call('tb_pack_sources', _ptr(charges_t), _ptr(jac_t), _ptr(pos_t), _ptr(src), N, _stream())
    return src


def dev_pack_current_sources(currents_t, jac_t, pos_t):
    torch = _torch()
    N = currents_t.shape[0]
    src = torch.empty((3, N * N_TRIANGLE_QUAD), dtype=torch.float64, device=currents_t.device)
    if N:
        _call('tb_pack_current_sources', _ptr(currents_t), _ptr(jac_t), _ptr(pos_t), _ptr(src), N, _stream())
    return src


def dev_field_points(points_t, sources_t, want_pot=True, want_field=True):
    torch = _torch()
    M = points_t.shape[0]
    pot = torch.empty(M, dtype=torch.float64, device=points_t.device) if want_pot else None
    field = torch.empty((M, 3), dtype=torch.float64, device=points_t.device) if want_field else None
    if M:
        _call('tb_field_radial_points', _ptr(points_t), M, _ptr(sources_t), sources_t.shape[1], _ptr(pot),
              _ptr(field), _stream())
    return pot, field


def dev_current_field_points(points_t, sources_t):
    torch = _torch()
    M = points_t.shape[0]
    field = torch.empty((M, 3), dtype=torch.float64, device=points_t.device)
    if M:
        _call('tb_current_field_points', _ptr(points_t), M, _ptr(sources_t), sources_t.shape[1], _ptr(field),
              _stream())
    return field


def dev_axial_derivatives(z_t, sources_t, current=False):
    torch = _torch()
    Nz = z_t.shape[0]
    d = torch.empty((Nz, DERIV_2D_MAX), dtype=torch.float64, device=z_t.device)
    if Nz:
        name = 'tb_current_axial_derivatives' if current else 'tb_axial_derivatives_radial'
        _call(name, _ptr(z_t), Nz, _ptr(sources_t), sources_t.shape[1], _ptr(d), _stream())
    return d


def dev_axial_coefficients(derivs_t, dz):
    torch = _torch()
    Nz = derivs_t.shape[0]
    c = torch.empty((Nz - 1, DERIV_2D_MAX, 6), dtype=torch.float64, device=derivs_t.device)
    _call('tb_axial_coefficients', _ptr(derivs_t), Nz, float(dz), _ptr(c), _stream())
    return c


def dev_axial_field_points(points_t, z_t, coeffs_t, want_pot=True, want_field=True):
    torch = _torch()
    M = points_t.shape[0]
    pot = torch.empty(M, dtype=torch.float64, device=points_t.device) if want_pot else None
    field = torch.empty((M, 3), dtype=torch.float64, device=points_t.device) if want_field else None
    if M:
        _call('tb_axial_field_points', _ptr(points_t), M, _ptr(z_t), z_t.shape[0], _ptr(coeffs_t), _ptr(pot),
              _ptr(field), _stream())
    return pot, field


def num_sms():
    return backend_lib.tb_num_sms()
