"""CPU oracle for the Traceon radial BEM path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU
baseline and reference arms) may import this module.  It is the test oracle
of the CUDA library, never a fallback for it.

Two CPU implementations are exposed through one interface:

* ``Oracle('port')`` -- ``oracle/liboracle.so``, this repository's C
  restatement of the reference backend (``oracle/traceon_oracle.c``);
* ``Oracle('ref')``  -- ``oracle/_ref/libtraceon_ref.so``, the reference C
  backend compiled from its own sources by ``oracle/Makefile``.

The parts of the reference path that run in third-party Python libraries are
restated here with the same libraries the reference calls:

* the singular diagonal: SciPy QUADPACK ``quad(..., -1, 1, points=(0,),
  epsabs=1e-9, epsrel=1e-9, limit=250)`` over the C self-integrand
  (traceon/backend/__init__.py:688-708, traceon/solver.py:239-247);
* the dense solve: ``numpy.linalg.solve`` (LAPACK dgesv, traceon/solver.py:173);
* the axial interpolation coefficients: SciPy ``BPoly.from_derivatives`` /
  ``PPoly.from_bernstein_basis`` / ``CubicSpline`` (traceon/field.py:906-937).
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, 'liboracle.so')
REF_LIB = os.path.join(HERE, '_ref', 'libtraceon_ref.so')
REF_STRICT_LIB = os.path.join(HERE, '_ref', 'libtraceon_ref_strict.so')

N_QUAD_2D = 16
N_TRIANGLE_QUAD = 12
DERIV_2D_MAX = 9
TRACING_BLOCK_SIZE = 100000
EM = -175882001077.2163  # q/m of the electron, definitions.c:29

dbl = C.c_double
dp = C.POINTER(C.c_double)
sz = C.c_size_t


def _p(a):
    return a.ctypes.data_as(dp)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class _Charges2D(C.Structure):
    """struct effective_point_charges_2d, traceon/backend/radial.c:10-15"""
    _fields_ = [('charges', dp), ('jacobians', dp), ('positions', dp), ('N', sz)]


class _FieldArgs(C.Structure):
    """struct field_evaluation_args, traceon/backend/radial.c:175-180"""
    _fields_ = [('elec', C.c_void_p), ('mag', C.c_void_p), ('current', C.c_void_p), ('bounds', dp)]


class _OrBemArgs(C.Structure):
    """struct or_bem_args of oracle/traceon_oracle.c"""
    _fields_ = [('eq', dp), ('ejac', dp), ('epos', dp), ('eN', sz),
                ('mq', dp), ('mjac', dp), ('mpos', dp), ('mN', sz),
                ('cI', dp), ('cjac', dp), ('cpos', dp), ('cN', sz),
                ('bounds', dp)]


class _OrAxialArgs(C.Structure):
    _fields_ = [('z', dp), ('ecoeff', dp), ('mcoeff', dp), ('Nz', sz)]


class _SelfFluxArgs(C.Structure):
    _fields_ = [('line_points', dp), ('K', dbl)]


def available(kind: str) -> bool:
    return os.path.isfile({'port': PORT_LIB, 'ref': REF_LIB, 'ref_strict': REF_STRICT_LIB}[kind])


class Oracle:
    """FP64 CPU implementation of the radial path (see module docstring)."""

    def __init__(self, kind: str = 'port'):
        self.kind = kind
        path = {'port': PORT_LIB, 'ref': REF_LIB, 'ref_strict': REF_STRICT_LIB}[kind]
        if not os.path.isfile(path):
            raise FileNotFoundError(f'{path} is not built (run make -C oracle)')
        self.lib = C.CDLL(path)
        self.is_port = kind == 'port'
        pre = 'or_' if self.is_port else ''
        self._pre = pre
        L = self.lib

        def fn(name, res, *args):
            f = getattr(L, pre + name)
            f.restype = res
            f.argtypes = list(args)
            return f

        self.f_ellipkm1 = fn('ellipkm1', dbl, dbl)
        self.f_ellipem1 = fn('ellipem1', dbl, dbl)
        self.f_ellipk = fn('ellipk', dbl, dbl)
        self.f_ellipe = fn('ellipe', dbl, dbl)
        if self.is_port:
            self.f_pot_ring = fn('potential_radial_ring', dbl, dbl, dbl, dbl, dbl)
            self.f_dr1_ring = fn('dr1_potential_radial_ring', dbl, dbl, dbl, dbl, dbl)
            self.f_dz1_ring = fn('dz1_potential_radial_ring', dbl, dbl, dbl, dbl, dbl)
        else:
            self.f_pot_ring = fn('potential_radial_ring', dbl, dbl, dbl, dbl, dbl, C.c_void_p)
            self.f_dr1_ring = fn('dr1_potential_radial_ring', dbl, dbl, dbl, dbl, dbl, C.c_void_p)
            self.f_dz1_ring = fn('dz1_potential_radial_ring', dbl, dbl, dbl, dbl, dbl, C.c_void_p)
        self.f_jacbuf = fn('fill_jacobian_buffer_radial', None, dp, dp, dp, sz)
        if self.is_port:
            self.f_fill = fn('fill_matrix_radial', C.c_int, dp, dp, C.POINTER(C.c_uint8), dp, dp, dp, sz, sz,
                             C.c_int, C.c_int)
        else:
            self.f_fill = fn('fill_matrix_radial', None, dp, dp, C.POINTER(C.c_uint8), dp, dp, dp, sz, sz,
                             C.c_int, C.c_int)
        self.f_pot = fn('potential_radial', dbl, dp, dp, dp, dp, sz)
        self.f_field = fn('field_radial', None, dp, dp, dp, dp, dp, sz)
        self.f_axial = fn('axial_derivatives_radial', None, dp, dp, dp, dp, sz, dp, sz)
        self.f_cur_field = fn('current_field_radial', None, dp, dp, dp, dp, dp, sz)
        self.f_cur_axial = fn('current_axial_derivatives_radial', None, dp, dp, dp, dp, sz, dp, sz)
        self.f_pot_derivs = fn('potential_radial_derivs', dbl, dp, dp, dp, sz)
        self.f_field_derivs = fn('field_radial_derivs', None, dp, dp, dp, dp, sz)
        self.f_normal = None
        if self.is_port:
            self.f_normal = fn('higher_order_normal_radial', None, dbl, dp, dp)
            self.f_charge = fn('charge_radial', dbl, dp, dbl)
            self.f_plane = fn('plane_intersection', C.c_int, dp, dp, dp, sz, dp)
            self.f_trace_bem = fn('trace_particle_bem', sz, dp, dp, dbl, C.POINTER(_OrBemArgs), dp, dbl, sz,
                                  C.c_longlong)
            self.f_trace_axial = fn('trace_particle_axial', sz, dp, dp, dbl, C.POINTER(_OrAxialArgs), dp, dbl,
                                    sz, C.c_longlong)
            self.f_field_batch = fn('field_radial_batch', None, dp, dp, sz, dp, dp, dp, sz)
            self.f_pot_batch = fn('potential_radial_batch', None, dp, dp, sz, dp, dp, dp, sz)
        else:
            self.f_normal = fn('higher_order_normal_radial', None, dbl, dp, dp, dp, dp, dp)
            self.f_charge = fn('charge_radial', dbl, dp, dbl)
            self.f_plane = fn('plane_intersection', C.c_bool, dp, dp, dp, sz, dp)
            self.f_trace = fn('trace_particle', sz, dp, dp, dbl, C.c_void_p, dp, dbl, C.c_void_p)
            self.addr_field_radial_traceable = C.cast(L.field_radial_traceable, C.c_void_p).value
            self.addr_field_radial_derivs_traceable = C.cast(L.field_radial_derivs_traceable, C.c_void_p).value
        self.addr_self_pot = C.cast(getattr(L, pre + 'self_potential_radial'), C.c_void_p).value
        self.addr_self_flux = C.cast(getattr(L, pre + 'self_field_dot_normal_radial'), C.c_void_p).value

    # ------------------------------------------------------------ scalars
    def ellipkm1(self, p):
        return np.vectorize(self.f_ellipkm1)(p)

    def ellipem1(self, p):
        return np.vectorize(self.f_ellipem1)(p)

    def ellipk(self, k):
        return np.vectorize(self.f_ellipk)(k)

    def ellipe(self, k):
        return np.vectorize(self.f_ellipe)(k)

    def potential_radial_ring(self, r0, z0, dr, dz):
        if self.is_port:
            return self.f_pot_ring(r0, z0, dr, dz)
        return self.f_pot_ring(r0, z0, dr, dz, None)

    def dr1_potential_radial_ring(self, r0, z0, dr, dz):
        if self.is_port:
            return self.f_dr1_ring(r0, z0, dr, dz)
        return self.f_dr1_ring(r0, z0, dr, dz, None)

    def dz1_potential_radial_ring(self, r0, z0, dr, dz):
        if self.is_port:
            return self.f_dz1_ring(r0, z0, dr, dz)
        return self.f_dz1_ring(r0, z0, dr, dz, None)

    def higher_order_normal_radial(self, alpha, vertices):
        v = _c(vertices)
        out = np.zeros(2)
        if self.is_port:
            self.f_normal(alpha, _p(v), _p(out))
        else:
            rows = [_c(v[i]) for i in (0, 2, 3, 1)]
            self.f_normal(alpha, *[_p(r) for r in rows], _p(out))
        return out

    def charge_radial(self, vertices, charge):
        v = _c(vertices)
        return self.f_charge(_p(v), charge)

    # ------------------------------------------------------------ buffers
    def fill_jacobian_buffer_radial(self, vertices):
        v = _c(vertices)
        N = len(v)
        jac = np.zeros((N, N_QUAD_2D))
        pos = np.zeros((N, N_QUAD_2D, 2))
        self.f_jacbuf(_p(jac), _p(pos), _p(v), N)
        return jac, pos

    def fill_matrix_radial(self, vertices, types, values, jac, pos, start=0, end=None, matrix=None):
        v = _c(vertices)
        N = len(v)
        end = N - 1 if end is None else end
        types = _c(types, np.uint8)
        values = _c(values)
        jac, pos = _c(jac), _c(pos)
        if matrix is None:
            matrix = np.zeros((N, N))
        r = self.f_fill(_p(matrix), _p(v), types.ctypes.data_as(C.POINTER(C.c_uint8)), _p(values), _p(jac),
                        _p(pos), N, matrix.shape[0], start, end)
        if self.is_port and r != 0:
            raise ValueError('unknown excitation type')
        return matrix

    def fill_matrix_threaded(self, vertices, types, values, jac, pos, threads=None):
        """Row-split fill over Python threads, as traceon/solver.py:226-236 does."""
        N = len(vertices)
        matrix = np.zeros((N, N))
        threads = threads or os.cpu_count() or 1
        chunks = [c for c in np.array_split(np.arange(N), threads) if len(c)]
        v, t, val, j, p = _c(vertices), _c(types, np.uint8), _c(values), _c(jac), _c(pos)

        def work(rows):
            self.fill_matrix_radial(v, t, val, j, p, int(rows[0]), int(rows[-1]), matrix=matrix)

        ts = [threading.Thread(target=work, args=(c,)) for c in chunks]
        for th in ts:
            th.start()
        for th in ts:
            th.join()
        return matrix

    @staticmethod
    def _quad(ll, shipped):
        from scipy.integrate import quad
        if shipped:
            # the reference's call, traceon/backend/__init__.py:692,708
            return quad(ll, -1, 1, points=(0,), epsabs=1e-9, epsrel=1e-9, limit=250)[0]
        # The same integral converged to ~1e-15: on mm-scale elements
        # (entries ~1e-5) the shipped epsabs = 1e-9 lets QUADPACK stop early
        # on some elements, by up to ~1e-5 relative depending on rounding.
        return sum(quad(ll, a, b, epsabs=1e-300, epsrel=1e-13, limit=500)[0] for a, b in ((-1, 0), (0, 1)))

    def self_potential_radial(self, vertices, shipped=False):
        """Diagonal entry of a voltage row: QUADPACK over the log-singular self
        integrand (radial.c:182-196), traceon/backend/__init__.py:688-692."""
        from scipy import LowLevelCallable
        v = _c(vertices)
        cb = C.CFUNCTYPE(dbl, dbl, C.c_void_p)(self.addr_self_pot)
        ll = LowLevelCallable(cb, user_data=v.ctypes.data_as(C.c_void_p))
        return self._quad(ll, shipped)

    def self_field_dot_normal_radial(self, vertices, K, shipped=False):
        """Diagonal term of a dielectric / magnetizable row before the -1
        (radial.c:203-222), traceon/backend/__init__.py:697-708."""
        from scipy import LowLevelCallable
        v = _c(vertices)
        args = _SelfFluxArgs()
        args.K = float(K)
        args.line_points = _p(v)
        cb = C.CFUNCTYPE(dbl, dbl, C.c_void_p)(self.addr_self_flux)
        ll = LowLevelCallable(cb, user_data=C.cast(C.pointer(args), C.c_void_p))
        return self._quad(ll, shipped)

    def diagonal(self, vertices, types, values, shipped=False):
        """Diagonal as traceon/solver.py:239-247 writes it."""
        d = np.zeros(len(vertices))
        for i, (v, t, val) in enumerate(zip(vertices, types, values)):
            if int(t) in (3, 6):
                d[i] = self.self_field_dot_normal_radial(v, val, shipped) - 1
            else:
                d[i] = self.self_potential_radial(v, shipped)
        return d

    def matrix(self, vertices, types, values, threads=None, shipped=False):
        """Full BEM matrix: threaded fill, then the QUADPACK diagonal."""
        jac, pos = self.fill_jacobian_buffer_radial(vertices)
        A = self.fill_matrix_threaded(vertices, types, values, jac, pos, threads)
        A[np.diag_indices(len(A))] = self.diagonal(vertices, types, values, shipped)
        return A

    # ------------------------------------------------------------ fields
    def potential_radial(self, point, q, jac, pos):
        pt = _c(point)
        q, jac, pos = _c(q), _c(jac), _c(pos)
        return self.f_pot(_p(pt), _p(q), _p(jac), _p(pos), len(q))

    def field_radial(self, point, q, jac, pos):
        pt = _c(point)
        q, jac, pos = _c(q), _c(jac), _c(pos)
        out = np.zeros(3)
        self.f_field(_p(pt), _p(out), _p(q), _p(jac), _p(pos), len(q))
        return out

    def _batched(self, points, fun, threads):
        points = _c(points).reshape(-1, 3)
        threads = threads or os.cpu_count() or 1
        with ThreadPoolExecutor(threads) as ex:
            return list(ex.map(fun, points))

    def field_radial_many(self, points, q, jac, pos, threads=None):
        q, jac, pos = _c(q), _c(jac), _c(pos)
        return np.array(self._batched(points, lambda p: self.field_radial(p, q, jac, pos), threads))

    def potential_radial_many(self, points, q, jac, pos, threads=None):
        q, jac, pos = _c(q), _c(jac), _c(pos)
        return np.array(self._batched(points, lambda p: self.potential_radial(p, q, jac, pos), threads))

    def axial_derivatives_radial(self, z, q, jac, pos):
        z, q, jac, pos = _c(z), _c(q), _c(jac), _c(pos)
        d = np.zeros((len(z), DERIV_2D_MAX))
        self.f_axial(_p(d), _p(q), _p(jac), _p(pos), len(q), _p(z), len(z))
        return d

    def current_field_radial(self, point, I, jac, pos):
        pt, I, jac, pos = _c(point), _c(I), _c(jac), _c(pos)
        out = np.zeros(3)
        self.f_cur_field(_p(pt), _p(out), _p(I), _p(jac), _p(pos), len(I))
        return out

    def current_axial_derivatives_radial(self, z, I, jac, pos):
        z, I, jac, pos = _c(z), _c(I), _c(jac), _c(pos)
        d = np.zeros((len(z), DERIV_2D_MAX))
        self.f_cur_axial(_p(d), _p(I), _p(jac), _p(pos), len(I), _p(z), len(z))
        return d

    def potential_radial_derivs(self, point, z, coeffs):
        pt, z, c = _c(point), _c(z), _c(coeffs)
        return self.f_pot_derivs(_p(pt), _p(z), _p(c), len(z))

    def field_radial_derivs(self, point, z, coeffs):
        pt, z, c = _c(point), _c(z), _c(coeffs)
        out = np.zeros(3)
        self.f_field_derivs(_p(pt), _p(out), _p(z), _p(c), len(z))
        return out

    # ------------------------------------------------------------ tracing
    def trace_bem(self, p0, v0, qm, q, jac, pos, bounds, atol, field_bounds=None, max_attempts=0, mag=None,
                  current=None):
        """One trajectory through a BEM field, returns (times, (n,6) states):
        electrostatic charges (q, jac, pos), and optionally magnetostatic
        charges mag = (q, jac (N,16), pos (N,16,2)) and current rings
        current = (I, jac (N,12), pos (N,12,3)) -- the Lorentz force of
        tracing.c:141-163.  Port: or_trace_particle_bem; ref: the reference
        trace_particle with its field_radial_traceable callback."""
        q, jac, pos = _c(q), _c(jac), _c(pos)
        bounds = _c(bounds).reshape(3, 2)
        times = np.zeros(TRACING_BLOCK_SIZE)
        states = np.zeros((TRACING_BLOCK_SIZE, 6))
        states[0, :3] = p0
        states[0, 3:] = v0
        mg = (np.zeros(0), np.zeros((0, N_QUAD_2D)), np.zeros((0, N_QUAD_2D, 2))) if mag is None else \
            tuple(_c(a) for a in mag)
        cu = (np.zeros(0), np.zeros((0, N_TRIANGLE_QUAD)), np.zeros((0, N_TRIANGLE_QUAD, 3))) if current is None \
            else tuple(_c(a) for a in current)
        fb = None if field_bounds is None else _c(field_bounds).reshape(3, 2)
        if self.is_port:
            a = _OrBemArgs(_p(q), _p(jac), _p(pos), len(q),
                           _p(mg[0]), _p(mg[1]), _p(mg[2]), len(mg[0]),
                           _p(cu[0]), _p(cu[1]), _p(cu[2]), len(cu[0]),
                           _p(fb) if fb is not None else None)
            n = self.f_trace_bem(_p(times), _p(states), qm, C.byref(a), _p(bounds), atol, TRACING_BLOCK_SIZE,
                                 max_attempts)
        else:
            e = _Charges2D(_p(q), _p(jac), _p(pos), len(q))
            m = _Charges2D(_p(mg[0]), _p(mg[1]), _p(mg[2]), len(mg[0]))
            c = _Charges2D(_p(cu[0]), _p(cu[1]), _p(cu[2]), len(cu[0]))
            a = _FieldArgs(C.cast(C.pointer(e), C.c_void_p), C.cast(C.pointer(m), C.c_void_p),
                           C.cast(C.pointer(c), C.c_void_p), _p(fb) if fb is not None else None)
            n = self.f_trace(_p(times), _p(states), qm, self.addr_field_radial_traceable, _p(bounds), atol,
                             C.cast(C.pointer(a), C.c_void_p))
        return times[:n].copy(), states[:n].copy()

    def trace_axial(self, p0, v0, qm, z, ecoeffs, mcoeffs, bounds, atol, max_attempts=0):
        """One trajectory through an axial-interpolated field."""
        z, ec, mc = _c(z), _c(ecoeffs), _c(mcoeffs)
        bounds = _c(bounds).reshape(3, 2)
        times = np.zeros(TRACING_BLOCK_SIZE)
        states = np.zeros((TRACING_BLOCK_SIZE, 6))
        states[0, :3] = p0
        states[0, 3:] = v0
        if self.is_port:
            a = _OrAxialArgs(_p(z), _p(ec), _p(mc), len(z))
            n = self.f_trace_axial(_p(times), _p(states), qm, C.byref(a), _p(bounds), atol, TRACING_BLOCK_SIZE,
                                   max_attempts)
        else:
            class _Derivs(C.Structure):
                _fields_ = [('z', dp), ('e', dp), ('m', dp), ('N', sz)]
            a = _Derivs(_p(z), _p(ec), _p(mc), len(z))
            n = self.f_trace(_p(times), _p(states), qm, self.addr_field_radial_derivs_traceable, _p(bounds), atol,
                             C.cast(C.pointer(a), C.c_void_p))
        return times[:n].copy(), states[:n].copy()

    def plane_intersection(self, states, p0, normal):
        s, p0, n = _c(states), _c(p0), _c(normal)
        out = np.zeros(6)
        ok = self.f_plane(_p(p0), _p(n), _p(s), len(s), _p(out))
        if not ok:
            raise ValueError('no plane crossing')
        return out


# -------------------------------------------------------------- helpers
def solve(A, F):
    """traceon/solver.py:173: charges = np.linalg.solve(A, F.T).T"""
    return np.linalg.solve(A, np.atleast_2d(F).T).T


def axial_coefficients(z, derivs):
    """_quintic_spline_coefficients, traceon/field.py:914-937, with the same
    SciPy calls: a quintic Hermite through (d_i, d_{i+1}, d_{i+2}) for i <= 6
    and a not-a-knot cubic spline for i = 7, 8.  derivs is (N_z, 9)."""
    from scipy.interpolate import BPoly, PPoly, CubicSpline
    z = np.asarray(z, dtype=np.float64)
    d = np.asarray(derivs, dtype=np.float64).T
    c = np.zeros((z.size - 1, 9, 6))
    for i in range(len(d)):
        if i + 2 < len(d):
            bp = BPoly.from_derivatives(z, np.array([d[i], d[i + 1], d[i + 2]]).T)
            pp = PPoly.from_bernstein_basis(bp)
            c[:, i, 0:] = pp.c.T
        else:
            pp = CubicSpline(z, d[i])
            c[:, i, 2:] = pp.c.T
    return c


def focus_position(positions):
    """traceon/focus.py:9-42, the same least-squares system solved by the
    same numpy.linalg.lstsq call: positions is a list of (N, 6)
    trajectories; returns (x, y, z)."""
    angles_x = np.array([p[-1, 3] / p[-1, 5] for p in positions])
    angles_y = np.array([p[-1, 4] / p[-1, 5] for p in positions])
    x, y, z = [np.array([p[-1, i] for p in positions]) for i in (0, 1, 2)]
    n = len(positions)
    a = np.array([np.concatenate((-angles_x, -angles_y)), np.concatenate((np.ones(n), np.zeros(n))),
                  np.concatenate((np.zeros(n), np.ones(n)))]).T
    rhs = np.concatenate((x - z * angles_x, y - z * angles_y))
    zf, xf, yf = np.linalg.lstsq(a, rhs, rcond=None)[0]
    return np.array([xf, yf, zf])


def hermite_plane_crossing(times, states, z_plane):
    """Crossing of the plane z = z_plane by cubic Hermite interpolation of
    position between the two accepted states that bracket it (position and
    velocity at both ends); searched from the end like tracing.c:184-223.
    Returns (x, y, z, vx, vy, vz) with the velocity linearly interpolated, or
    None when the trajectory does not cross."""
    z = states[:, 2] - z_plane
    for i in range(len(states) - 2, -1, -1):
        if (z[i] > 0) != (z[i + 1] > 0):
            return _hermite_root(times[i + 1] - times[i], states[i], states[i + 1], z_plane)
    return None


def hermite_position_at(times, states, t):
    """Position (x, y, z) of a stored trajectory at time t: cubic Hermite
    interpolation of position between the two accepted states that bracket t
    (positions and velocities at both ends); beyond the last state, the last
    interval's polynomial is extended.  Test infrastructure (endpoint checks
    at equal times)."""
    times = np.asarray(times)
    n = len(times)
    i = int(np.searchsorted(times, t, side='right')) - 1
    i = min(max(i, 0), n - 2)
    h = times[i + 1] - times[i]
    s0, s1 = states[i], states[i + 1]
    u = (t - times[i]) / h
    h00 = 2 * u**3 - 3 * u**2 + 1
    h10 = u**3 - 2 * u**2 + u
    h01 = -2 * u**3 + 3 * u**2
    h11 = u**3 - u**2
    return np.array([h00 * s0[c] + h10 * h * s0[3 + c] + h01 * s1[c] + h11 * h * s1[3 + c] for c in range(3)])


def _hermite_root(h, s0, s1, z_plane):
    def pos(u, c):
        h00 = 2 * u**3 - 3 * u**2 + 1
        h10 = u**3 - 2 * u**2 + u
        h01 = -2 * u**3 + 3 * u**2
        h11 = u**3 - u**2
        return h00 * s0[c] + h10 * h * s0[3 + c] + h01 * s1[c] + h11 * h * s1[3 + c]

    def dpos(u, c):
        return ((6 * u**2 - 6 * u) * s0[c] + (3 * u**2 - 4 * u + 1) * h * s0[3 + c] +
                (-6 * u**2 + 6 * u) * s1[c] + (3 * u**2 - 2 * u) * h * s1[3 + c])

    u = (z_plane - s0[2]) / (s1[2] - s0[2])
    lo, hi = 0.0, 1.0
    for _ in range(60):
        f = pos(u, 2) - z_plane
        if (f > 0) == (s0[2] - z_plane > 0):
            lo = u
        else:
            hi = u
        d = dpos(u, 2)
        un = u - f / d if d != 0 else 0.5 * (lo + hi)
        if not (lo < un < hi):
            un = 0.5 * (lo + hi)
        if abs(un - u) < 1e-16:
            u = un
            break
        u = un
    out = np.array([pos(u, 0), pos(u, 1), z_plane, 0.0, 0.0, 0.0])
    out[3:] = (1 - u) * s0[3:] + u * s1[3:]
    return out
