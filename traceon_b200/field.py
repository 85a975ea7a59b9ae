"""Field objects of the radial path: BEM fields from surface charges and
axial-interpolated fields, mirroring traceon/field.py of the reference.

Every evaluation runs on the GPU.  Besides the reference's one-point methods
(``electrostatic_field_at_point`` etc., traceon/field.py:272-421) the BEM and
axial fields offer batched ``*_at_points`` methods that evaluate an (M, 3)
array of points in one kernel launch; the reference has no batched API
(every point is a separate Python -> C call).

Units: SI, lengths in metres; charges are sigma / eps0 (traceon/__init__.py).
"""
from __future__ import annotations

import copy

import numpy as np

from . import backend as B

FACTOR_AXIAL_DERIV_SAMPLING_2D = 0.2  # traceon/field.py:819


def _is_numeric(x):
    return isinstance(x, (int, float, np.generic))


class EffectivePointCharges:
    """charges (N,), jacobians (N, Q), positions (N, Q, 2|3) with the +, *, -
    algebra of traceon/field.py:46-130."""

    def __init__(self, charges, jacobians, positions, directions=None):
        self.charges = np.array(charges, dtype=np.float64)
        self.jacobians = np.array(jacobians, dtype=np.float64)
        self.positions = np.array(positions, dtype=np.float64)
        self.directions = None if directions is None else np.array(directions, dtype=np.float64)
        N = len(self.charges)
        assert self.charges.shape == (N,) and self.jacobians.shape[0] == N
        assert self.positions.shape[:2] == self.jacobians.shape

    @staticmethod
    def empty_2d():
        return EffectivePointCharges(np.empty((0,)), np.empty((0, B.N_QUAD_2D)), np.empty((0, B.N_QUAD_2D, 2)))

    @staticmethod
    def empty_3d():
        return EffectivePointCharges(np.empty((0,)), np.empty((0, B.N_TRIANGLE_QUAD)),
                                     np.empty((0, B.N_TRIANGLE_QUAD, 3)))

    def is_2d(self):
        return self.jacobians.shape[1] == B.N_QUAD_2D

    def is_3d(self):
        return self.jacobians.shape[1] == B.N_TRIANGLE_QUAD

    def _matches_geometry(self, other):
        return (self.positions.shape == other.positions.shape and np.allclose(self.positions, other.positions)
                and self.jacobians.shape == other.jacobians.shape and np.allclose(self.jacobians, other.jacobians))

    def __len__(self):
        return len(self.charges)

    def __add__(self, other):
        if not isinstance(other, EffectivePointCharges) or self.is_2d() != other.is_2d():
            return NotImplemented
        if self._matches_geometry(other):
            return EffectivePointCharges(self.charges + other.charges, self.jacobians, self.positions)
        return EffectivePointCharges(np.concatenate([self.charges, other.charges]),
                                     np.concatenate([self.jacobians, other.jacobians]),
                                     np.concatenate([self.positions, other.positions]))

    def __radd__(self, other):
        return self.__add__(other)

    def __mul__(self, other):
        if _is_numeric(other):
            return EffectivePointCharges(other * self.charges, self.jacobians, self.positions)
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def __neg__(self):
        return -1 * self

    def __sub__(self, other):
        return self.__add__(-other)

    # ---- device form
    def device_sources(self):
        """Packed (3, N*Q) device rings (r, z, charge*jac), cached."""
        key = (self.charges.tobytes(), self.jacobians.shape)
        cache = getattr(self, '_dev_cache', None)
        if cache is not None and cache[0] == key:
            return cache[1]
        torch = B._torch()
        q = B.to_dev(self.charges, torch.float64)
        j = B.to_dev(self.jacobians, torch.float64)
        p = B.to_dev(self.positions, torch.float64)
        if self.is_3d():
            src = B.dev_pack_current_sources(q, j, p)
        else:
            src = B.dev_pack_sources(q, j, p)
        self._dev_cache = (key, src)
        return src


class Field:
    """Base field: affine frame and bounds (traceon/field.py:133-421)."""

    def __init__(self):
        self._origin = np.zeros(3)
        self._basis = np.eye(3)
        self.field_bounds = None

    def copy(self):
        return copy.copy(self)

    def map_points(self, fun):
        """Copy of the field in the frame moved by the point map `fun`
        (traceon/field.py:168-177): the origin goes to fun(origin), the basis
        vectors to fun(b + origin) - fun(origin)."""
        f = self.copy()
        f._origin = np.asarray(fun(self._origin), dtype=np.float64)
        assert f._origin.shape == (3,), 'Transformation of field did not map origin to a 3D point'
        f._basis = np.array([np.asarray(fun(b + self._origin), dtype=np.float64) - f._origin for b in self._basis])
        assert f._basis.shape == (3, 3), 'Transformation of field did not map unit vectors to a 3D vector'
        assert np.linalg.det(f._basis) != 0, 'Transformations of field have resulted in a two-dimensional system'
        return f

    def move(self, dx=0.0, dy=0.0, dz=0.0):
        """Translated copy (traceon/mesher.py:46-65)."""
        d = np.array([dx, dy, dz], dtype=np.float64)
        return self.map_points(lambda p: np.asarray(p, dtype=np.float64) + d)

    def map_points_to_local(self, point):
        # global = basis @ local + origin (traceon/field.py:154-200)
        p = np.asarray(point, dtype=np.float64) - self._origin
        return p if np.array_equal(self._basis, np.eye(3)) else np.linalg.solve(self._basis, p)

    def set_bounds(self, bounds):
        bounds = np.array(bounds, dtype=np.float64)
        assert bounds.shape == (3, 2)
        self.field_bounds = bounds

    def _within_field_bounds(self, point):
        return self.field_bounds is None or bool(np.all((self.field_bounds[:, 0] <= point) &
                                                        (point <= self.field_bounds[:, 1])))

    def is_electrostatic(self):
        return False

    def is_magnetostatic(self):
        return False

    # one-point API (traceon/field.py:232-336)
    def field_at_point(self, point):
        elec, mag = self.is_electrostatic(), self.is_magnetostatic()
        if elec and not mag:
            return self.electrostatic_field_at_point(point)
        if mag and not elec:
            return self.magnetostatic_field_at_point(point)
        raise RuntimeError("Cannot use field_at_point when both electric and magnetic fields are present, "
                           "use electrostatic_field_at_point or magnetostatic_field_at_point")

    def potential_at_point(self, point):
        elec, mag = self.is_electrostatic(), self.is_magnetostatic()
        if elec and not mag:
            return self.electrostatic_potential_at_point(point)
        if mag and not elec:
            return self.magnetostatic_potential_at_point(point)
        raise RuntimeError("Cannot use potential_at_point when both electric and magnetic fields are present")

    def _global(self, fun_local, point, vector):
        local = self.map_points_to_local(point)
        if not self._within_field_bounds(local):
            return np.zeros(3) if vector else 0.0
        v = fun_local(local)
        return self._basis @ v if vector else v

    def electrostatic_field_at_point(self, point):
        return self._global(self.electrostatic_field_at_local_point, point, True)

    def magnetostatic_field_at_point(self, point):
        return self._global(self.magnetostatic_field_at_local_point, point, True)

    def current_field_at_point(self, point):
        return self._global(self.current_field_at_local_point, point, True)

    def electrostatic_potential_at_point(self, point):
        return self._global(self.electrostatic_potential_at_local_point, point, False)

    def magnetostatic_potential_at_point(self, point):
        return self._global(self.magnetostatic_potential_at_local_point, point, False)

    def electrostatic_field_at_local_point(self, point):
        return np.zeros(3)

    def magnetostatic_field_at_local_point(self, point):
        return np.zeros(3)

    def current_field_at_local_point(self, point):
        return np.zeros(3)

    def electrostatic_potential_at_local_point(self, point):
        return 0.0

    def magnetostatic_potential_at_local_point(self, point):
        return 0.0

    def __add__(self, other):
        if isinstance(other, Field) and not isinstance(other, FieldSuperposition):
            return FieldSuperposition([self, other])
        return NotImplemented

    def __mul__(self, other):
        if _is_numeric(other):
            return FieldSuperposition([self], [other])
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def __neg__(self):
        return -1 * self

    def __sub__(self, other):
        return self + (-other)

    def get_tracer(self, bounds):
        from .tracing import Tracer
        return Tracer(self, bounds)


def _axial_shift(field):
    """z offset of a field whose frame keeps the symmetry axis: origin on the z
    axis and a basis that maps z to z (any rotation about z).  A radially
    symmetric field in such a frame is the same field shifted along z, which
    is what lets superposed radial fields be traced as one source set."""
    o, b = field._origin, field._basis
    if abs(o[0]) > 0 or abs(o[1]) > 0 or not np.allclose(b[:, 2], [0.0, 0.0, 1.0]) or \
            not np.allclose(b[2, :2], 0.0) or not np.allclose(b.T @ b, np.eye(3)):
        raise NotImplementedError('GPU tracing of a superposition needs every member field to keep the z axis '
                                  '(origin on the axis, rotations about z only)')
    return float(o[2])


class FieldSuperposition(Field):
    """Linear combination of fields (traceon/field.py:424-507).  Point
    evaluations sum the member fields.  Tracing is GPU-native (the reference
    calls back into Python for every field evaluation of a superposition,
    traceon/field.py:464-465, tracing.py): radial BEM members collapse into
    one source set (charges times factors, concatenated, shifted along z by
    their origins) and radial axial members on one z grid into one
    coefficient table; mixing BEM and axial members, field bounds on members,
    and frames that move the symmetry axis are not supported."""

    def __init__(self, fields, factors=None):
        super().__init__()
        self.fields = list(fields)
        self.factors = np.ones(len(self.fields)) if factors is None else np.array(factors, dtype=np.float64)

    def electrostatic_field_at_point(self, point):
        return np.sum([fa * f.electrostatic_field_at_point(point) for fa, f in zip(self.factors, self.fields)], axis=0)

    def magnetostatic_field_at_point(self, point):
        return np.sum([fa * f.magnetostatic_field_at_point(point) for fa, f in zip(self.factors, self.fields)], axis=0)

    def electrostatic_potential_at_point(self, point):
        return sum(fa * f.electrostatic_potential_at_point(point) for fa, f in zip(self.factors, self.fields))

    def magnetostatic_potential_at_point(self, point):
        return sum(fa * f.magnetostatic_potential_at_point(point) for fa, f in zip(self.factors, self.fields))

    def is_electrostatic(self):
        return any(f.is_electrostatic() for f in self.fields)

    def is_magnetostatic(self):
        return any(f.is_magnetostatic() for f in self.fields)

    def __add__(self, other):
        if isinstance(other, FieldSuperposition):
            return FieldSuperposition(self.fields + other.fields, np.concatenate([self.factors, other.factors]))
        return FieldSuperposition(self.fields + [other], np.concatenate([self.factors, [1.0]]))

    def __radd__(self, other):
        if isinstance(other, Field):
            return FieldSuperposition([other] + self.fields, np.concatenate([[1.0], self.factors]))
        return NotImplemented

    def __mul__(self, other):
        if _is_numeric(other):
            return FieldSuperposition(self.fields, other * self.factors)
        return NotImplemented

    def __len__(self):
        return len(self.fields)

    def _members(self):
        """(factor, field) pairs with nested superpositions expanded."""
        out = []
        for fa, f in zip(self.factors, self.fields):
            if isinstance(f, FieldSuperposition):
                out += [(float(fa) * g_fa, g) for g_fa, g in f._members()]
            else:
                out.append((float(fa), f))
        return out

    def _trace_field(self):
        """(tb_field_t, keep-alive tensors) of the whole superposition."""
        torch = B._torch()
        members = self._members()
        if not members:
            raise ValueError('empty superposition')
        if any(f.field_bounds is not None for _, f in members):
            raise NotImplementedError('GPU tracing of a superposition whose members have field bounds')
        if all(isinstance(f, FieldRadialBEM) for _, f in members):
            groups = ([], [], [])
            for fa, f in members:
                dz = _axial_shift(f)
                for lst, pc in zip(groups, (f.electrostatic_point_charges, f.magnetostatic_point_charges,
                                            f.current_point_charges)):
                    if len(pc):
                        src = pc.device_sources().clone()
                        src[1] += dz
                        src[2] *= fa
                        lst.append(src)
            dev = B.device()
            e, m, c = (torch.cat(lst, 1).contiguous() if lst else torch.empty((3, 0), dtype=torch.float64, device=dev)
                       for lst in groups)
            f = B.TbField(e.data_ptr() if e.numel() else None, e.shape[1], m.data_ptr() if m.numel() else None,
                          m.shape[1], c.data_ptr() if c.numel() else None, c.shape[1], None, None, None, None, 0)
            return f, (e, m, c)
        if all(isinstance(f, FieldRadialAxial) for _, f in members):
            fa0, f0 = members[0]
            z0 = f0.z + _axial_shift(f0)
            ec = np.zeros_like(f0.electrostatic_coeffs)
            mc = np.zeros_like(f0.magnetostatic_coeffs)
            for fa, f in members:
                if f.z.shape != f0.z.shape or not np.allclose(f.z + _axial_shift(f), z0, rtol=0, atol=1e-15):
                    raise NotImplementedError('GPU tracing of a superposition of axial fields on different z grids')
                ec += fa * f.electrostatic_coeffs
                mc += fa * f.magnetostatic_coeffs
            zt, ect, mct = B.to_dev(z0, torch.float64), B.to_dev(ec, torch.float64), B.to_dev(mc, torch.float64)
            f = B.TbField(None, 0, None, 0, None, 0, None, zt.data_ptr(), ect.data_ptr(), mct.data_ptr(), len(z0))
            return f, (zt, ect, mct)
        raise NotImplementedError('GPU tracing of a superposition that mixes BEM and axial fields')


class FieldBEM(Field):
    """Field of surface charges (traceon/field.py:509-617)."""

    def __init__(self, electrostatic_point_charges, magnetostatic_point_charges, current_point_charges):
        super().__init__()
        self.electrostatic_point_charges = electrostatic_point_charges
        self.magnetostatic_point_charges = magnetostatic_point_charges
        self.current_point_charges = current_point_charges

    def is_electrostatic(self):
        return len(self.electrostatic_point_charges) > 0

    def is_magnetostatic(self):
        return len(self.magnetostatic_point_charges) > 0 or len(self.current_point_charges) > 0

    def _matches_geometry(self, other):
        return (self.__class__ == other.__class__ and np.allclose(self._origin, other._origin)
                and np.allclose(self._basis, other._basis))

    def __add__(self, other):
        if isinstance(other, FieldBEM) and self._matches_geometry(other):
            f = self.copy()
            f.electrostatic_point_charges = self.electrostatic_point_charges + other.electrostatic_point_charges
            f.magnetostatic_point_charges = self.magnetostatic_point_charges + other.magnetostatic_point_charges
            f.current_point_charges = self.current_point_charges + other.current_point_charges
            return f
        return super().__add__(other)

    def __radd__(self, other):
        return self.__add__(other)

    def __mul__(self, other):
        if _is_numeric(other):
            f = self.copy()
            f.electrostatic_point_charges = self.electrostatic_point_charges * other
            f.magnetostatic_point_charges = self.magnetostatic_point_charges * other
            f.current_point_charges = self.current_point_charges * other
            return f
        return super().__mul__(other)

    def __rmul__(self, other):
        return self.__mul__(other)

    def __neg__(self):
        return self.__mul__(-1.0)

    def __sub__(self, other):
        return self.__add__(-other)

    def area_of_element(self, i):
        jac = self.electrostatic_point_charges.jacobians
        pos = self.electrostatic_point_charges.positions
        return 2 * np.pi * np.sum(jac[i] * pos[i, :, 0])

    def charge_on_element(self, i):
        return self.area_of_element(i) * self.electrostatic_point_charges.charges[i]

    def charge_on_elements(self, indices):
        return sum(self.charge_on_element(i) for i in indices)


class FieldRadialBEM(FieldBEM):
    """Radially symmetric BEM field (traceon/field.py:620-816)."""

    def __init__(self, electrostatic_point_charges=None, magnetostatic_point_charges=None,
                 current_point_charges=None):
        super().__init__(electrostatic_point_charges or EffectivePointCharges.empty_2d(),
                         magnetostatic_point_charges or EffectivePointCharges.empty_2d(),
                         current_point_charges or EffectivePointCharges.empty_3d())

    # ---- batched device evaluation
    def _points_t(self, points):
        torch = B._torch()
        pts = B.to_dev(np.asarray(points, dtype=np.float64).reshape(-1, 3), torch.float64)
        return pts

    def electrostatic_potential_at_points(self, points):
        pts = self._points_t(points)
        pot, _ = B.dev_field_points(pts, self.electrostatic_point_charges.device_sources(), True, False)
        return pot.cpu().numpy()

    def electrostatic_field_at_points(self, points):
        pts = self._points_t(points)
        _, f = B.dev_field_points(pts, self.electrostatic_point_charges.device_sources(), False, True)
        return f.cpu().numpy()

    def magnetostatic_field_at_points(self, points):
        pts = self._points_t(points)
        _, f = B.dev_field_points(pts, self.magnetostatic_point_charges.device_sources(), False, True)
        if len(self.current_point_charges):
            f = f + B.dev_current_field_points(pts, self.current_point_charges.device_sources())
        return f.cpu().numpy()

    def magnetostatic_potential_at_points(self, points):
        pts = self._points_t(points)
        pot, _ = B.dev_field_points(pts, self.magnetostatic_point_charges.device_sources(), True, False)
        return pot.cpu().numpy()

    # ---- one-point API
    def electrostatic_field_at_local_point(self, point):
        return self.electrostatic_field_at_points(np.asarray(point, dtype=np.float64)[None])[0]

    def magnetostatic_field_at_local_point(self, point):
        return self.magnetostatic_field_at_points(np.asarray(point, dtype=np.float64)[None])[0]

    def current_field_at_local_point(self, point):
        if not len(self.current_point_charges):
            return np.zeros(3)
        pts = self._points_t(np.asarray(point, dtype=np.float64)[None])
        return B.dev_current_field_points(pts, self.current_point_charges.device_sources()).cpu().numpy()[0]

    def electrostatic_potential_at_local_point(self, point):
        return float(self.electrostatic_potential_at_points(np.asarray(point, dtype=np.float64)[None])[0])

    def magnetostatic_potential_at_local_point(self, point):
        return float(self.magnetostatic_potential_at_points(np.asarray(point, dtype=np.float64)[None])[0])

    def get_electrostatic_axial_potential_derivatives(self, z):
        torch = B._torch()
        zt = B.to_dev(np.asarray(z, dtype=np.float64), torch.float64)
        return B.dev_axial_derivatives(zt, self.electrostatic_point_charges.device_sources()).cpu().numpy()

    def get_magnetostatic_axial_potential_derivatives(self, z):
        torch = B._torch()
        zt = B.to_dev(np.asarray(z, dtype=np.float64), torch.float64)
        d = B.dev_axial_derivatives(zt, self.magnetostatic_point_charges.device_sources())
        if len(self.current_point_charges):
            d = d + B.dev_axial_derivatives(zt, self.current_point_charges.device_sources(), current=True)
        return d.cpu().numpy()

    def get_current_axial_potential_derivatives(self, z):
        torch = B._torch()
        zt = B.to_dev(np.asarray(z, dtype=np.float64), torch.float64)
        return B.dev_axial_derivatives(zt, self.current_point_charges.device_sources(), current=True).cpu().numpy()

    # ---- tracing
    def _trace_field(self):
        """(tb_field_t, keep-alive tensors) for the GPU tracer."""
        torch = B._torch()
        e = self.electrostatic_point_charges.device_sources()
        m = self.magnetostatic_point_charges.device_sources()
        c = self.current_point_charges.device_sources()
        fb = None if self.field_bounds is None else B.to_dev(self.field_bounds, torch.float64)
        f = B.TbField(e.data_ptr() if e.numel() else None, e.shape[1], m.data_ptr() if m.numel() else None,
                      m.shape[1], c.data_ptr() if c.numel() else None, c.shape[1],
                      None if fb is None else fb.data_ptr(), None, None, None, 0)
        return f, (e, m, c, fb)

    def get_low_level_trace_function(self):
        """(field_fun, args) of traceon/field.py:814-816 for backend.trace_particle."""
        args = B.FieldEvaluationArgsRadial(self.electrostatic_point_charges, self.magnetostatic_point_charges,
                                           self.current_point_charges, self.field_bounds)
        return B.FIELD_RADIAL_TRACEABLE, args


class FieldAxial(Field):
    """Axial series field (traceon/field.py:821-904)."""

    def __init__(self, field, z, electrostatic_coeffs=None, magnetostatic_coeffs=None):
        super().__init__()
        self.field = field
        self._origin = field._origin
        self._basis = field._basis
        N = len(z)
        assert z.shape == (N,) and z[0] < z[-1], "z values in axial interpolation should be ascending"
        self.z = z
        self.electrostatic_coeffs = electrostatic_coeffs if electrostatic_coeffs is not None \
            else np.zeros_like(magnetostatic_coeffs)
        self.magnetostatic_coeffs = magnetostatic_coeffs if magnetostatic_coeffs is not None \
            else np.zeros_like(electrostatic_coeffs)
        self.has_electrostatic = bool(np.any(self.electrostatic_coeffs != 0.))
        self.has_magnetostatic = bool(np.any(self.magnetostatic_coeffs != 0.))

    def is_electrostatic(self):
        return self.has_electrostatic

    def is_magnetostatic(self):
        return self.has_magnetostatic

    def __add__(self, other):
        if isinstance(other, FieldAxial) and self.z.shape == other.z.shape and np.allclose(self.z, other.z):
            f = self.copy()
            f.electrostatic_coeffs = self.electrostatic_coeffs + other.electrostatic_coeffs
            f.magnetostatic_coeffs = self.magnetostatic_coeffs + other.magnetostatic_coeffs
            f._dev = None
            return f
        return super().__add__(other)

    def __mul__(self, other):
        # The reference's FieldAxial.__mul__ scales the electrostatic
        # coefficients into the magnetostatic slot (traceon/field.py:895);
        # here both are scaled by their own values.
        if _is_numeric(other):
            f = self.copy()
            f.electrostatic_coeffs = other * self.electrostatic_coeffs
            f.magnetostatic_coeffs = other * self.magnetostatic_coeffs
            f._dev = None
            return f
        return super().__mul__(other)

    def __rmul__(self, other):
        return self.__mul__(other)

    def __neg__(self):
        return self.__mul__(-1.0)


class FieldRadialAxial(FieldAxial):
    """Axial-derivative interpolation of a radial BEM field
    (traceon/field.py:940-1066): derivatives at N equally spaced z on the
    axis (GPU ring sums), then quintic-Hermite / cubic-spline coefficients
    (GPU), evaluated through the radial series expansion."""

    def __init__(self, field, zmin, zmax, N=None):
        assert isinstance(field, FieldRadialBEM)
        z, ec, mc = FieldRadialAxial._get_interpolation_coefficients(field, zmin, zmax, N=N)
        super().__init__(field, z, ec, mc)
        assert self.electrostatic_coeffs.shape == (len(z) - 1, B.DERIV_2D_MAX, 6)

    @staticmethod
    def _get_interpolation_coefficients(field, zmin, zmax, N=None):
        assert zmax > zmin, "zmax should be bigger than zmin"
        torch = B._torch()
        N_charges = max(len(field.electrostatic_point_charges.charges), len(field.magnetostatic_point_charges.charges))
        N = N if N is not None else int(FACTOR_AXIAL_DERIV_SAMPLING_2D * N_charges)
        z = np.linspace(zmin, zmax, N)
        zt = B.to_dev(z, torch.float64)
        dz = z[1] - z[0]
        ed = B.dev_axial_derivatives(zt, field.electrostatic_point_charges.device_sources())
        md = B.dev_axial_derivatives(zt, field.magnetostatic_point_charges.device_sources())
        if len(field.current_point_charges):
            md = md + B.dev_axial_derivatives(zt, field.current_point_charges.device_sources(), current=True)
        ec = B.dev_axial_coefficients(ed, dz)
        mc = B.dev_axial_coefficients(md, dz)
        return z, ec.cpu().numpy(), mc.cpu().numpy()

    def _device(self):
        dev = getattr(self, '_dev', None)
        if dev is None:
            torch = B._torch()
            dev = (B.to_dev(self.z, torch.float64), B.to_dev(self.electrostatic_coeffs, torch.float64),
                   B.to_dev(self.magnetostatic_coeffs, torch.float64))
            self._dev = dev
        return dev

    def _eval(self, points, mag, want_pot):
        torch = B._torch()
        zt, ec, mc = self._device()
        pts = B.to_dev(np.asarray(points, dtype=np.float64).reshape(-1, 3), torch.float64)
        pot, f = B.dev_axial_field_points(pts, zt, mc if mag else ec, want_pot, not want_pot)
        return (pot if want_pot else f).cpu().numpy()

    def electrostatic_field_at_points(self, points):
        return self._eval(points, False, False)

    def magnetostatic_field_at_points(self, points):
        return self._eval(points, True, False)

    def electrostatic_potential_at_points(self, points):
        return self._eval(points, False, True)

    def magnetostatic_potential_at_points(self, points):
        return self._eval(points, True, True)

    def electrostatic_field_at_local_point(self, point):
        return B.field_radial_derivs(np.asarray(point, dtype=np.float64), self.z, self.electrostatic_coeffs)

    def magnetostatic_field_at_local_point(self, point):
        return B.field_radial_derivs(np.asarray(point, dtype=np.float64), self.z, self.magnetostatic_coeffs)

    def electrostatic_potential_at_local_point(self, point):
        return B.potential_radial_derivs(np.asarray(point, dtype=np.float64), self.z, self.electrostatic_coeffs)

    def magnetostatic_potential_at_local_point(self, point):
        return B.potential_radial_derivs(np.asarray(point, dtype=np.float64), self.z, self.magnetostatic_coeffs)

    def _trace_field(self):
        zt, ec, mc = self._device()
        f = B.TbField(None, 0, None, 0, None, 0, None, zt.data_ptr(), ec.data_ptr(), mc.data_ptr(), len(self.z))
        return f, (zt, ec, mc)

    def get_low_level_trace_function(self):
        args = B.FieldDerivsArgs(self.z, self.electrostatic_coeffs, self.magnetostatic_coeffs)
        return B.FIELD_RADIAL_DERIVS_TRACEABLE, args
