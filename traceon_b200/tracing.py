"""Particle tracing on the GPU, mirroring traceon/tracing.py of the reference.

``Tracer(field, bounds)`` keeps the reference's interface (``trace_single``,
``trace_multiple``, ``__call__``; traceon/tracing.py:104-245).  Where the
reference traces particles one after another on one CPU core, every call
here launches one persistent GPU kernel for all particles
(``tb_trace_rk45``).  ``trace_endpoints`` is the batched form used for
throughput: it returns only the final state and the crossing of an exit
plane z = const (cubic Hermite interpolation between the two accepted steps
that bracket it) instead of whole trajectories.
"""
from __future__ import annotations

import ctypes as C
from math import sqrt, sin, cos

import numpy as np
from scipy.constants import m_e, e

from . import backend as B

DEFAULT_MAX_ATTEMPTS = 100_000
DEFAULT_ROWS = 4096


def _convert_velocity_to_SI(velocity, mass):
    speed_eV = np.linalg.norm(velocity)
    speed = sqrt(2 * speed_eV * e / mass)
    direction = np.array(velocity) / speed_eV
    return speed * direction


def velocity_vec(eV, direction, mass=m_e):
    """traceon/tracing.py:32-56"""
    assert eV > 0.0, "Please provide a positive energy in eV"
    direction_ = np.array(direction, dtype=np.float64)
    assert direction_.shape == (3,), "Please provide a three dimensional direction vector"
    return _convert_velocity_to_SI(eV * direction_ / np.linalg.norm(direction_), mass)


def velocity_vec_spherical(eV, theta, phi):
    return velocity_vec(eV, [sin(theta) * cos(phi), sin(theta) * sin(phi), cos(theta)])


def velocity_vec_xz_plane(eV, angle, downward=True):
    sign = -1 if downward else 1
    return velocity_vec(eV, [sin(angle), 0.0, sign * cos(angle)])


class TraceResult:
    """Device-side result of a batched trace (all tensors on the GPU)."""

    def __init__(self, status, final, plane, counters, rows=None, nrows=None):
        self.status = status          # (n,) int32, backend.TRACE_*
        self.final = final            # (n, 7) t, x, y, z, vx, vy, vz
        self.plane = plane            # (n, 7) crossing of the exit plane (NaN if none)
        self.counters = counters      # (n, 2) accepted steps, attempts
        self.rows = rows              # (n, max_rows, 7) or None
        self.nrows = nrows            # (n,) int64 or None

    def plane_intersection(self, p0, normal):
        """Crossing of every stored trajectory with the plane through p0
        with normal `normal`, nearest the trajectory's end, by linear
        interpolation (traceon/tracing.py:247-272 for one trajectory), on the
        device.  Needs a trace with max_rows > 0.  Returns device tensors
        (out (n, 7) t, x..vz, NaN where none; found (n) bool)."""
        if self.rows is None:
            raise ValueError('plane_intersection needs stored trajectories (trace with max_rows > 0)')
        return B.dev_plane_intersection_rows(self.rows, self.nrows, p0, normal)

    def xy_plane_intersection(self, z):
        return self.plane_intersection([0, 0, z], [0, 0, 1])

    def xz_plane_intersection(self, y):
        return self.plane_intersection([0, y, 0], [0, 1, 0])

    def yz_plane_intersection(self, x):
        return self.plane_intersection([x, 0, 0], [1, 0, 0])

    def axis_intersection(self):
        """z of each trajectory's crossing of x = 0 (traceon/tracing.py:317-335),
        a device tensor (n,); NaN where there is none."""
        return self.yz_plane_intersection(0.0)[0][:, 3]

    def focus_position(self, plane=False):
        """Least-squares focus of the traced beam from its final states
        (traceon/focus.py:9-42), or from the exit-plane crossings when
        `plane`: a device tensor (3,) = (x, y, z)."""
        return B.dev_focus_position(self.plane if plane else self.final)


class Tracer:
    """General tracer (traceon/tracing.py:104-245) on the GPU."""

    def __init__(self, field, bounds):
        self.field = field
        bounds = np.array(bounds).astype(np.float64)
        assert bounds.shape == (3, 2)
        self.bounds = bounds
        if not hasattr(field, '_trace_field'):
            raise NotImplementedError(f'{type(field).__name__} cannot be traced on the GPU; trace a '
                                      'FieldRadialBEM or FieldRadialAxial')

    def __str__(self):
        b = ' '.join(f'({lo:.2e}, {hi:.2e})' for lo, hi in self.bounds)
        return f'<traceon_b200 Tracer of {self.field.__class__.__name__}, bounds: {b} m>'

    def __call__(self, *args, **kwargs):
        return self.trace_single(*args, **kwargs)

    # ------------------------------------------------------------ device core
    def trace_device(self, start, qm, t0=None, atol=1e-8, plane_z=None, max_rows=0,
                     max_attempts=DEFAULT_MAX_ATTEMPTS, team_warps=0, stream=None):
        """Traces particles whose start states (n, 6) and charge/mass (n,) are
        already device tensors; returns a TraceResult of device tensors.
        team_warps: warps per particle for BEM fields (1, 2, 4, 8), 0 for the
        built-in rule, or 'tune' for the measured choice (traceon_b200.autotune,
        cached per device and problem size)."""
        torch = B._torch()
        n = start.shape[0]
        dev = start.device
        f, keep = self.field._trace_field()
        if team_warps == 'tune':
            from . import autotune
            team_warps = 0
            if f.axial_z is None and n:
                team_warps = autotune.best_team_warps(self, start, qm, atol, max_attempts, f.n_elec + f.n_mag)
        o = B.TbTraceOpts()
        for i, v in enumerate(self.bounds.reshape(-1)):
            o.bounds[i] = float(v)
        o.atol = float(atol)
        o.plane_z = 0.0 if plane_z is None else float(plane_z)
        o.record_plane = 0 if plane_z is None else 1
        o.max_attempts = int(max_attempts)
        o.max_rows = int(max_rows)
        o.team_warps = int(team_warps)
        status = torch.empty(n, dtype=torch.int32, device=dev)
        final = torch.empty((n, 7), dtype=torch.float64, device=dev)
        plane = torch.empty((n, 7), dtype=torch.float64, device=dev) if plane_z is not None else None
        counters = torch.empty((n, 2), dtype=torch.int64, device=dev)
        rows = torch.empty((n, max_rows, 7), dtype=torch.float64, device=dev) if max_rows else None
        nrows = torch.empty(n, dtype=torch.int64, device=dev) if max_rows else None
        work = torch.empty(1, dtype=torch.int32, device=dev)
        s = B._stream() if stream is None else stream
        r = B.backend_lib.tb_trace_rk45(start.data_ptr(), None if t0 is None else t0.data_ptr(), qm.data_ptr(), n,
                                        C.byref(f), C.byref(o), B._ptr(rows), B._ptr(nrows), status.data_ptr(),
                                        final.data_ptr(), B._ptr(plane), counters.data_ptr(), work.data_ptr(), s)
        if r != B.TB_OK:
            raise B.BackendError(f'tb_trace_rk45 failed with status {r}')
        res = TraceResult(status, final, plane, counters, rows, nrows)
        res._keep = (keep, start, qm, t0, work)
        return res

    def _start(self, position, velocity, mass, charge):
        torch = B._torch()
        positions = np.atleast_2d(np.asarray(position, dtype=np.float64))
        velocities = np.atleast_2d(np.asarray(velocity, dtype=np.float64))
        positions, velocities = np.broadcast_arrays(positions, velocities)
        n = len(positions)
        masses = np.broadcast_to(np.asarray(mass, dtype=np.float64), (n,))
        charges = np.broadcast_to(np.asarray(charge, dtype=np.float64), (n,))
        start = B.to_dev(np.concatenate([positions, velocities], axis=1), torch.float64)
        qm = B.to_dev(charges / masses, torch.float64)
        return start, qm

    # ------------------------------------------------------------ reference API
    def trace_multiple(self, position, velocity, mass=m_e, charge=-e, atol=1e-8, max_rows=DEFAULT_ROWS):
        """Traces all particles in one GPU launch; returns a list of
        (times, states (n, 6)) like traceon/tracing.py:210-245.  Trajectories
        longer than `max_rows` continue in further launches from their last
        state (the block continuation of traceon/backend/__init__.py:397-412)."""
        torch = B._torch()
        start, qm = self._start(position, velocity, mass, charge)
        n = start.shape[0]
        times = [[] for _ in range(n)]
        states = [[] for _ in range(n)]
        active = np.arange(n)
        t0 = torch.zeros(n, dtype=torch.float64, device=start.device)
        first = True
        while len(active):
            res = self.trace_device(start, qm, t0=t0, atol=atol, max_rows=max_rows)
            st = res.status.cpu().numpy()
            nr = res.nrows.cpu().numpy()
            rows = res.rows.cpu().numpy()
            for k, i in enumerate(active):
                rk = rows[k, :nr[k]]
                skip = 0 if first else 1
                times[i].append(rk[skip:, 0])
                states[i].append(rk[skip:, 1:])
            bad = st[(st != B.TRACE_EXITED) & (st != B.TRACE_ROWS_FULL)]
            if len(bad):
                raise B.BackendError(f'tracing ended with status {int(bad[0])} (1 = attempt cap, 3 = non-finite)')
            cont = np.nonzero(st == B.TRACE_ROWS_FULL)[0]
            if not len(cont):
                break
            last = torch.as_tensor(rows[cont, nr[cont] - 1], device=start.device)
            start = last[:, 1:].contiguous()
            t0 = last[:, 0].contiguous()
            qm = qm[torch.as_tensor(cont, device=start.device)].contiguous()
            active = active[cont]
            first = False
        return [(np.concatenate(t), np.concatenate(s)) for t, s in zip(times, states)]

    def trace_single(self, position, velocity, mass=m_e, charge=-e, atol=1e-8):
        """traceon/tracing.py:144-185"""
        return self.trace_multiple(np.asarray(position)[None], np.asarray(velocity)[None], mass, charge, atol)[0]

    def trace_endpoints(self, position, velocity, plane_z, mass=m_e, charge=-e, atol=1e-8,
                        max_attempts=DEFAULT_MAX_ATTEMPTS, team_warps=0):
        """Batched endpoint tracing: host arrays in, host arrays out.  Returns
        (plane (n, 7), final (n, 7), status (n,), counters (n, 2))."""
        start, qm = self._start(position, velocity, mass, charge)
        res = self.trace_device(start, qm, atol=atol, plane_z=plane_z, max_attempts=max_attempts,
                                team_warps=team_warps)
        return (res.plane.cpu().numpy(), res.final.cpu().numpy(), res.status.cpu().numpy(),
                res.counters.cpu().numpy())


def trace_geometries(fields, bounds, positions, velocities, plane_z, mass=m_e, charge=-e, atol=1e-8,
                     max_attempts=DEFAULT_MAX_ATTEMPTS, team_warps=0):
    """Endpoint tracing of particles through several geometries in one GPU
    launch (tb_trace_rk45_geometries): fields[g] is a FieldRadialBEM
    (electrostatic charges only, no field bounds) and positions[g],
    velocities[g] (n_g, 3) its particles.  The reference traces one field at
    a time.  Returns, per geometry, (plane (n_g, 7), final (n_g, 7),
    status (n_g,), counters (n_g, 2)) like Tracer.trace_endpoints."""
    from .field import FieldRadialBEM
    torch = B._torch()
    if len(fields) != len(positions) or len(fields) != len(velocities) or not fields:
        raise ValueError('one list entry of positions and velocities per field')
    srcs, offsets = [], [0]
    for f in fields:
        if not isinstance(f, FieldRadialBEM) or f.field_bounds is not None or \
                len(f.magnetostatic_point_charges) or len(f.current_point_charges):
            raise NotImplementedError('trace_geometries takes electrostatic FieldRadialBEM fields without bounds')
        src = f.electrostatic_point_charges.device_sources()
        srcs.append(src)
        offsets.append(offsets[-1] + src.shape[1])
    esrc = torch.cat(srcs, 1).contiguous()
    counts = [len(np.atleast_2d(p)) for p in positions]
    geom = np.repeat(np.arange(len(fields), dtype=np.int32), counts)
    pos = np.concatenate([np.atleast_2d(np.asarray(p, dtype=np.float64)) for p in positions])
    vel = np.concatenate([np.atleast_2d(np.asarray(v, dtype=np.float64)) for v in velocities])
    n = len(pos)
    dev = esrc.device
    start = B.to_dev(np.concatenate([pos, vel], axis=1), torch.float64)
    qm = torch.full((n,), float(charge) / float(mass), dtype=torch.float64, device=dev)
    geom_t = B.to_dev(geom, torch.int32)
    off_t = B.to_dev(np.array(offsets, dtype=np.int64), torch.int64)
    f = B.TbField(esrc.data_ptr() if esrc.numel() else None, esrc.shape[1], None, 0, None, 0, None, None, None,
                  None, 0)
    o = B.TbTraceOpts()
    for i, v in enumerate(np.asarray(bounds, dtype=np.float64).reshape(-1)):
        o.bounds[i] = float(v)
    o.atol, o.plane_z, o.record_plane = float(atol), float(plane_z), 1
    o.max_attempts, o.max_rows, o.team_warps = int(max_attempts), 0, int(team_warps)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    final = torch.empty((n, 7), dtype=torch.float64, device=dev)
    plane = torch.empty((n, 7), dtype=torch.float64, device=dev)
    counters = torch.empty((n, 2), dtype=torch.int64, device=dev)
    work = torch.empty(1, dtype=torch.int32, device=dev)
    B._call('tb_trace_rk45_geometries', start.data_ptr(), None, qm.data_ptr(), geom_t.data_ptr(), n, C.byref(f),
            off_t.data_ptr(), len(fields), None, C.byref(o), None, None, status.data_ptr(), final.data_ptr(),
            plane.data_ptr(), counters.data_ptr(), work.data_ptr(), B._stream())
    out = [a.cpu().numpy() for a in (plane, final, status, counters)]
    cuts = np.cumsum(counts)[:-1]
    return [tuple(x) for x in zip(*(np.split(a, cuts) for a in out))]


def plane_intersection(positions, p0, normal):
    """traceon/tracing.py:247-272 (linear interpolation, searched from the end)."""
    positions = np.array(positions, dtype=np.float64)
    assert positions.shape == (len(positions), 6), "The positions array should have shape (N, 6)"
    return B.plane_intersection(positions, np.array(p0, dtype=np.float64), np.array(normal, dtype=np.float64))


def xy_plane_intersection(positions, z):
    return plane_intersection(positions, [0, 0, z], [0, 0, 1])


def xz_plane_intersection(positions, y):
    return plane_intersection(positions, [0, y, 0], [0, 1, 0])


def yz_plane_intersection(positions, x):
    return plane_intersection(positions, [x, 0, 0], [1, 0, 0])


def axis_intersection(positions):
    return yz_plane_intersection(positions, 0)[2]
