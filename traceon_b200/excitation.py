"""Meshes and excitations for the radial solver, mirroring the parts of
traceon/mesher.py (``Mesh``, :182-236) and traceon/excitation.py
(``Excitation``, :90-451) that the radial BEM path reads.

The solver accepts either these objects or the reference's own ``Mesh`` /
``Excitation`` (it only calls ``get_electrostatic_active_elements``,
``get_magnetostatic_active_elements``, ``excitation_types``, ``mesh`` and
``_split_for_superposition``).  Lengths are metres.
"""
from __future__ import annotations

from enum import IntEnum

import numpy as np


class Symmetry(IntEnum):
    RADIAL = 0
    THREE_D = 2


class ExcitationType(IntEnum):
    """traceon/excitation.py:49-58"""
    VOLTAGE_FIXED = 1
    VOLTAGE_FUN = 2
    DIELECTRIC = 3
    CURRENT = 4
    MAGNETOSTATIC_POT = 5
    MAGNETIZABLE = 6
    PERMANENT_MAGNET = 7

    def is_electrostatic(self):
        return self in (ExcitationType.VOLTAGE_FIXED, ExcitationType.VOLTAGE_FUN, ExcitationType.DIELECTRIC)

    def is_magnetostatic(self):
        return self in (ExcitationType.MAGNETOSTATIC_POT, ExcitationType.MAGNETIZABLE, ExcitationType.CURRENT,
                        ExcitationType.PERMANENT_MAGNET)


class Mesh:
    """Line4 (cubic) line mesh with named groups: points (P, 3), lines (N, 4)
    as [start, end, 1/3-point, 2/3-point] point indices, physical_to_lines
    name -> line indices."""

    def __init__(self, points=None, lines=None, physical_to_lines=None):
        self.points = np.empty((0, 3)) if points is None else np.array(points, dtype=np.float64)
        self.lines = np.empty((0, 4), dtype=np.uint64) if lines is None else np.array(lines, dtype=np.uint64)
        self.physical_to_lines = {k: np.asarray(v) for k, v in (physical_to_lines or {}).items()}
        self.triangles = np.empty((0, 3), dtype=np.uint64)
        self.physical_to_triangles = {}
        assert self.lines.ndim == 2 and self.lines.shape[1] in (2, 4)
        assert np.all(self.lines < max(len(self.points), 1))

    @staticmethod
    def from_geometry(geo):
        """Mesh of a traceon_b200.geometry.LensGeometry."""
        N = len(geo)
        lines = np.arange(4 * N).reshape(N, 4)
        phys = {name: np.nonzero(geo.electrode_index == e)[0] for e, name in enumerate(geo.names)}
        return Mesh(geo.vertices.reshape(-1, 3), lines, phys)

    def is_higher_order(self):
        return self.lines.shape[1] == 4

    def is_2d(self):
        return True

    def is_3d(self):
        return False

    def get_electrodes(self):
        return list(self.physical_to_lines.keys())


class Excitation:
    """Named-electrode excitations (traceon/excitation.py:90-451), radial only."""

    def __init__(self, mesh, symmetry=Symmetry.RADIAL):
        assert symmetry == Symmetry.RADIAL, 'only radial symmetry is implemented'
        self.mesh = mesh
        self.symmetry = symmetry
        self.excitation_types = {}

    def _check(self, name):
        assert name in self.mesh.physical_to_lines, f"Electrode '{name}' is not present in the mesh"

    def add_voltage(self, **kwargs):
        for name, v in kwargs.items():
            self._check(name)
            if callable(v):
                self.excitation_types[name] = (ExcitationType.VOLTAGE_FUN, v)
            else:
                self.excitation_types[name] = (ExcitationType.VOLTAGE_FIXED, float(v))

    def add_dielectric(self, **kwargs):
        for name, k in kwargs.items():
            self._check(name)
            self.excitation_types[name] = (ExcitationType.DIELECTRIC, float(k))

    def add_electrostatic_boundary(self, *names):
        """A boundary is a dielectric of permittivity 0 (excitation.py:263-285)."""
        self.add_dielectric(**{n: 0.0 for n in names})

    def add_magnetostatic_potential(self, **kwargs):
        for name, v in kwargs.items():
            self._check(name)
            self.excitation_types[name] = (ExcitationType.MAGNETOSTATIC_POT, float(v))

    def add_magnetizable(self, **kwargs):
        for name, mu in kwargs.items():
            self._check(name)
            self.excitation_types[name] = (ExcitationType.MAGNETIZABLE, float(mu))

    def add_magnetostatic_boundary(self, *names):
        self.add_magnetizable(**{n: 0.0 for n in names})

    def has_current(self):
        return any(t == ExcitationType.CURRENT for t, _ in self.excitation_types.values())

    def has_permanent_magnet(self):
        return any(t == ExcitationType.PERMANENT_MAGNET for t, _ in self.excitation_types.values())

    def is_electrostatic(self):
        return any(t in (ExcitationType.VOLTAGE_FIXED, ExcitationType.VOLTAGE_FUN)
                   for t, _ in self.excitation_types.values())

    def is_magnetostatic(self):
        return any(t in (ExcitationType.MAGNETOSTATIC_POT, ExcitationType.PERMANENT_MAGNET, ExcitationType.CURRENT)
                   for t, _ in self.excitation_types.values())

    def _get_active_elements(self, type_):
        """traceon/excitation.py:348-373"""
        elements = self.mesh.lines
        physicals = self.mesh.physical_to_lines

        def type_check(t):
            if type_ == 'electrostatic':
                return ExcitationType(t).is_electrostatic()
            return t in (ExcitationType.MAGNETIZABLE, ExcitationType.MAGNETOSTATIC_POT)

        inactive = np.full(len(elements), True)
        for name, value in self.excitation_types.items():
            if type_check(value[0]):
                inactive[physicals[name]] = False
        map_index = np.arange(len(elements)) - np.cumsum(inactive)
        names = {n: map_index[i] for n, i in physicals.items()
                 if n in self.excitation_types and type_check(self.excitation_types[n][0])}
        return self.mesh.points[elements[~inactive].astype(np.int64)], names

    def assemble_device(self, type_='electrostatic'):
        """The active elements of `type_` ('electrostatic' or
        'magnetostatic') assembled on the device: (vertices (N, 4, 3) float64,
        excitation types (N,) uint8, values (N,) float64), in the element order
        of _get_active_elements (traceon/excitation.py:348-373) and with the
        per-element type and value of traceon/solver.py:46-61 -- a scatter of
        each named group's type and value over all lines, then one gather of
        the active lines' points.  VOLTAGE_FUN rows get NaN values (the solver
        evaluates the functions on the element centres)."""
        from . import backend as B
        torch = B._torch()
        dev = B.device()
        n = len(self.mesh.lines)
        types = torch.zeros(n, dtype=torch.uint8, device=dev)
        values = torch.zeros(n, dtype=torch.float64, device=dev)
        active = torch.zeros(n, dtype=torch.bool, device=dev)
        for name, (t, v) in self.excitation_types.items():
            ok = ExcitationType(t).is_electrostatic() if type_ == 'electrostatic' else \
                t in (ExcitationType.MAGNETIZABLE, ExcitationType.MAGNETOSTATIC_POT)
            if not ok:
                continue
            idx = torch.as_tensor(np.asarray(self.mesh.physical_to_lines[name], dtype=np.int64), device=dev)
            active[idx] = True
            types[idx] = int(t)
            values[idx] = float('nan') if t == ExcitationType.VOLTAGE_FUN else float(v)
        sel = torch.nonzero(active).squeeze(1)
        points = torch.as_tensor(self.mesh.points, dtype=torch.float64, device=dev)
        lines = torch.as_tensor(self.mesh.lines.astype(np.int64), device=dev)
        return points[lines[sel]].contiguous(), types[sel].contiguous(), values[sel].contiguous()

    def get_electrostatic_active_elements(self):
        return self._get_active_elements('electrostatic')

    def get_magnetostatic_active_elements(self):
        return self._get_active_elements('magnetostatic')

    @staticmethod
    def _is_part_of_superposition(t):
        return t in (ExcitationType.VOLTAGE_FIXED, ExcitationType.VOLTAGE_FUN, ExcitationType.CURRENT,
                     ExcitationType.PERMANENT_MAGNET)

    def _split_for_superposition(self):
        """traceon/excitation.py:318-346"""
        types = self.excitation_types.items()
        parts = [(n, ExcitationType(t).is_electrostatic()) for n, (t, v) in types if self._is_part_of_superposition(t)]
        elec, mag = {}, {}
        for name, is_elec in parts:
            d = {}
            for n, (t, v) in types:
                if n == name or not self._is_part_of_superposition(t):
                    d[n] = (t, v)
                elif t == ExcitationType.VOLTAGE_FUN:
                    d[n] = (t, lambda *_: 0.0)
                else:
                    d[n] = (t, np.zeros_like(v) if isinstance(v, np.ndarray) else 0.0)
            exc = Excitation(self.mesh, self.symmetry)
            exc.excitation_types = d
            (elec if is_elec else mag)[name] = exc
        return elec, mag
