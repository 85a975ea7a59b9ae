"""BEM assembly and charge solve on the GPU, mirroring traceon/solver.py.

``solve_direct`` / ``solve_direct_superposition`` keep the reference's
interface (traceon/solver.py:364-431).  The matrix never leaves the device:

1. jacobian / position buffers (``tb_jacobian_buffer_radial``),
2. off-diagonal fill, 16-point Gauss sums per element pair
   (``tb_fill_matrix_radial``; reference fill_matrix_radial, radial.c:249-310),
3. singular diagonal (``tb_self_integrals``; the reference integrates it with
   SciPy QUADPACK one element at a time, solver.py:239-247),
4. FP64 LU with partial pivoting and triangular solves for all right-hand
   sides at once (``tb_lu_factor_perm`` / ``tb_lu_solve_perm``; reference
   numpy.linalg.solve, solver.py:173),
5. non-finite checks as the reference asserts (solver.py:146,175,251).
"""
from __future__ import annotations

import numpy as np

from . import backend as B
from .excitation import ExcitationType as ET
from .field import EffectivePointCharges, FieldRadialBEM


class SolverRadial:
    """Radial solver over the active elements of an excitation
    (traceon/solver.py:39-253)."""

    def __init__(self, excitation):
        self.excitation = excitation
        vertices, names = self.get_active_elements()
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.names = names
        N = len(self.vertices)
        types = np.zeros(N, dtype=np.uint8)
        values = np.zeros(N)
        self._dev = None
        self._centers = None
        for n, indices in names.items():
            t, v = excitation.excitation_types[n]
            types[indices] = int(t)
            if int(t) != int(ET.VOLTAGE_FUN):
                values[indices] = v
            else:
                values[indices] = self._voltage_function_values(v, np.atleast_1d(indices))
        self.excitation_types = types
        self.excitation_values = values
        self.jac_buffer, self.pos_buffer = (None, None)

    def _element_centers_device(self):
        """(N, 2) device tensor of the elements' collocation points (r, z) at
        alpha = 0 and (N, 2) normals (tb_element_targets)."""
        if self._centers is None:
            torch = B._torch()
            v = B.to_dev(self.vertices, torch.float64)
            self._centers = B.dev_element_targets(v)
        return self._centers

    def _voltage_function_values(self, fun, indices):
        """A VOLTAGE_FUN excitation at the centres of the given elements
        (traceon/solver.py:57-61 calls it once per element).  The centres are
        computed on the device, and the function is first called once on the
        device tensors x = r, y = 0, z, so that a function written with
        arithmetic and torch operations is evaluated on the GPU in one call;
        then once on NumPy arrays; a function that accepts neither (Python
        control flow on its arguments, math-module calls) is called per
        element as in the reference.  Returns a float64 array."""
        torch = B._torch()
        tgt, _ = self._element_centers_device()
        idx = torch.as_tensor(indices, dtype=torch.int64, device=tgt.device)
        r, z = tgt[idx, 0], tgt[idx, 1]
        n = len(indices)
        for args in ((r, torch.zeros_like(r), z), None):
            try:
                if args is None:
                    rn, zn = r.cpu().numpy(), z.cpu().numpy()
                    out = fun(rn, np.zeros_like(rn), zn)
                else:
                    out = fun(*args)
                if isinstance(out, torch.Tensor):
                    out = out.to(torch.float64).cpu().numpy()
                out = np.broadcast_to(np.asarray(out, dtype=np.float64), (n,)).copy()
                if np.all(np.isfinite(out)):
                    return out
            except Exception:
                pass
        c = tgt[idx].cpu().numpy()
        return np.array([fun(c[k, 0], 0.0, c[k, 1]) for k in range(n)], dtype=np.float64)

    # ---- device state
    def device(self):
        if self._dev is None:
            torch = B._torch()
            v = B.to_dev(self.vertices, torch.float64)
            t = B.to_dev(self.excitation_types, torch.uint8)
            val = B.to_dev(self.excitation_values, torch.float64)
            jac, pos = B.dev_jacobian_buffer(v)
            self._dev = (v, t, val, jac, pos)
        return self._dev

    def jacobians_and_positions(self):
        if self.jac_buffer is None:
            _, _, _, jac, pos = self.device()
            self.jac_buffer, self.pos_buffer = jac.cpu().numpy(), pos.cpu().numpy()
        return self.jac_buffer, self.pos_buffer

    def get_number_of_matrix_elements(self):
        return len(self.vertices)

    def get_center_of_element(self, index):
        jac, pos = B.position_and_jacobian_radial(0.0, *[self.vertices[index][i] for i in (0, 2, 3, 1)])
        return np.array([pos[0], 0.0, pos[1]])

    def get_normal_vectors(self):
        return np.array([B.higher_order_normal_radial(0.0, v) for v in self.vertices]).reshape(-1, 2)

    def get_preexisting_field(self, point):
        return np.zeros(3)

    def preexisting_field_device(self, centers):
        """Pre-existing field (N, 3) at the collocation points (r, 0, z) given
        as (N, 2) device tensor, or None when there is none."""
        return None

    def get_right_hand_side_device(self):
        """traceon/solver.py:118-150 on the device: voltage rows take their
        value, dielectric rows 0, magnetizable rows -factor(mu) H . n with the
        pre-existing field H at each element's collocation point, all in one
        launch (tb_rhs_radial_field).  Returns an (N,) device tensor."""
        torch = B._torch()
        v, t, val, _, _ = self.device()
        N = len(self.vertices)
        F = torch.empty(N, dtype=torch.float64, device=v.device)
        if N == 0:
            return F
        tgt, nrm = self._element_centers_device()
        field = self.preexisting_field_device(tgt) if (self.excitation_types == ET.MAGNETIZABLE).any() else None
        B._call('tb_rhs_radial_field', t.data_ptr(), val.data_ptr(), nrm.data_ptr(), B._ptr(field), F.data_ptr(), N,
                B._stream())
        return F

    def get_right_hand_side(self):
        """traceon/solver.py:118-150"""
        F = self.get_right_hand_side_device().cpu().numpy()
        assert np.all(np.isfinite(F))
        return F

    def get_matrix_device(self):
        """The full BEM matrix as an (N, N) FP64 device tensor."""
        torch = B._torch()
        pre = getattr(self, '_prefilled', None)
        if pre is not None:  # filled by solve_direct_batch
            self._prefilled = None
            return pre
        v, t, val, jac, pos = self.device()
        N = len(self.vertices)
        A = torch.empty((N, N), dtype=torch.float64, device=v.device)
        B.dev_fill_matrix(A, v, t, val, jac, pos)
        B.dev_self_integrals(v, t, val, A)
        return A

    def get_matrix(self):
        A = self.get_matrix_device().cpu().numpy()
        assert np.all(np.isfinite(A)), "Matrix contains non-finite values."
        return A

    def solve_charges_device(self, F, method='mixed'):
        """Charges (nrhs, N) device tensor for right-hand sides F (nrhs, N).

        method 'mixed': FP32 factors of the equilibrated matrix refined in
        FP64 against the FP64 matrix (tb_solve_mixed); falls back to 'lu' if
        refinement does not converge.  method 'lu': FP64 LU with partial
        pivoting, the factorisation of numpy.linalg.solve (solver.py:173)."""
        torch = B._torch()
        A = self.get_matrix_device()
        if not bool(torch.isfinite(A).all()):
            raise ValueError('Matrix contains non-finite values.')
        Ft = B.to_dev(np.atleast_2d(F), torch.float64)
        self.solve_info = {'method': method}
        if method == 'mixed' and Ft.shape[0] <= 16:
            try:
                X, iters, rel = B.dev_solve_mixed(A, Ft)
                self.solve_info.update(iterations=iters, last_correction=rel)
                return X
            except B.BackendError as e:
                self.solve_info.update(fallback=f'mixed refinement failed (status {getattr(e, "status", "?")})')
        ipiv, perm = B.dev_lu_factor(A)
        X = B.dev_lu_solve(A, perm, Ft)
        self.solve_info['method'] = 'lu'
        return X

    def solve_matrix(self, right_hand_side=None, method='mixed'):
        """traceon/solver.py:160-180"""
        F = np.array([self.get_right_hand_side()]) if right_hand_side is None else np.atleast_2d(right_hand_side)
        N = self.get_number_of_matrix_elements()
        if N == 0:
            return [self.charges_to_field(EffectivePointCharges.empty_2d()) for _ in range(len(F))]
        assert all(f.shape == (N,) for f in F)
        charges = self.solve_charges_device(F, method).cpu().numpy()
        assert np.all(np.isfinite(charges)) and charges.shape == F.shape, 'non-finite charges (singular matrix?)'
        jac, pos = self.jacobians_and_positions()
        return [self.charges_to_field(EffectivePointCharges(c, jac, pos)) for c in charges]


class ElectrostaticSolverRadial(SolverRadial):
    def get_active_elements(self):
        return self.excitation.get_electrostatic_active_elements()

    def charges_to_field(self, charges):
        return FieldRadialBEM(electrostatic_point_charges=charges)


class MagnetostaticSolverRadial(SolverRadial):
    """Magnetizable / magnetostatic-potential rows (traceon/solver.py:267-353).
    Pre-existing fields from current rings can be given as
    ``current_point_charges`` (an EffectivePointCharges of (N, 12, 3)
    positions); permanent magnets are not supported."""

    def __init__(self, excitation, current_point_charges=None):
        super().__init__(excitation)
        self.current_point_charges = current_point_charges if current_point_charges is not None \
            else EffectivePointCharges.empty_3d()
        self.preexisting_field = FieldRadialBEM(current_point_charges=self.current_point_charges)

    def get_active_elements(self):
        return self.excitation.get_magnetostatic_active_elements()

    def get_preexisting_field(self, point):
        return self.preexisting_field.magnetostatic_field_at_point(point)

    def preexisting_field_device(self, centers):
        """The current rings' field at all collocation points in one launch
        (tb_current_field_points)."""
        if not len(self.current_point_charges):
            return None
        torch = B._torch()
        pts = torch.zeros((centers.shape[0], 3), dtype=torch.float64, device=centers.device)
        pts[:, 0] = centers[:, 0]
        pts[:, 2] = centers[:, 1]
        return B.dev_current_field_points(pts, self.current_point_charges.device_sources())

    def charges_to_field(self, charges):
        return FieldRadialBEM(magnetostatic_point_charges=charges,
                              current_point_charges=self.current_point_charges)


def solve_direct_superposition(excitation):
    """One field per excited electrode from one factorisation
    (traceon/solver.py:364-400)."""
    elec, mag = excitation._split_for_superposition()
    out = {}
    if elec:
        names = list(elec.keys())
        F = np.array([ElectrostaticSolverRadial(elec[n]).get_right_hand_side() for n in names])
        for n, f in zip(names, ElectrostaticSolverRadial(excitation).solve_matrix(F)):
            out[n] = f
    if mag:
        names = list(mag.keys())
        F = np.array([MagnetostaticSolverRadial(mag[n]).get_right_hand_side() for n in names])
        for n, f in zip(names, MagnetostaticSolverRadial(excitation).solve_matrix(F)):
            out[n] = f
    return out


def solve_direct_batch(excitations, method='mixed'):
    """Electrostatic fields of many excitations (geometries of uneven N): all
    matrices are filled in one persistent launch (tb_fill_matrix_radial_batched)
    plus one launch for every self term, then each geometry's charges are
    solved on the device.  No counterpart in the reference, which solves one
    excitation at a time (traceon/solver.py:402-431); each result equals
    solve_direct(excitation)."""
    torch = B._torch()
    solvers = [ElectrostaticSolverRadial(e) for e in excitations]
    items = []
    for s_ in solvers:
        v, t, val, jac, pos = s_.device()
        N = len(s_.vertices)
        items.append((v, t, val, jac, pos, torch.empty((N, N), dtype=torch.float64, device=v.device)))
    B.dev_fill_batched(items)
    out = []
    for s_, item in zip(solvers, items):
        s_._prefilled = item[5]
        out.append(s_.solve_matrix(method=method)[0])
    return out


def solve_direct(excitation):
    """traceon/solver.py:402-431"""
    mag, elec = excitation.is_magnetostatic(), excitation.is_electrostatic()
    if mag and elec:
        return ElectrostaticSolverRadial(excitation).solve_matrix()[0] + \
            MagnetostaticSolverRadial(excitation).solve_matrix()[0]
    if elec:
        return ElectrostaticSolverRadial(excitation).solve_matrix()[0]
    if mag:
        return MagnetostaticSolverRadial(excitation).solve_matrix()[0]
    raise RuntimeError("Solving for an empty excitation")
