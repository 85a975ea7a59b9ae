"""The charge solve on the GPU: FP64 LU with partial pivoting (the reference's
numpy.linalg.solve, solver.py:173), LU without pivoting, and the mixed
solve (FP32 factors + FP64 refinement) -- all against LAPACK on the same
FP64 matrix.  Tolerance: 1e-10 relative to max |charge|, the contract of
the charge solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrix(cuda, n):
    import torch
    from traceon_b200.geometry import einzel_lens
    geo = einzel_lens(n)
    v = cuda.to_dev(geo.vertices, torch.float64)
    t = cuda.to_dev(np.ones(n, np.uint8), torch.uint8)
    val = cuda.to_dev(np.zeros(n), torch.float64)
    jac, pos = cuda.dev_jacobian_buffer(v)
    A = torch.empty((n, n), dtype=torch.float64, device=v.device)
    cuda.dev_fill_matrix(A, v, t, val, jac, pos)
    cuda.dev_self_integrals(v, t, val, A)
    rng = np.random.default_rng(n)
    F = np.vstack([geo.unit_rhs(), geo.voltages_to_values(rng.uniform(-3000, 3000, (5, 3)).T).T])
    return A, F


def _close(X, X_ref):
    return max(np.max(np.abs(X[k] - X_ref[k])) / np.abs(X_ref[k]).max() for k in range(len(X_ref)))


@pytest.mark.parametrize('n', [300, 1000, 2500])
def test_solvers_agree_with_lapack(cuda, n):
    import torch
    A, F = _matrix(cuda, n)
    A_h = A.cpu().numpy()
    X_ref = np.linalg.solve(A_h, F.T).T
    Ft = torch.as_tensor(F, device='cuda')
    # pivoted FP64
    LU = A.clone()
    _, perm = cuda.dev_lu_factor(LU)
    assert _close(cuda.dev_lu_solve(LU, perm, Ft).cpu().numpy(), X_ref) < 1e-10
    # unpivoted FP64: factors reproduce A, solution agrees
    LU = A.clone()
    cuda.dev_lu_nopiv(LU)
    L = np.tril(LU.cpu().numpy(), -1) + np.eye(n)
    U = np.triu(LU.cpu().numpy())
    assert np.abs(L @ U - A_h).max() < 1e-12 * np.abs(A_h).max()
    X_np = np.linalg.solve(U, np.linalg.solve(L, F.T)).T
    assert _close(X_np, X_ref) < 1e-10
    # mixed precision
    X, iters, rel = cuda.dev_solve_mixed(A, Ft)
    assert iters <= 8 and rel <= 1e-12
    assert _close(X.cpu().numpy(), X_ref) < 1e-10


@pytest.mark.parametrize('reserve', [0, 8, 40])
def test_mixed_solve_lookahead_same_factors(cuda, reserve):
    """Lookahead (the rest of each trailing update on a second stream beside
    the next panel's factorisation; on by default) or none: the mixed solve
    returns the same charges, bit for bit, on 3,000 elements (12 panels)."""
    import torch
    A, F = _matrix(cuda, 3000)
    Ft = torch.as_tensor(F, device='cuda')
    X0, it0, _ = cuda.dev_solve_mixed(A, Ft)
    old = cuda.set_solve_lookahead(reserve)
    try:
        X1, it1, _ = cuda.dev_solve_mixed(A, Ft)
    finally:
        cuda.set_solve_lookahead(old)
    assert it1 == it0 and torch.equal(X0, X1)


def test_lookahead_tuner_sets_a_candidate(cuda):
    """autotune.tune_solve_lookahead times every candidate width on the
    matrix, leaves the fastest set, reuses it from its table for the same
    size bucket, and the tuned solve gives the default's charges bit for
    bit."""
    import torch
    from traceon_b200 import autotune
    A, F = _matrix(cuda, 3000)
    Ft = torch.as_tensor(F, device='cuda')
    X0, _, _ = cuda.dev_solve_mixed(A, Ft)
    old = cuda.set_solve_lookahead(-1)
    autotune.clear()
    try:
        hit = autotune.tune_solve_lookahead(A, Ft)
        sms = cuda.num_sms()
        cands = {int(round(f * sms)) for f in autotune.LOOKAHEAD_FRACTIONS}
        assert set(hit['times_ms']) == cands and hit['reserve_sms'] in cands
        assert hit['times_ms'][hit['reserve_sms']] == min(hit['times_ms'].values())
        assert cuda.set_solve_lookahead(hit['reserve_sms']) == hit['reserve_sms']
        assert autotune.tune_solve_lookahead(A, Ft) is not None and len(autotune.table()) == 1
        X1, _, _ = cuda.dev_solve_mixed(A, Ft)
        assert torch.equal(X0, X1)
    finally:
        cuda.set_solve_lookahead(old)
        autotune.clear()


@pytest.mark.parametrize('nrhs', [1, 9, 16])
def test_mixed_solve_right_hand_side_counts(cuda, nrhs):
    """1, 9 and 16 (the maximum) right-hand sides against LAPACK on a
    1,100-element matrix (the last sweep block partial); 17 are refused."""
    import torch
    A, F = _matrix(cuda, 1100)
    rng = np.random.default_rng(nrhs)
    F = np.vstack([F, rng.normal(size=(16, 1100))])[:nrhs]
    X_ref = np.linalg.solve(A.cpu().numpy(), F.T).T
    X, iters, rel = cuda.dev_solve_mixed(A, torch.as_tensor(F, device='cuda'))
    assert iters <= 8 and rel <= 1e-12
    assert _close(X.cpu().numpy(), X_ref) < 1e-10
    with pytest.raises(cuda.BackendError):
        cuda.dev_solve_mixed(A, torch.as_tensor(np.vstack([F] * 17)[:17], device='cuda'))


def test_mixed_solve_reports_failure_and_solver_falls_back(cuda):
    """A system that needs pivoting (zero diagonal): the unpivoted mixed
    solve reports failure, and the solver then uses the pivoted FP64 LU."""
    import torch
    rng = np.random.default_rng(1)
    n = 200
    A_h = rng.normal(size=(n, n))
    A_h[np.arange(0, n, 7), np.arange(0, n, 7)] = 0.0
    A = torch.as_tensor(A_h, device='cuda')
    F = torch.as_tensor(rng.normal(size=(2, n)), device='cuda')
    with pytest.raises(cuda.BackendError):
        cuda.dev_solve_mixed(A, F, max_iter=6)
    from traceon_b200.solver import SolverRadial

    class Fixed(SolverRadial):
        def __init__(self):
            self.excitation_types = np.ones(n, np.uint8)
            self.vertices = np.zeros((n, 4, 3))

        def get_matrix_device(self):
            return A.clone()

    s = Fixed()
    X = s.solve_charges_device(F.cpu().numpy(), method='mixed').cpu().numpy()
    assert s.solve_info['method'] == 'lu' and 'fallback' in s.solve_info
    assert _close(X, np.linalg.solve(A_h, F.cpu().numpy().T).T) < 1e-10


@pytest.mark.parametrize('presplit', [False, True])
@pytest.mark.parametrize('M,N,K', [(128, 256, 32), (300, 500, 256), (1000, 700, 100), (37, 9, 5),
                                   (4100, 4000, 256)])  # the last: several tiles per CTA of the persistent kernel
def test_gemm_tf32x3_vs_fp64(cuda, M, N, K, presplit):
    """The tensor-core update C -= A B (tcgen05, 3xTF32) against FP64 numpy,
    on strided sub-matrices with sizes that are not multiples of the 128 x 256
    tile or the 32-wide K chunk: FP32-level accuracy."""
    import torch
    rng = np.random.default_rng(M + N + K)
    big_a = rng.normal(size=(M + 3, K + 5)).astype(np.float32)
    big_b = rng.normal(size=(K + 2, N + 7)).astype(np.float32)
    big_c = rng.normal(size=(M + 1, N + 3)).astype(np.float32)
    At = torch.as_tensor(big_a, device='cuda')[1:M + 1, 2:K + 2]
    Bt = torch.as_tensor(big_b, device='cuda')[1:K + 1, 3:N + 3]
    Ct = torch.as_tensor(big_c, device='cuda')
    cuda.dev_gemm_sub_tf32x3(Ct[1:M + 1, 1:N + 1], At, Bt, presplit=presplit)
    out = Ct.cpu().numpy().astype(np.float64)
    ref = big_c.astype(np.float64)
    ref[1:M + 1, 1:N + 1] -= big_a[1:M + 1, 2:K + 2].astype(np.float64) @ big_b[1:K + 1, 3:N + 3].astype(np.float64)
    scale = np.abs(big_a[1:M + 1, 2:K + 2]).astype(np.float64) @ np.abs(big_b[1:K + 1, 3:N + 3]).astype(np.float64)
    inner = np.abs(out[1:M + 1, 1:N + 1] - ref[1:M + 1, 1:N + 1]) / (scale + 1.0)
    assert inner.max() < 1e-5
    # everything outside the sub-matrix untouched
    mask = np.ones_like(out, dtype=bool)
    mask[1:M + 1, 1:N + 1] = False
    assert np.array_equal(out[mask], ref[mask])


@pytest.mark.parametrize('n', [700, 1000])
def test_lu_nopiv_tc_factors(cuda, n):
    """The FP32 LU of the mixed solve (256-column panels, tensor-core
    updates): on BEM matrices of 700 elements (three
    panels, the last partial, 700 = 10 x 64 + 60) and 1,000 elements, L U
    reproduces the column-equilibrated FP32 matrix to FP32 accuracy."""
    import torch
    A, F = _matrix(cuda, n)
    A_h = A.cpu().numpy()
    c = 1.0 / np.abs(A_h).max(axis=0)
    S_h = (A_h * c).astype(np.float32)
    S = torch.as_tensor(S_h, device='cuda')
    cuda.dev_lu_nopiv_tc(S)
    LU = S.cpu().numpy().astype(np.float64)
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    assert np.abs(L @ U - S_h).max() < 2e-5 * np.abs(S_h).max()
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    with pytest.raises(cuda.BackendError):  # the workspace is required
        cuda._call('tb_lu_nopiv_f32_tc', S.data_ptr(), n, n, None, 0, err.data_ptr(), cuda._stream())


def test_mixed_solve_with_dielectric_rows(cuda, port):
    """Flux (dielectric) rows in the matrix: the default mixed solve either
    converges or falls back to the pivoted FP64 LU -- either way the charges
    match LAPACK on the oracle's matrix to 1e-10."""
    from traceon_b200 import geometry as G
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.solver import ElectrostaticSolverRadial
    geo = G.einzel_lens(600)
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(ground_in=0.0, ground_out=800.0)
    exc.add_dielectric(lens=4.0)
    s = ElectrostaticSolverRadial(exc)
    F = np.array([s.get_right_hand_side()])
    X = s.solve_charges_device(F).cpu().numpy()[0]
    A = port.matrix(s.vertices, s.excitation_types, s.excitation_values, threads=8)
    q = np.linalg.solve(A, F[0])
    assert s.solve_info['method'] in ('mixed', 'lu')
    assert np.max(np.abs(X - q)) / np.max(np.abs(q)) < 1e-10


def test_magnetostatic_solve_with_current_rings(cuda, port):
    """MagnetostaticSolverRadial (solver.py:267-353): a magnetizable tube
    (mu_r = 1000) in the field of coil current rings.  The right-hand side
    -factor(mu) H_coil . n (solver.py:128-144) and the charges against the
    oracle: coil field by the oracle's current_field_radial, matrix by the
    oracle's fill of the flux rows, LAPACK solve."""
    from traceon_b200 import geometry as G
    from traceon_b200 import backend as B
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.field import EffectivePointCharges
    from traceon_b200.solver import MagnetostaticSolverRadial
    from test_oracle import _coil_rings
    geo = G.einzel_lens(300)
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_magnetizable(lens=1000.0)
    I, jac, pos = _coil_rings(7, n=30)
    s = MagnetostaticSolverRadial(exc, current_point_charges=EffectivePointCharges(I, jac, pos))
    F = s.get_right_hand_side()
    normals = s.get_normal_vectors()
    F_or = np.zeros(len(F))
    for i in range(len(F)):
        H = port.current_field_radial(s.get_center_of_element(i), I, jac, pos)
        F_or[i] = -B.flux_density_to_charge_factor(s.excitation_values[i]) * (H[0] * normals[i][0] + H[2] * normals[i][1])
    assert np.max(np.abs(F - F_or)) < 1e-11 * np.max(np.abs(F_or))
    field = s.solve_matrix()[0]
    A = port.matrix(s.vertices, s.excitation_types, s.excitation_values, threads=8)
    q = np.linalg.solve(A, F_or)
    got = field.magnetostatic_point_charges.charges
    assert np.max(np.abs(got - q)) / np.max(np.abs(q)) < 1e-10


def test_voltage_function_rows(cuda, port):
    """VOLTAGE_FUN excitations (traceon/solver.py:57-61): the function is
    evaluated at the element centres computed on the device -- once on
    device tensors (arithmetic / torch operations), once on NumPy arrays
    (NumPy functions), or per element (Python control flow) -- and the
    values equal the reference's per-element calls at the host-computed
    centres.  The charges of the resulting system agree with LAPACK on the
    oracle's matrix to 1e-10."""
    import math
    from traceon_b200 import geometry as G
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.solver import ElectrostaticSolverRadial
    geo = G.einzel_lens(600)
    funs = {'ground_in': lambda x, y, z: 100.0 + 2.0e5 * z + 3.0e7 * x * x,        # device tensors
            'lens': lambda x, y, z: 900.0 + 50.0 * np.cos(1e3 * z),                # NumPy arrays
            'ground_out': lambda x, y, z: -200.0 if z > 3e-3 else math.sin(1e3 * z)}  # per element
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**funs)
    s = ElectrostaticSolverRadial(exc)
    for name, idx in s.names.items():
        want = np.array([funs[name](*s.get_center_of_element(i)) for i in np.atleast_1d(idx)])
        got = s.excitation_values[idx]
        assert np.allclose(got, want, rtol=1e-13, atol=1e-12 * np.abs(want).max()), name
    F = s.get_right_hand_side()
    assert np.array_equal(F, s.excitation_values)
    field = s.solve_matrix()[0]
    A = port.matrix(s.vertices, s.excitation_types, s.excitation_values, threads=8)
    q = np.linalg.solve(A, F)
    got = field.electrostatic_point_charges.charges
    assert np.max(np.abs(got - q)) / np.max(np.abs(q)) < 1e-10


def test_dielectric_rows_at_scale(cuda, port):
    """Flux (dielectric) rows at N = 4,002 (the middle electrode a
    dielectric of permittivity 4): the GPU fill of the flux rows against the
    oracle's fill of the same matrix (row sample, 1e-12 of the largest
    entry); the GPU solve against LAPACK on the GPU-filled matrix (1e-10);
    and the charges against LAPACK on the oracle's matrix within what the
    matrix agreement allows for this system's condition number (flux rows
    make it far less well conditioned than voltage rows alone)."""
    from traceon_b200 import geometry as G
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.solver import ElectrostaticSolverRadial
    geo = G.einzel_lens(4002)
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(ground_in=0.0, ground_out=800.0)
    exc.add_dielectric(lens=4.0)
    s = ElectrostaticSolverRadial(exc)
    A_gpu = s.get_matrix()
    A = port.matrix(s.vertices, s.excitation_types, s.excitation_values, threads=16)
    flux = np.nonzero(s.excitation_types == 3)[0]
    assert len(flux) > 1000
    rows = np.concatenate([flux[::97], np.nonzero(s.excitation_types == 1)[0][::211]])
    assert np.max(np.abs(A_gpu[rows] - A[rows])) <= 1e-12 * np.max(np.abs(A))
    F = s.get_right_hand_side()
    X = s.solve_charges_device(np.array([F])).cpu().numpy()[0]
    # FP64 solves of this system agree only to about cond(A) x 1e-16 (far
    # looser than the charge tolerance of the voltage-row systems)
    cond = np.linalg.cond(A_gpu)
    q_same = np.linalg.solve(A_gpu, F)
    assert np.max(np.abs(X - q_same)) / np.max(np.abs(q_same)) < max(1e-10, 10 * cond * 1e-16)
    q = np.linalg.solve(A, F)
    assert np.max(np.abs(X - q)) / np.max(np.abs(q)) < 10 * cond * 1e-12
