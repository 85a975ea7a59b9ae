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
