"""Failure paths of the kernels' bounded waits, made to run out on purpose
without faulting the GPU: the library's wait limit (tb_set_wait_limit) is cut
to one clock cycle, so that every progress wait that does not find its
condition met at the first poll gives up.  The kernels then drain the work
they have in flight, release their memory and report the failure: the mixed
solve returns TB_TIMEOUT, the tensor-core surrogate engine marks points and
particles with its timeout status.  Afterwards, with the default limit
restored, the same calls on the same CUDA context give correct results."""
import contextlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def wait_limit(cuda, cycles):
    prev = cuda.set_wait_limit(cycles)
    try:
        yield prev
    finally:
        cuda.set_wait_limit(prev)


def test_wait_limit_setter(cuda):
    prev = cuda.set_wait_limit(12345)
    assert cuda.set_wait_limit(0) == 12345  # 0 restores the default
    assert cuda.set_wait_limit(prev) == 2_000_000_000


def test_mixed_solve_times_out_and_recovers(cuda):
    """N = 4,096 (64 sweep blocks, tensor-core trailing updates): with a
    one-cycle limit the GEMM stages and the sweeps' waits for published
    blocks run out and tb_solve_mixed returns TB_TIMEOUT; with the default
    limit the same solve agrees with LAPACK."""
    import torch
    from traceon_b200.geometry import einzel_lens
    n = 4096
    geo = einzel_lens(n)
    v = cuda.to_dev(geo.vertices, torch.float64)
    t = cuda.to_dev(np.ones(n, np.uint8), torch.uint8)
    val = cuda.to_dev(np.zeros(n), torch.float64)
    jac, pos = cuda.dev_jacobian_buffer(v)
    A = torch.empty((n, n), dtype=torch.float64, device=v.device)
    cuda.dev_fill_matrix(A, v, t, val, jac, pos)
    cuda.dev_self_integrals(v, t, val, A)
    F = torch.as_tensor(geo.unit_rhs(), device='cuda')
    with wait_limit(cuda, 1):
        with pytest.raises(cuda.BackendError) as e:
            cuda.dev_solve_mixed(A, F)
        assert e.value.status == cuda.TB_TIMEOUT
    torch.cuda.synchronize()  # the context is still usable
    X, iters, rel = cuda.dev_solve_mixed(A, F)
    X_ref = np.linalg.solve(A.cpu().numpy(), geo.unit_rhs().T).T
    err = max(np.abs(X.cpu().numpy()[k] - X_ref[k]).max() / np.abs(X_ref[k]).max() for k in range(3))
    assert err < 1e-10


@pytest.fixture(scope='module')
def untrained_surrogate():
    """A surrogate field with an untrained network: enough to exercise the
    tensor-core engine's waits (accuracy is not the point here)."""
    from traceon_b200 import geometry as G
    from traceon_b200.surrogate import SurrogateTrainer, SurrogateModel, FieldSurrogate
    geo = G.einzel_lens(120)
    tr = SurrogateTrainer(geo, nz=401)
    model = SurrogateModel(3, tr.r_max, tr.z_lo, tr.z_hi, np.full(32, 1e-3), tr.env_power, seed=0)
    return FieldSurrogate(model, tr.fields, tr.z, tr.tabs, np.array([0.0, 1000.0, 0.0]), geo.segments, engine='tc')


def test_surrogate_engine_times_out_and_recovers(cuda, untrained_surrogate):
    """Field points: with a one-cycle limit the MMA-chain waits run out and
    the points report used_bem = -1 (NaN field); tracing: the particles end
    with TB_TRACE_ENGINE_TIMEOUT, every one of them with a defined status and
    no particle beyond its start-state row.  With the default limit both
    calls complete normally."""
    from traceon_b200 import geometry as G
    fs = untrained_surrogate
    rng = np.random.default_rng(3)
    n = 1000
    pts = np.stack([rng.uniform(0.0, 0.8e-3, n), np.zeros(n), rng.uniform(-9e-3, 9e-3, n)], 1)
    with wait_limit(cuda, 1):
        E_t, used_t = fs.kernel_field_at_points(pts)
        p0, v0 = G.surrogate_beam(700, 5)
        plane, final, status, counters = fs.trace_endpoints(p0, v0, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
    assert (used_t == -1).any()
    assert np.isnan(E_t[used_t == -1]).all()
    assert set(np.unique(status)) <= {cuda.TRACE_EXITED, cuda.TRACE_ENGINE_TIMEOUT}
    assert (status == cuda.TRACE_ENGINE_TIMEOUT).any()
    untraced = (status == cuda.TRACE_ENGINE_TIMEOUT) & (counters[:, 1] == 0)
    assert np.array_equal(final[untraced, 1:4], p0[untraced])
    E, used = fs.kernel_field_at_points(pts)
    assert (used >= 0).all() and np.isfinite(E).all()
    plane, final, status, counters = fs.trace_endpoints(p0, v0, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
    assert (status == cuda.TRACE_EXITED).all()
