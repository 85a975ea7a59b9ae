"""Device math of the ring-pair loops against the CUDA library functions
(tb_probe_math of the test library tests/probe): the branch-free reciprocal, reciprocal square root and
logarithm of tb_fastmath.cuh stay within a few ulp over the argument ranges
the loops produce."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probe(cuda, x, fn):
    import torch
    xt = torch.as_tensor(x, device='cuda', dtype=torch.float64)
    out = torch.empty_like(xt)
    from conftest import load_probe
    rc = load_probe().tb_probe_math(xt.data_ptr(), xt.numel(), fn, out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    return out.cpu().numpy()


def _ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


@pytest.mark.parametrize('fn, lo, hi', [(0, -60, 30), (1, -60, 30)])
def test_reciprocals(cuda, fn, lo, hi):
    rng = np.random.default_rng(fn)
    x = 10.0 ** rng.uniform(lo, hi, 200000)
    mine, lib = _probe(cuda, x, fn), _probe(cuda, x, fn + 10)
    assert np.max(_ulps(mine, lib)) <= 2


def test_log(cuda):
    rng = np.random.default_rng(3)
    # t = rho^2 / D of a ring pair lies in (0, 1]; include values near 1
    x = np.concatenate([10.0 ** rng.uniform(-300, 0, 100000), 1 - 10.0 ** rng.uniform(-16, -1, 50000),
                        rng.uniform(0.5, 1.0, 50000), [1.0, 0.5, 2.0 ** -600]])
    mine, lib = _probe(cuda, x, 2), _probe(cuda, x, 12)
    err = np.abs(mine - lib)
    # absolute error in units of the result's ulp, or relative to 1 near t = 1
    assert np.max(err / np.maximum(np.spacing(np.abs(lib)), 1e-300)) <= 4
    assert np.all(mine[x == 1.0] == 0.0)
