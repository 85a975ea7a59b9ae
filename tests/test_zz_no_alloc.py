"""tb_lu_solve_noalloc: the dense charge solve for callers that cannot
allocate device memory (a plug-in in an application that owns the GPU's
memory pool, a control loop that may not allocate after start-up).  Its
pivots live in a static device array of the library, shared by all calls.

Checked through the C ABI against the allocating entry points
(tb_lu_factor_perm + tb_lu_solve_perm), within the charge tolerance of the
parity suite (1e-10 relative to max |charge|), on two calls in a row so that
contents left in the shared array by the first call cannot leak into the
second.  Kept in its own file so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from traceon_b200 import build
    lib = C.CDLL(build.LIB)
    f = lib.tb_lu_solve_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64,
                  C.c_void_p]
    return f


def _system(cuda, n, volts):
    import torch
    from traceon_b200.geometry import einzel_lens
    geo = einzel_lens(n)
    v = cuda.to_dev(geo.vertices, torch.float64)
    t = cuda.to_dev(np.ones(n, np.uint8), torch.uint8)
    val = cuda.to_dev(geo.voltages_to_values(np.asarray(volts)), torch.float64)
    jac, pos = cuda.dev_jacobian_buffer(v)
    A = torch.empty((n, n), dtype=torch.float64, device=v.device)
    cuda.dev_fill_matrix(A, v, t, val, jac, pos)
    cuda.dev_self_integrals(v, t, val, A)
    F = torch.as_tensor(np.vstack([geo.voltages_to_values(np.asarray(volts)), geo.unit_rhs()]),
                        device=v.device).contiguous()
    return A, F


def _reference_solution(cuda, A, F):
    LU = A.clone()
    _, perm = cuda.dev_lu_factor(LU)
    return cuda.dev_lu_solve(LU, perm, F).cpu().numpy()


def test_noalloc_solve_matches_allocating_solve(cuda):
    """Two calls in a row (a larger system, then a smaller one, so that the
    second runs over pivots the first left in the shared array) against the
    allocating entry points; the device's free memory (cudaMemGetInfo) is the
    same before and after the two calls.  A first call on a throw-away system
    loads the library's kernels beforehand, because loading a module on
    first use takes device memory itself."""
    import torch
    solve = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = []
    for n, volts in ((517, (0.0, 1500.0, 0.0)), (300, (-200.0, 900.0, 100.0))):
        A, F = _system(cuda, n, volts)
        cases.append((n, A, F, _reference_solution(cuda, A, F), A.clone(), torch.empty_like(F)))
    n, A, F, _, _, _ = cases[1]
    warm_lu, warm_x = A.clone(), torch.empty_like(F)
    assert solve(warm_lu.data_ptr(), n, n, F.data_ptr(), n, warm_x.data_ptr(), n, F.shape[0], stream) == cuda.TB_OK
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for n, A, F, expected, LU, X in cases:
        rc = solve(LU.data_ptr(), n, n, F.data_ptr(), n, X.data_ptr(), n, F.shape[0], stream)
        assert rc == cuda.TB_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    for n, A, F, expected, LU, X in cases:
        got = X.cpu().numpy()
        for k in range(F.shape[0]):
            scale = np.abs(expected[k]).max()
            assert np.max(np.abs(got[k] - expected[k])) / scale < 1e-10, (n, k)


def test_noalloc_rejects_oversized_systems(cuda):
    import torch
    solve = _lib()
    n = 32769
    stream = torch.cuda.current_stream().cuda_stream
    # rejected before any device memory is touched
    assert solve(None, n, n, None, n, None, n, 1, stream) == cuda.TB_BAD_ARG
