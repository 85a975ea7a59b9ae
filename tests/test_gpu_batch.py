"""Batched fill of geometries of uneven N (the batching workload's lenses):
one persistent launch for every off-diagonal entry and one for every self
term give exactly the single-geometry fills, and solve_direct_batch gives
the oracle's charges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lenses():
    from traceon_b200.geometry import random_lens
    return [random_lens(s, n_range=(64, 1200)) for s in range(5)]


def test_batched_fill_equals_single_fills(cuda):
    import torch
    items, singles = [], []
    for geo, _ in _lenses():
        n = len(geo)
        v = cuda.to_dev(geo.vertices, torch.float64)
        t = cuda.to_dev(np.ones(n, np.uint8), torch.uint8)
        val = cuda.to_dev(np.zeros(n), torch.float64)
        jac, pos = cuda.dev_jacobian_buffer(v)
        A = torch.full((n, n), float('nan'), dtype=torch.float64, device='cuda')
        items.append((v, t, val, jac, pos, A))
        S = torch.empty((n, n), dtype=torch.float64, device='cuda')
        cuda.dev_fill_matrix(S, v, t, val, jac, pos)
        cuda.dev_self_integrals(v, t, val, S)
        singles.append(S)
    cuda.dev_fill_batched(items)
    for (_, _, _, _, _, A), S in zip(items, singles):
        assert torch.equal(A, S)


def test_solve_direct_batch_vs_oracle(cuda, port):
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.solver import solve_direct_batch
    lenses = _lenses()
    excs = []
    for geo, volts in lenses:
        exc = Excitation(Mesh.from_geometry(geo))
        exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, volts)})
        excs.append(exc)
    fields = solve_direct_batch(excs)
    for (geo, volts), f in list(zip(lenses, fields))[:3]:
        values = geo.voltages_to_values(volts)
        A = port.matrix(geo.vertices, np.ones(len(geo), np.uint8), values, threads=8)
        q = np.linalg.solve(A, values)
        got = f.electrostatic_point_charges.charges
        assert np.max(np.abs(got - q)) / np.max(np.abs(q)) < 1e-10
