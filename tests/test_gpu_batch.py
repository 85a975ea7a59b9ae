"""Batched fill of geometries of uneven N (the batching workload's lenses):
one persistent launch for every off-diagonal entry and one for every self
term give exactly the single-geometry fills, and solve_direct_batch gives
the oracle's charges; excitations assembled on the device match the host
assembly."""
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


def test_trace_geometries_equals_single_traces(cuda):
    """Particles of several geometries traced in one launch (each particle
    sums only its own geometry's rings) give exactly the endpoints of tracing
    each geometry on its own with the same team size; uneven particle counts
    per geometry."""
    from traceon_b200.solver import solve_direct_batch
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.geometry import random_lens
    from traceon_b200.tracing import Tracer, trace_geometries, velocity_vec_xz_plane
    lenses = [random_lens(s, n_range=(100, 400)) for s in (7, 8, 9)]
    excs = []
    for geo, volts in lenses:
        exc = Excitation(Mesh.from_geometry(geo))
        exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, volts)})
        excs.append(exc)
    fields = solve_direct_batch(excs)
    bounds = np.array([[-0.4e-3, 0.4e-3], [-0.4e-3, 0.4e-3], [-16e-3, 16e-3]])
    rng = np.random.default_rng(5)
    pos, vel = [], []
    for count in (24, 17, 31):
        r0 = rng.uniform(0, 0.1e-3, count)
        pos.append(np.stack([r0, np.zeros(count), np.full(count, -15e-3)], 1))
        vel.append(np.array([velocity_vec_xz_plane(1000.0, a, downward=False) for a in rng.uniform(-5e-3, 5e-3, count)]))
    batched = trace_geometries(fields, bounds, pos, vel, 15e-3, atol=1e-9, team_warps=2)
    for f, p, v, got in zip(fields, pos, vel, batched):
        want = Tracer(f, bounds).trace_endpoints(p, v, 15e-3, atol=1e-9, team_warps=2)
        for a, b in zip(got, want):
            assert np.array_equal(np.nan_to_num(a, nan=7.0), np.nan_to_num(b, nan=7.0))
        assert (want[2] == cuda.TRACE_EXITED).all()
    # each particle sees its own geometry: the same start states through two
    # geometries in one launch end differently
    same = trace_geometries(fields[:2], bounds, [pos[0], pos[0]], [vel[0], vel[0]], 15e-3, atol=1e-9, team_warps=2)
    assert np.array_equal(same[0][1], batched[0][1])
    assert not np.array_equal(same[0][1], same[1][1])


def test_graded_mesh_on_device(cuda):
    """Graded cubic meshes generated on the GPU (tb_mesh_segments) against the
    host mesher (geometry.polyline_elements): the einzel lens and three
    batching lenses from their segments and element counts, and segments
    with zero elements.  The GPU's cosine may differ from the host's in the
    last bit, which the 16-bit mantissa truncation almost always removes: at
    most one truncation step (2^-36 relative) anywhere."""
    from traceon_b200 import geometry as G
    geos = [G.einzel_lens(1000)] + [G.random_lens(s)[0] for s in range(3)]
    for geo in geos:
        v = geo.vertices_device().cpu().numpy()
        assert v.shape == geo.vertices.shape
        d = np.abs(v - geo.vertices)
        assert d.max() <= 2.0 ** -35 * np.abs(geo.vertices).max()
        assert (d > 0).mean() < 0.01
        assert np.array_equal(v[:, :, 1], np.zeros_like(v[:, :, 1]))
    seg = np.array([[1e-3, -2e-3, 1e-3, 2e-3], [1e-3, 2e-3, 2e-3, 2e-3], [2e-3, 2e-3, 2e-3, 3e-3]])
    v = G.mesh_segments_device(seg, [5, 0, 3]).cpu().numpy()
    host = np.concatenate([G.polyline_elements([seg[0, :2], seg[0, 2:]], [5]),
                           G.polyline_elements([seg[2, :2], seg[2, 2:]], [3])])
    assert np.max(np.abs(v - host)) <= 2.0 ** -35 * 3e-3
    with pytest.raises(ValueError):
        G.mesh_segments_device(seg, [5, 0])


def test_excitation_assembled_on_device(cuda):
    """Excitation.assemble_device gives the host solver's active elements,
    types and values (a voltage group, a dielectric group, a function group
    and an inactive group)."""
    from traceon_b200.excitation import Excitation, Mesh, ExcitationType as ET
    from traceon_b200.geometry import random_lens
    from traceon_b200.solver import ElectrostaticSolverRadial
    geo, volts = random_lens(11, n_range=(400, 400), tubes_range=(4, 4))
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{geo.names[0]: 100.0, geo.names[1]: lambda x, y, z: 3.0 + 0 * z})
    exc.add_dielectric(**{geo.names[2]: 4.0})
    verts, types, values = exc.assemble_device('electrostatic')
    s = ElectrostaticSolverRadial(exc)
    assert np.array_equal(verts.cpu().numpy(), s.vertices)
    assert np.array_equal(types.cpu().numpy(), s.excitation_types)
    v, ref = values.cpu().numpy(), s.excitation_values
    fun = s.excitation_types == int(ET.VOLTAGE_FUN)
    assert fun.any() and np.isnan(v[fun]).all() and np.array_equal(v[~fun], ref[~fun])
