"""Trajectory post-processing on the device: plane crossings of stored
trajectories (traceon/backend/tracing.c:184-223) and the least-squares
focus (traceon/focus.py:9-42), against the oracle (the C restatement of
plane_intersection, numpy lstsq for the focus)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _traced_rows(max_rows=4096):
    """The golden lens's particles and 29 more (r0 U[0, 0.15] mm in the
    xz-plane, angles U[-5, 5] mrad, 1 keV), traced through the golden lens
    field with their trajectories stored on the device."""
    from traceon_b200 import backend as B
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.tracing import Tracer, velocity_vec_xz_plane, m_e, e
    g = golden('lens96.npz')
    rng = np.random.default_rng(11)
    p0 = np.concatenate([g['p0'], np.stack([rng.uniform(0, 1.5e-4, 29), np.zeros(29), np.full(29, -9.5e-3)], 1)])
    v0 = np.concatenate([g['v0'], [velocity_vec_xz_plane(1000.0, a, downward=False)
                                   for a in rng.uniform(-5e-3, 5e-3, 29)]])
    f = FieldRadialBEM(EffectivePointCharges(g['charges'], g['jac'], g['pos']))
    tr = Tracer(f, g['bounds'])
    start, qm = tr._start(p0, v0, m_e, -e)
    res = tr.trace_device(start, qm, atol=1e-10, max_rows=max_rows)
    assert np.all(res.status.cpu().numpy() == B.TRACE_EXITED)
    return g, res


def test_plane_intersections_match_oracle(cuda, port):
    g, res = _traced_rows()
    rows = res.rows.cpu().numpy()
    nrows = res.nrows.cpu().numpy()
    planes = [([0, 0, 9.5e-3], [0, 0, 1]), ([0, 0, 0.0], [0, 0, 1]), ([0, 0, 1e-3], [0.3, 0.1, 1.0]),
              ([0, 0, -2e-3], [0, 0, -2.0])]
    for p0, nv in planes:
        out, found = res.plane_intersection(p0, nv)
        out, found = out.cpu().numpy(), found.cpu().numpy()
        for k in range(len(rows)):
            s = rows[k, :nrows[k], 1:]
            try:
                want = port.plane_intersection(s, p0, nv)
            except ValueError:
                assert not found[k] and np.all(np.isnan(out[k]))
                continue
            assert found[k]
            # the same weights on the same rows; only FMA contraction differs
            assert np.max(np.abs(out[k, 1:4] - want[:3])) < 1e-15 + 1e-13 * np.max(np.abs(want[:3]))
            assert np.max(np.abs(out[k, 4:] - want[3:])) < 1e-13 * np.max(np.abs(want[3:]))
            # t is interpolated with the same weights
            t = rows[k, :nrows[k], 0]
            assert t[0] <= out[k, 0] <= t[-1]


def test_plane_intersection_none_and_edges(cuda, port):
    """No crossing -> found False and NaN (the reference raises ValueError);
    one-row trajectories have no pair to test."""
    import torch
    g, res = _traced_rows()
    out, found = res.plane_intersection([0, 0, 1.0], [0, 0, 1])  # far outside the bounds
    assert not found.any().item() and torch.isnan(out).all().item()
    one = res.nrows.clone()
    one[:] = 1
    out, found = cuda.dev_plane_intersection_rows(res.rows, one, [0, 0, 9.5e-3], [0, 0, 1])
    assert not found.any().item()
    with pytest.raises(cuda.BackendError):
        cuda.dev_plane_intersection_rows(res.rows, res.nrows, [0, 0, 0], [0, 0, 0])


def test_axis_intersection(cuda, port):
    """Electrons launched off axis in the xz-plane, focused back through
    x = 0: the z of the crossing nearest the end, as axis_intersection."""
    import torch
    g, res = _traced_rows()
    z = res.axis_intersection().cpu().numpy()
    rows, nrows = res.rows.cpu().numpy(), res.nrows.cpu().numpy()
    for k in range(len(rows)):
        s = rows[k, :nrows[k], 1:]
        try:
            want = port.plane_intersection(s, [0, 0, 0], [1, 0, 0])[2]
        except ValueError:
            assert np.isnan(z[k])
            continue
        assert abs(z[k] - want) < 1e-15 + 1e-13 * abs(want)


def test_focus_known_answers(cuda):
    """The reference's focus tests (tests/test_focus.py:10-43) on the device."""
    from test_oracle import _focus_beams
    from traceon_b200.focus import focus_position
    for beams, expected in _focus_beams():
        assert np.allclose(focus_position(beams), expected)


def test_focus_matches_lstsq(cuda):
    """A converging beam with scattered final states: the device's centred
    sums against the reference's lstsq."""
    import torch
    from traceon_b200.focus import focus_position
    from oracle.oracle import focus_position as focus_oracle
    rng = np.random.default_rng(7)
    n = 100_000
    f = np.array([1e-4, -2e-4, 3e-3])
    z_end = 9.5e-3 + rng.uniform(-1e-4, 1e-4, n)
    ang = rng.uniform(-0.02, 0.02, (n, 2))
    pos = np.stack([f[0] + ang[:, 0] * (z_end - f[2]), f[1] + ang[:, 1] * (z_end - f[2]), z_end], axis=1)
    pos[:, :2] += rng.normal(0, 1e-7, (n, 2))  # aberrations
    vz = rng.uniform(1.8e7, 1.9e7, n)
    vel = np.stack([ang[:, 0] * vz, ang[:, 1] * vz, vz], axis=1)
    states = np.concatenate([pos, vel], axis=1)
    beams = [s[None] for s in states]
    want = focus_oracle(beams)
    got = focus_position(beams)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
    assert np.max(np.abs(got - f)) < 1e-6
    # through TraceResult-shaped (n, 7) states
    st7 = torch.as_tensor(np.concatenate([np.zeros((n, 1)), states], axis=1), device='cuda')
    from traceon_b200 import backend as B
    got7 = B.dev_focus_position(st7).cpu().numpy()
    assert np.array_equal(got7, got)
    # rank deficient: all directions equal -> NaN
    par = states.copy()
    par[:, 3:] = par[0, 3:]
    assert np.all(np.isnan(focus_position([s[None] for s in par[:10]])))


def test_focus_of_traced_beam(cuda):
    """focus_position of a device trace equals the oracle's on its final states."""
    from oracle.oracle import focus_position as focus_oracle
    g, res = _traced_rows()
    final = res.final.cpu().numpy()
    want = focus_oracle([s[None, 1:] for s in final])
    got = res.focus_position().cpu().numpy()
    assert np.max(np.abs(got - want)) < 1e-11 * np.max(np.abs(want))
