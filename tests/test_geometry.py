"""Host-side geometry bookkeeping the device mesher relies on: a lens's
recorded segments and element counts regenerate exactly its vertices with the
host mesher, and the element counts split as documented.  CPU only."""
import numpy as np

from traceon_b200 import geometry as G


def _remesh(geo):
    return np.concatenate([G.polyline_elements([s[:2], s[2:]], [c])
                           for s, c in zip(geo.segments, geo.segment_counts)])


def test_segments_and_counts_regenerate_the_mesh():
    geos = [G.einzel_lens(1000), G.einzel_lens(96)] + [G.random_lens(s)[0] for s in range(4)]
    for geo in geos:
        assert geo.segment_counts.sum() == len(geo)
        assert len(geo.segment_counts) == len(geo.segments)
        assert np.array_equal(_remesh(geo), geo.vertices)


def test_split_counts():
    c = G.split_counts(100, [1.0, 8.0, 1.0])
    assert sum(c) == 100 and min(c) >= 2 and c[1] > c[0] == c[2]
    assert G.split_counts(6, [1.0, 100.0, 1.0]) == [2, 2, 2]
    # fewer than 2 per segment: at least 1 each, and the total is kept
    assert G.split_counts(3, [1.0, 1.0, 1.0]) == [1, 1, 1]
    c = G.split_counts(5, [1.0, 1.0, 1.0])
    assert sum(c) == 5 and min(c) >= 1
    # fewer elements than segments cannot be split
    import pytest
    for total, lengths in ((1, [1, 1, 1]), (2, [1, 1, 1]), (0, [1, 2]), (3, [])):
        with pytest.raises(ValueError):
            G.split_counts(total, lengths)


def test_graded_nodes_dense_at_both_ends():
    s = G.graded_nodes(10)
    assert s[0] == 0.0 and s[-1] == 1.0
    d = np.diff(s)
    assert d[0] < d[5] and d[-1] < d[5] and np.allclose(d, d[::-1])


def test_device_entry_points_reject_bad_arguments_on_the_host():
    """Argument checks that run before any device work (no GPU needed)."""
    import pytest
    from conftest import golden
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.tracing import trace_geometries
    g = golden('lens96.npz')
    f = FieldRadialBEM(EffectivePointCharges(g['charges'], g['jac'], g['pos']))
    p, v = np.zeros((2, 3)), np.zeros((2, 3))
    with pytest.raises(ValueError):
        trace_geometries([f, f], g['bounds'], [p], [v], 0.0)
    with pytest.raises(ValueError):
        trace_geometries([], g['bounds'], [], [], 0.0)
    bounded = FieldRadialBEM(EffectivePointCharges(g['charges'], g['jac'], g['pos']))
    bounded.field_bounds = np.array([[-1e-3, 1e-3], [-1e-3, 1e-3], [-1e-2, 1e-2]])
    with pytest.raises(NotImplementedError):
        trace_geometries([bounded], g['bounds'], [p], [v], 0.0)
    with pytest.raises(ValueError):
        G.mesh_segments_device(np.zeros((2, 4)), [3])
    with pytest.raises(ValueError):
        G.mesh_segments_device(np.zeros((2, 4)), [3, -1])
