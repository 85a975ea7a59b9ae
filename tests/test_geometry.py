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


def test_mirror_lens_workload_properties():
    """The batching workload's lenses: N ~ U[500, 6000] elements in all, the
    last electrode a mirror plate at -1.1 x the beam voltage holding about
    10 % (at least 24) of the elements, the trace box inside the mirror's
    bore and the beam start before the first tube."""
    for seed in (1000, 1001, 1005, 1063):
        m = G.mirror_lens(seed)
        geo = m.geometry
        n = len(geo)
        assert 500 <= n <= 6000
        assert geo.names[-1] == 'mirror' and m.voltages[-1] == -1.1 * 1000.0
        assert len(m.voltages) == len(geo.names)
        n_mirror = int(np.sum(geo.electrode_index == len(geo.names) - 1))
        assert n_mirror == max(24, n // 10)
        assert geo.segment_counts.sum() == n
        r_vert = geo.vertices[:, :, 0]
        bore = r_vert[geo.electrode_index == len(geo.names) - 1].min()
        assert m.bounds[0, 1] < bore and m.bounds[1, 1] < bore and m.bounds[0, 0] == -m.bounds[0, 1]
        z_tubes = geo.vertices[geo.electrode_index < len(geo.names) - 1][:, :, 2]
        assert m.bounds[2, 0] < m.z_start < z_tubes.min()
        assert m.bounds[2, 1] > geo.vertices[:, :, 2].max()


def test_mirror_beam_distributions():
    """Lognormal energies (median 1 keV) clipped to [100 eV, 10 keV], start
    radius up to 50 µm at y = 0, angles within ±50 mrad in the xz-plane."""
    from scipy.constants import e, m_e
    pos, vel = G.mirror_beam(20000, 7, z0=-3e-3)
    energy = 0.5 * m_e * np.sum(vel ** 2, axis=1) / e
    assert energy.min() >= 100.0 - 1e-6 and energy.max() <= 10000.0 + 1e-3
    assert abs(np.median(energy) / 1000.0 - 1.0) < 0.05
    assert np.any(np.isclose(energy, 100.0)) and np.any(np.isclose(energy, 10000.0))  # both clips reached
    assert np.all((pos[:, 0] >= 0) & (pos[:, 0] <= 0.05e-3)) and np.all(pos[:, 1] == 0) and np.all(pos[:, 2] == -3e-3)
    ang = np.arctan2(vel[:, 0], vel[:, 2])
    assert np.all(np.abs(ang) <= 50e-3 + 1e-12) and np.all(vel[:, 1] == 0)


def test_combined_lens_and_beam():
    """The combined workload: the einzel lens plus the pole piece meshed with
    the asked element counts (normals out of the iron), coils in the yoke's
    window, and the 5 keV beam."""
    from scipy.constants import e, m_e
    cl = G.combined_lens(1, n_elec=600, n_mag=400)
    geo = cl.geometry
    assert len(geo) == 1000 and geo.names[-1] == 'pole'
    pole = geo.vertices[geo.electrode_index == len(geo.names) - 1]
    assert len(pole) == 400
    assert np.array_equal(G.outward_oriented(pole), pole)  # already oriented outward
    r, z, current = cl.coil_r, cl.coil_z, cl.coil_current
    assert np.all((3e-3 <= r) & (r <= 6e-3)) and np.all(np.abs(z) <= 4e-3)
    assert np.all((500.0 <= current) & (current <= 5000.0))
    pos, vel = G.combined_beam(5000, 3)
    energy = 0.5 * m_e * np.sum(vel ** 2, axis=1) / e
    assert abs(np.median(energy) / 5000.0 - 1.0) < 0.005 and np.std(np.log(energy)) < 0.03
    assert np.all(pos[:, 0] <= 0.2e-3) and np.all(pos[:, 2] == -9.5e-3)
