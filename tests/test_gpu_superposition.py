"""GPU-native tracing of field superpositions.

The reference traces a FieldSuperposition through a Python callback per
field evaluation (traceon/field.py:464-465 hands the superposition itself to
the tracer).  Here a superposition of radial BEM fields collapses into one
source set (charges times factors, shifted along z by each member's origin)
and a superposition of axial fields on one z grid into one coefficient
table, so the GPU tracer runs unchanged.  Checked against the CPU oracle's
tracer on the equivalent combined charges (trace endpoints within 1e-12 m,
the BEM tracer's parity tolerance)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _lens_field():
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    g = golden('lens96.npz')
    return g, FieldRadialBEM(EffectivePointCharges(g['charges'], g['jac'], g['pos']))


def test_superposition_of_moved_bem_fields(cuda, port):
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM, FieldSuperposition
    from traceon_b200.tracing import Tracer
    from oracle.oracle import EM, hermite_plane_crossing
    g, A = _lens_field()
    dz = 2.5e-3
    S = 0.7 * A + 1.3 * A.move(dz=dz)  # different origins: a superposition, not one BEM field
    assert isinstance(S, FieldSuperposition) and len(S) == 2
    # the equivalent single source set
    pos_b = g['pos'].copy()
    pos_b[..., 1] += dz
    q = np.concatenate([0.7 * g['charges'], 1.3 * g['charges']])
    jac = np.concatenate([g['jac'], g['jac']])
    pos = np.concatenate([g['pos'], pos_b])
    combined = FieldRadialBEM(EffectivePointCharges(q, jac, pos))
    for p in ([1e-4, 0.0, 1e-3], [3e-4, 2e-4, -2e-3], [0.0, 0.0, 6e-3]):
        e_s, e_c = S.electrostatic_field_at_point(p), combined.electrostatic_field_at_point(p)
        assert np.max(np.abs(e_s - e_c)) < 1e-11 * np.max(np.abs(e_c))
    plane, final, status, counters = Tracer(S, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
    assert np.all(status == cuda.TRACE_EXITED)
    for i in range(len(g['p0'])):
        t, s = port.trace_bem(g['p0'][i], g['v0'][i], EM, q, jac, pos, g['bounds'], 1e-10)
        h = hermite_plane_crossing(t, s, 9.5e-3)
        assert np.max(np.abs(plane[i, 1:4] - h[:3])) < 1e-12  # metres
        assert counters[i, 0] == len(s) - 1


def test_nested_superposition_and_scaling(cuda):
    """Nested superpositions expand with their factors multiplied."""
    from traceon_b200.tracing import Tracer
    g, A = _lens_field()
    S1 = 0.5 * (A + A.move(dz=1e-3))
    S2 = 0.5 * A + 0.5 * A.move(dz=1e-3)
    p1, _, st1, _ = Tracer(2.0 * S1, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
    p2, _, st2, _ = Tracer(2.0 * S2, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
    assert np.all(st1 == 0) and np.all(st2 == 0)
    assert np.max(np.abs(p1[:, 1:4] - p2[:, 1:4])) < 1e-12


def test_superposition_of_axial_fields(cuda):
    """Axial members on one z grid collapse into one coefficient table:
    0.4 ax + 0.6 ax traces like ax."""
    from traceon_b200.field import FieldRadialAxial, FieldSuperposition
    from traceon_b200.tracing import Tracer
    g, A = _lens_field()
    z = g['z_axial']
    ax = FieldRadialAxial(A, z[0], z[-1], N=len(z))
    S = FieldSuperposition([ax, ax], [0.4, 0.6])
    p_s, _, st_s, _ = Tracer(S, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
    p_a, _, st_a, _ = Tracer(ax, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
    assert np.all(st_s == 0) and np.all(st_a == 0)
    assert np.max(np.abs(p_s[:, 1:4] - p_a[:, 1:4])) < 1e-12


def test_unsupported_superpositions_raise(cuda):
    from traceon_b200.field import FieldRadialAxial, FieldSuperposition
    from traceon_b200.tracing import Tracer
    g, A = _lens_field()
    z = g['z_axial']
    ax = FieldRadialAxial(A, z[0], z[-1], N=len(z))
    cases = [FieldSuperposition([A, ax]),                     # BEM mixed with axial
             FieldSuperposition([A, A.move(dx=1e-4)]),        # symmetry axis moved off z
             FieldSuperposition([ax, FieldRadialAxial(A, z[0], z[-1], N=len(z) + 1)])]  # different z grids
    for S in cases:
        with pytest.raises(NotImplementedError):
            Tracer(S, g['bounds']).trace_endpoints(g['p0'], g['v0'], 9.5e-3, atol=1e-10)
