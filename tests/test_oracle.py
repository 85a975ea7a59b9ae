"""Pins the CPU oracle (oracle/traceon_oracle.c + oracle/oracle.py) to the
reference: against the golden vectors the reference Python package produced
(tests/golden/make_golden.py) and, when it is built, against the reference C
backend compiled from its own sources (oracle/_ref).  CPU only."""
import numpy as np
import pytest

from conftest import golden
from oracle.oracle import Oracle, axial_coefficients, solve, EM, hermite_plane_crossing, focus_position


def rel(a, b, floor=0.0):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))


def test_elliptic_golden(port):
    g = golden('elliptic.npz')
    # reference tolerance tests/test_elliptic.py:20-30 is 1e-12
    assert rel(port.ellipkm1(g['p']), g['ellipkm1']) < 1e-14
    assert rel(port.ellipem1(g['p']), g['ellipem1']) < 1e-14
    assert rel(port.ellipk(g['k']), g['ellipk']) < 1e-14
    assert rel(port.ellipe(g['k']), g['ellipe']) < 1e-14


def test_elliptic_scipy(port):
    from scipy.special import ellipkm1, ellipe
    p = 10.0 ** -np.linspace(1, 100, 5)
    assert rel(port.ellipkm1(p), ellipkm1(p)) < 1e-12
    assert rel(port.ellipem1(p), ellipe(1 - p)) < 1e-12


def test_ring_kernels_golden(port):
    g = golden('rings.npz')
    args = list(zip(g['r0'], g['z0'], g['dr'], g['dz']))
    pot = np.array([port.potential_radial_ring(*a) for a in args])
    dr1 = np.array([port.dr1_potential_radial_ring(*a) for a in args])
    dz1 = np.array([port.dz1_potential_radial_ring(*a) for a in args])
    assert rel(pot, g['pot']) < 1e-12
    assert rel(dr1, g['dr1'], 1e-9 * np.abs(g['dr1']).max()) < 1e-10
    assert rel(dz1, g['dz1'], 1e-9 * np.abs(g['dz1']).max()) < 1e-10


def test_jacobian_buffer_golden(port):
    g = golden('lens96.npz')
    jac, pos = port.fill_jacobian_buffer_radial(g['vertices'])
    assert rel(jac, g['jac']) < 1e-12
    assert np.max(np.abs(pos - g['pos'])) < 1e-18
    normals = np.array([port.higher_order_normal_radial(0.0, v) for v in g['vertices']])
    assert np.max(np.abs(normals - g['normals'])) < 1e-14


def test_fill_golden(port):
    g = golden('lens96.npz')
    v = g['vertices']
    N = len(v)
    A = port.fill_matrix_radial(v, np.ones(N, np.uint8), np.zeros(N), g['jac'], g['pos'])
    off = ~np.eye(N, dtype=bool)
    assert rel(A[off], g['fill'][off]) < 1e-11
    # the reference's own 16-point diagonal, later overwritten by the solver
    assert rel(np.diag(A), np.diag(g['fill'])) < 1e-11


def test_diagonal_golden(port):
    g = golden('lens96.npz')
    N = len(g['vertices'])
    d = port.diagonal(g['vertices'], np.ones(N, np.uint8), np.zeros(N))
    assert rel(d, g['diag']) < 1e-12
    assert rel(d, np.diag(g['matrix'])) < 1e-12


def test_dielectric_golden(port):
    g = golden('dielectric24.npz')
    v = g['vertices']
    jac, pos = port.fill_jacobian_buffer_radial(v)
    A = port.fill_matrix_radial(v, np.full(24, 3, np.uint8), g['values'], jac, pos)
    off = ~np.eye(24, dtype=bool)
    assert rel(A[off], g['fill'][off], 1e-9 * np.abs(g['fill']).max()) < 1e-10
    d = port.diagonal(v, np.full(24, 3, np.uint8), g['values'])
    assert rel(d, g['diag']) < 1e-10


def test_charges_golden(port):
    g = golden('lens96.npz')
    v = g['vertices']
    N = len(v)
    types = np.ones(N, np.uint8)
    from traceon_b200.geometry import einzel_lens
    values = einzel_lens(96).voltages_to_values(g['volts'])
    A = port.matrix(v, types, values, threads=4)
    q = solve(A, values)[0]
    assert rel(q, g['charges'], 1e-6 * np.abs(g['charges']).max()) < 1e-10
    # superposition: one RHS per electrode (traceon/solver.py:364-400)
    F = np.zeros((3, N))
    idx = einzel_lens(96).electrode_index
    for e in range(3):
        F[e, idx == e] = g['volts'][e]
    Q = solve(A, F)
    assert rel(Q, g['sup_charges'], 1e-6 * np.abs(g['sup_charges']).max()) < 1e-9
    assert rel(Q.sum(0), q, 1e-6 * np.abs(q).max()) < 1e-9


def test_fields_golden(port):
    g = golden('lens96.npz')
    q, jac, pos = g['charges'], g['jac'], g['pos']
    E = port.field_radial_many(g['points'], q, jac, pos)
    V = port.potential_radial_many(g['points'], q, jac, pos)
    scale = np.abs(g['E_points']).max()
    assert np.max(np.abs(E - g['E_points'])) / scale < 1e-12
    assert rel(V, g['V_points'], 1e-9 * np.abs(g['V_points']).max()) < 1e-12


def test_axial_golden(port):
    g = golden('lens96.npz')
    d = port.axial_derivatives_radial(g['z_axial'], g['charges'], g['jac'], g['pos'])
    for l in range(9):
        s = np.abs(g['derivs'][:, l]).max()
        assert np.max(np.abs(d[:, l] - g['derivs'][:, l])) / s < 1e-11, l
    c = axial_coefficients(g['z_axial'], g['derivs'])
    for l in range(9):
        s = np.abs(g['coeffs'][:, l]).max()
        assert np.max(np.abs(c[:, l] - g['coeffs'][:, l])) / s < 1e-10, l
    E = np.array([port.field_radial_derivs(p, g['z_axial'], g['coeffs']) for p in g['axial_points']])
    assert np.max(np.abs(E - g['E_axial'])) / np.abs(g['E_axial']).max() < 1e-12


def test_traces_golden(port):
    g = golden('lens96.npz')
    for i in range(3):
        t, s = port.trace_bem(g['p0'][i], g['v0'][i], EM, g['charges'], g['jac'], g['pos'], g['bounds'], 1e-10)
        ts, ss = g[f'bem_t{i}'], g[f'bem_s{i}']
        assert len(s) == len(ss)
        # The shipped reference build updates h with -ffast-math pow, so its
        # step times drift ~1e-9 relative from the strict port: states along
        # the path differ by < 0.5 nm, the plane crossings by < 1 pm.
        assert np.max(np.abs(s[:, :3] - ss[:, :3])) < 5e-10
        lin = port.plane_intersection(s, [0, 0, 9.5e-3], [0, 0, 1])
        assert np.max(np.abs(lin - g['cross'][i])[:3]) < 1e-12
        t, s = port.trace_axial(g['p0'][i], g['v0'][i], EM, g['z_axial'], g['coeffs'], np.zeros_like(g['coeffs']),
                                g['bounds'], 1e-10)
        assert len(s) == len(g[f'ax_s{i}'])
        assert np.max(np.abs(s[:, :3] - g[f"ax_s{i}"][:, :3])) < 5e-10
        lin = port.plane_intersection(s, [0, 0, 9.5e-3], [0, 0, 1])
        assert np.max(np.abs(lin - g['cross_axial'][i])[:3]) < 1e-12


def test_hermite_crossing_exact_on_cubic():
    # a trajectory whose z(t) is exactly cubic must give the exact crossing
    t0, h = 0.0, 2.0
    z = lambda t: 0.1 * t**3 - 0.2 * t**2 + t
    dz = lambda t: 0.3 * t**2 - 0.4 * t + 1
    s0 = np.array([0, 0, z(t0), 0, 0, dz(t0)])
    s1 = np.array([0, 0, z(t0 + h), 0, 0, dz(t0 + h)])
    zp = 1.0
    out = hermite_plane_crossing(np.array([t0, t0 + h]), np.stack([s0, s1]), zp)
    assert abs(out[2] - zp) < 1e-15


def _focus_beams():
    """The beams of the reference's focus tests (tests/test_focus.py:10-43)
    with the focus each one pins."""
    from traceon_b200.tracing import velocity_vec, velocity_vec_spherical
    v1, v2 = velocity_vec(10, [-1e-3, 0., -1]), velocity_vec(10, [1e-3, 0., -1])
    p1 = np.concatenate((3 * v1, v1))[np.newaxis, :]
    p2 = np.concatenate((3 * v2, v2))[np.newaxis, :]
    cases = [([p1.copy(), p2.copy()], [0, 0, 0])]
    p1[0, 0] += 1
    p2[0, 0] += 1
    cases.append(([p1.copy(), p2.copy()], [1, 0, 0]))
    for p in (p1, p2):
        p[0, 1] += 1
        p[0, 2] += 1
    cases.append(([p1.copy(), p2.copy()], [1, 1, 1]))
    w1, w2, w3 = (velocity_vec_spherical(1, 0, 0), velocity_vec_spherical(5, 1 / 30, 1 / 30),
                  velocity_vec_spherical(10, 1 / 30, np.pi / 2))
    cases.append(([np.concatenate((w, w))[np.newaxis, :] for w in (w1, w2, w3)], [0, 0, 0]))
    return cases


def test_focus_known_answers():
    """The oracle's focus_position against the reference's focus tests."""
    for beams, expected in _focus_beams():
        assert np.allclose(focus_position(beams), expected)


def test_oracle_vs_reference_build(port, ref):
    """The restatement against the reference compiled from its sources."""
    from traceon_b200.geometry import einzel_lens
    geo = einzel_lens(120)
    v = geo.vertices
    N = len(v)
    jp, pp = port.fill_jacobian_buffer_radial(v)
    jr, pr = ref.fill_jacobian_buffer_radial(v)
    assert rel(jp, jr) < 1e-12 and np.max(np.abs(pp - pr)) < 1e-18
    Ap = port.fill_matrix_radial(v, np.ones(N, np.uint8), np.zeros(N), jp, pp)
    Ar = ref.fill_matrix_radial(v, np.ones(N, np.uint8), np.zeros(N), jr, pr)
    assert rel(Ap, Ar) < 1e-11
    q = np.random.default_rng(1).normal(size=N)
    pts = np.array([[2e-4, 1e-4, -1e-3], [5e-4, 0, 2e-3], [0, 0, 0.1e-3]])
    for p in pts:
        assert rel(port.field_radial(p, q, jp, pp), ref.field_radial(p, q, jr, pr),
                   1e-9 * np.abs(ref.field_radial(p, q, jr, pr)).max()) < 1e-11
        assert rel(port.potential_radial(p, q, jp, pp), ref.potential_radial(p, q, jr, pr)) < 1e-12


def test_diagonal_converged_vs_shipped_call(port, ref):
    """The oracle's diagonal is the reference's self integral converged to
    ~1e-15.  The reference's own call (epsabs = epsrel = 1e-9) agrees with it
    to 1e-12 on most elements but is off by up to ~1e-5 on a few mm-scale
    elements, and which ones depends on the build's rounding."""
    from traceon_b200.geometry import einzel_lens
    v = einzel_lens(1000).vertices[::5]
    acc = np.array([port.self_potential_radial(x) for x in v])
    shipped = np.array([ref.self_potential_radial(x, shipped=True) for x in v])
    r = np.abs(acc - shipped) / np.abs(acc)
    assert np.median(r) < 1e-13
    assert r.max() < 1e-4


def _coil_rings(seed, n=20):
    """Synthetic coil cross-section quadrature: n triangles in r in [3, 6] mm,
    z in [-1, 1] mm, 12 points each (y = 0), weights = area / 12; currents
    U[0.5, 5] kA-turns spread over the triangles."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 12, 3))
    pos[:, :, 0] = rng.uniform(3e-3, 6e-3, (n, 12))
    pos[:, :, 2] = rng.uniform(-1e-3, 1e-3, (n, 12))
    jac = np.full((n, 12), 1e-8 / 12)
    I = rng.uniform(500.0, 5000.0, n) / n
    return I, jac, pos


def test_current_rings_vs_reference_build(port, ref):
    """current_field_radial (radial.c:55-83) and current_axial_derivatives_radial
    (radial.c:85-103): the oracle's restatement against the reference build."""
    I, jac, pos = _coil_rings(3)
    rng = np.random.default_rng(4)
    pts = np.stack([rng.uniform(0, 2e-3, 30), rng.uniform(-1e-3, 1e-3, 30), rng.uniform(-8e-3, 8e-3, 30)], 1)
    for p in pts:
        a, b = port.current_field_radial(p, I, jac, pos), ref.current_field_radial(p, I, jac, pos)
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    z = np.linspace(-8e-3, 8e-3, 41)
    a, b = port.current_axial_derivatives_radial(z, I, jac, pos), ref.current_axial_derivatives_radial(z, I, jac, pos)
    for c in range(b.shape[1]):
        assert np.max(np.abs(a[:, c] - b[:, c])) <= 1e-11 * np.max(np.abs(b[:, c]))
