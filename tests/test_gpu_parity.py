"""GPU parity: every kernel of libtraceon_b200.so against the CPU oracle and
the golden vectors of the reference, called through the C ABI.

Tolerances (FP64 throughout, the reference's arithmetic type):
  off-diagonal matrix entries      1e-12 relative
  self integrals (diagonal)        1e-12 relative to the converged integral
  charges                          1e-10 relative to max |charge|
  fields / potentials              1e-11 relative to max |value|
  axial derivatives / coefficients 1e-11 / 1e-10 relative per column
  trace endpoints                  1 nm (and in practice < 1 pm)
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b, floor=0.0):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def poly_values(c, h):
    """Values of every (interval, derivative) polynomial of an axial
    coefficient table (N_z-1, 9, 6) at x = 0, h/3, 2h/3, h."""
    x = np.array([0.0, h / 3, 2 * h / 3, h])
    return sum(c[:, :, k, None] * x ** (5 - k) for k in range(6))


def assert_same_polynomials(c, c_ref, h, tol):
    """Coefficient tables agree where it matters: the evaluated pieces, per
    derivative column, relative to that column's largest value.  (The
    highest-order coefficients themselves carry cancellation error in any
    FP64 construction: SciPy's Bernstein route and the closed form here
    differ there by ~1e-6 relative while the pieces agree to ~1e-14.)"""
    a, b = poly_values(c, h), poly_values(c_ref, h)
    for l in range(c.shape[1]):
        s = np.abs(b[:, l]).max()
        assert np.max(np.abs(a[:, l] - b[:, l])) / s < tol, l


def lens(n=96):
    from traceon_b200.geometry import einzel_lens
    return einzel_lens(n)


@pytest.fixture(scope='module')
def g96():
    return golden('lens96.npz')


def test_library_is_the_cuda_build(cuda):
    import torch
    assert torch.cuda.is_available()
    assert cuda.num_sms() > 0
    assert cuda.backend_lib._name.endswith('libtraceon_b200.so')


def test_jacobian_buffer(cuda, g96):
    import torch
    v = cuda.to_dev(g96['vertices'], torch.float64)
    jac, pos = cuda.dev_jacobian_buffer(v)
    assert rel(jac.cpu().numpy(), g96['jac']) < 1e-13
    assert np.max(np.abs(pos.cpu().numpy() - g96['pos'])) < 1e-18
    # reference-compatible host entry point
    jh, ph = cuda.fill_jacobian_buffer_radial(g96['vertices'])
    assert rel(jh, g96['jac']) < 1e-13


@pytest.mark.parametrize('n', [96, 517])
def test_fill_offdiagonal(cuda, port, n):
    import torch
    geo = lens(n)
    v = geo.vertices
    types = np.ones(n, np.uint8)
    values = np.zeros(n)
    jac, pos = port.fill_jacobian_buffer_radial(v)
    A_or = port.fill_matrix_radial(v, types, values, jac, pos)
    vt = cuda.to_dev(v, torch.float64)
    jt, pt = cuda.dev_jacobian_buffer(vt)
    A = torch.zeros((n, n), dtype=torch.float64, device=vt.device)
    cuda.dev_fill_matrix(A, vt, cuda.to_dev(types, torch.uint8), cuda.to_dev(values, torch.float64), jt, pt,
                         gauss_diagonal=True)
    A = A.cpu().numpy()
    assert rel(A, A_or) < 1e-12


def test_fill_golden_and_compat_rows(cuda, g96):
    v = g96['vertices']
    N = len(v)
    types = np.ones(N, np.uint8)
    M = np.zeros((N, N))
    # row-split calls as traceon/solver.py:226-236 makes them
    for rows in np.array_split(np.arange(N), 5):
        cuda.fill_matrix_radial(M, v, types, np.zeros(N), g96['jac'], g96['pos'], rows[0], rows[-1])
    assert rel(M, g96['fill']) < 1e-12
    # accumulation semantics (+=)
    cuda.fill_matrix_radial(M, v, types, np.zeros(N), g96['jac'], g96['pos'], 0, N - 1)
    assert rel(M, 2 * g96['fill']) < 1e-12


def test_fill_unknown_type_is_reported(cuda, g96):
    v = g96['vertices']
    N = len(v)
    types = np.ones(N, np.uint8)
    types[3] = 9
    M = np.zeros((N, N))
    with pytest.raises(cuda.BackendError):
        cuda.fill_matrix_radial(M, v, types, np.zeros(N), g96['jac'], g96['pos'], 0, N - 1)
    assert not M.any()


def test_self_integrals(cuda, port, g96):
    v = g96['vertices']
    N = len(v)
    d = cuda.dev_self_integrals_np(v, np.ones(N, np.uint8), np.zeros(N))
    d_acc = port.diagonal(v, np.ones(N, np.uint8), np.zeros(N))
    assert rel(d, d_acc) < 1e-12
    assert rel(d, g96['diag']) < 1e-11
    # dielectric rows: self flux - 1 (solver.py:239-244)
    gd = golden('dielectric24.npz')
    dd = cuda.dev_self_integrals_np(gd['vertices'], np.full(24, 3, np.uint8), gd['values'])
    dd_acc = port.diagonal(gd['vertices'], np.full(24, 3, np.uint8), gd['values'])
    assert rel(dd, dd_acc) < 1e-12
    assert rel(dd, gd['diag']) < 1e-10
    # compat single-element form
    assert abs(cuda.self_potential_radial(v[5]) - d_acc[5]) / abs(d_acc[5]) < 1e-12


def test_self_integrals_1000(cuda, port):
    geo = lens(1000)
    idx = np.arange(0, 1000, 37)
    v = geo.vertices
    d = cuda.dev_self_integrals_np(v, np.ones(1000, np.uint8), np.zeros(1000))[idx]
    d_acc = np.array([port.self_potential_radial(v[i]) for i in idx])
    assert rel(d, d_acc) < 1e-12


def _solve_gpu(cuda, v, types, values, F):
    import torch
    vt = cuda.to_dev(v, torch.float64)
    tt = cuda.to_dev(types, torch.uint8)
    valt = cuda.to_dev(values, torch.float64)
    jt, pt = cuda.dev_jacobian_buffer(vt)
    n = len(v)
    A = torch.empty((n, n), dtype=torch.float64, device=vt.device)
    cuda.dev_fill_matrix(A, vt, tt, valt, jt, pt)
    cuda.dev_self_integrals(vt, tt, valt, A)
    A0 = A.clone()
    ipiv, perm = cuda.dev_lu_factor(A)
    X = cuda.dev_lu_solve(A, perm, cuda.to_dev(np.atleast_2d(F), torch.float64))
    return A0.cpu().numpy(), X.cpu().numpy()


@pytest.mark.parametrize('n', [96, 1000])
def test_charges(cuda, port, n):
    geo = lens(n)
    volts = np.array([0.0, 1500.0, 0.0])
    values = geo.voltages_to_values(volts)
    types = np.ones(n, np.uint8)
    F = np.vstack([values, geo.unit_rhs()])
    A, X = _solve_gpu(cuda, geo.vertices, types, values, F)
    A_or = port.matrix(geo.vertices, types, values, threads=8)
    assert rel(A, A_or) < 1e-12
    X_or = np.linalg.solve(A_or, F.T).T
    for k in range(len(F)):
        assert np.max(np.abs(X[k] - X_or[k])) / np.abs(X_or[k]).max() < 1e-10
    # residual with the FP64 matrix
    r = A_or @ X.T - F.T
    assert np.max(np.abs(r)) / np.abs(F).max() < 1e-12


def test_charges_golden(cuda, g96):
    geo = lens(96)
    values = geo.voltages_to_values(g96['volts'])
    _, X = _solve_gpu(cuda, g96['vertices'], np.ones(96, np.uint8), values, values)
    assert np.max(np.abs(X[0] - g96['charges'])) / np.abs(g96['charges']).max() < 1e-10


@pytest.mark.parametrize('M', [1, 64, 5000])
def test_field_points(cuda, port, g96, M):
    import torch
    rng = np.random.default_rng(M)
    if M == 64:
        pts = g96['points']
    else:
        pts = np.stack([rng.uniform(-9e-4, 9e-4, M), rng.uniform(-9e-4, 9e-4, M), rng.uniform(-8e-3, 8e-3, M)], 1)
    q, jac, pos = g96['charges'], g96['jac'], g96['pos']
    src = cuda.dev_pack_sources(cuda.to_dev(q, torch.float64), cuda.to_dev(jac, torch.float64),
                                cuda.to_dev(pos, torch.float64))
    pot, f = cuda.dev_field_points(cuda.to_dev(pts, torch.float64), src)
    pot, f = pot.cpu().numpy(), f.cpu().numpy()
    sel = np.arange(M) if M <= 64 else rng.choice(M, 64, replace=False)
    E_or = port.field_radial_many(pts[sel], q, jac, pos)
    V_or = port.potential_radial_many(pts[sel], q, jac, pos)
    assert np.max(np.abs(f[sel] - E_or)) / np.abs(E_or).max() < 1e-11
    assert np.max(np.abs(pot[sel] - V_or)) / np.abs(V_or).max() < 1e-12
    if M == 64:
        assert np.max(np.abs(f - g96['E_points'])) / np.abs(g96['E_points']).max() < 1e-11
        assert np.max(np.abs(pot - g96['V_points'])) / np.abs(g96['V_points']).max() < 1e-12


def test_field_points_thread_kernel(cuda, port, g96):
    """Enough points for the one-thread-per-point kernel (>= 2048 per SM)."""
    import torch
    M = cuda.num_sms() * 2048 + 17
    rng = np.random.default_rng(5)
    pts = np.stack([rng.uniform(0, 9e-4, M), np.zeros(M), rng.uniform(-8e-3, 8e-3, M)], 1)
    q, jac, pos = g96['charges'], g96['jac'], g96['pos']
    src = cuda.dev_pack_sources(cuda.to_dev(q, torch.float64), cuda.to_dev(jac, torch.float64),
                                cuda.to_dev(pos, torch.float64))
    pot, f = cuda.dev_field_points(cuda.to_dev(pts, torch.float64), src)
    sel = np.concatenate([rng.choice(M, 48, replace=False), [M - 1]])
    E_or = port.field_radial_many(pts[sel], q, jac, pos)
    V_or = port.potential_radial_many(pts[sel], q, jac, pos)
    assert np.max(np.abs(f.cpu().numpy()[sel] - E_or)) / np.abs(E_or).max() < 1e-11
    assert np.max(np.abs(pot.cpu().numpy()[sel] - V_or)) / np.abs(V_or).max() < 1e-12


def test_compat_field_and_potential(cuda, g96):
    q, jac, pos = g96['charges'], g96['jac'], g96['pos']
    for p, E, V in list(zip(g96['points'], g96['E_points'], g96['V_points']))[:5]:
        assert np.max(np.abs(cuda.field_radial(p, q, jac, pos) - E)) < 1e-11 * np.abs(g96['E_points']).max()
        assert abs(cuda.potential_radial(p, q, jac, pos) - V) < 1e-12 * np.abs(g96['V_points']).max()


def test_axial(cuda, port, g96):
    import torch
    q, jac, pos = g96['charges'], g96['jac'], g96['pos']
    z = g96['z_axial']
    src = cuda.dev_pack_sources(cuda.to_dev(q, torch.float64), cuda.to_dev(jac, torch.float64),
                                cuda.to_dev(pos, torch.float64))
    d = cuda.dev_axial_derivatives(cuda.to_dev(z, torch.float64), src)
    dn = d.cpu().numpy()
    for l in range(9):
        s = np.abs(g96['derivs'][:, l]).max()
        assert np.max(np.abs(dn[:, l] - g96['derivs'][:, l])) / s < 1e-11, l
    c = cuda.dev_axial_coefficients(cuda.to_dev(g96['derivs'], torch.float64), z[1] - z[0]).cpu().numpy()
    assert_same_polynomials(c, g96['coeffs'], z[1] - z[0], 1e-12)
    # compat accumulate semantics
    dd = cuda.axial_derivatives_radial(z, q, jac, pos)
    assert np.max(np.abs(dd - g96['derivs'])) <= 1e-11 * np.abs(g96['derivs']).max(axis=0).max()
    # axial field evaluation at points
    pot, f = cuda.dev_axial_field_points(cuda.to_dev(g96['axial_points'], torch.float64),
                                         cuda.to_dev(z, torch.float64), cuda.to_dev(g96['coeffs'], torch.float64))
    assert np.max(np.abs(f.cpu().numpy() - g96['E_axial'])) / np.abs(g96['E_axial']).max() < 1e-13
    assert np.max(np.abs(pot.cpu().numpy() - g96['V_axial'])) / np.abs(g96['V_axial']).max() < 1e-13


@pytest.mark.parametrize('nz', [2, 3, 4, 7, 2000])
def test_axial_spline_sizes(cuda, nz):
    """Coefficients of the not-a-knot cubic and quintic Hermite pieces
    against SciPy for the edge sizes CubicSpline special-cases."""
    import torch
    from oracle.oracle import axial_coefficients
    z = np.linspace(-1e-3, 2e-3, nz)
    rng = np.random.default_rng(nz)
    d = rng.normal(size=(nz, 9)) * 10.0 ** np.arange(9)
    c = cuda.dev_axial_coefficients(cuda.to_dev(d, torch.float64), z[1] - z[0]).cpu().numpy()
    c_or = axial_coefficients(z, d)
    assert_same_polynomials(c, c_or, z[1] - z[0], 1e-11)


def _geometry_field(cuda, port, n=300, volts=(0.0, 1200.0, 0.0)):
    geo = lens(n)
    values = geo.voltages_to_values(np.array(volts))
    A = port.matrix(geo.vertices, np.ones(n, np.uint8), values, threads=8)
    q = np.linalg.solve(A, values)
    jac, pos = port.fill_jacobian_buffer_radial(geo.vertices)
    return q, jac, pos


def test_trace_endpoints_vs_oracle(cuda, port):
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.tracing import Tracer
    from traceon_b200 import geometry as G
    from oracle.oracle import EM, hermite_plane_crossing
    q, jac, pos = _geometry_field(cuda, port)
    field = FieldRadialBEM(EffectivePointCharges(q, jac, pos))
    p0, v0 = G.electron_beam(24, 3)
    tr = Tracer(field, G.LENS_BOUNDS)
    for tw in (0, 1, 2, 8):
        plane, final, status, counters = tr.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=1e-10, team_warps=tw)
        assert np.all(status == cuda.TRACE_EXITED)
        for i in range(0, 24, 5):
            t, s = port.trace_bem(p0[i], v0[i], EM, q, jac, pos, G.LENS_BOUNDS, 1e-10)
            h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
            assert np.max(np.abs(plane[i, 1:4] - h[:3])) < 1e-12  # metres
            assert counters[i, 0] == len(s) - 1
            assert np.max(np.abs(final[i, 1:4] - s[-1, :3])) < 1e-9


def test_trace_multiple_trajectories(cuda, g96):
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    field = FieldRadialBEM(EffectivePointCharges(g96['charges'], g96['jac'], g96['pos']))
    tr = field.get_tracer(g96['bounds'])
    res = tr.trace_multiple(g96['p0'], g96['v0'], atol=1e-10)
    for i, (t, s) in enumerate(res):
        ss = g96[f'bem_s{i}']
        assert len(s) == len(ss)
        assert np.max(np.abs(s[:, :3] - ss[:, :3])) < 5e-10
        from traceon_b200.tracing import xy_plane_intersection
        assert np.max(np.abs(xy_plane_intersection(s, 9.5e-3)[:3] - g96['cross'][i][:3])) < 1e-12


def test_trace_compat_entry_point(cuda, g96):
    """backend.trace_particle through the reference's field callback + args."""
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from scipy.constants import e, m_e
    field = FieldRadialBEM(EffectivePointCharges(g96['charges'], g96['jac'], g96['pos']))
    fun, args = field.get_low_level_trace_function()
    import ctypes as C
    t, s = cuda.trace_particle(g96['p0'][0], g96['v0'][0], -e / m_e, fun, g96['bounds'], 1e-10,
                               C.cast(C.pointer(args), C.c_void_p))
    ss = g96['bem_s0']
    assert len(s) == len(ss)
    assert np.max(np.abs(s[:, :3] - ss[:, :3])) < 5e-10
    with pytest.raises(NotImplementedError):
        cuda.trace_particle(g96['p0'][0], g96['v0'][0], -e / m_e, cuda.wrap_field_fun(lambda p, v: (p, v)),
                            g96['bounds'], 1e-10, None)


def test_trace_axial(cuda, g96):
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM, FieldRadialAxial
    field = FieldRadialBEM(EffectivePointCharges(g96['charges'], g96['jac'], g96['pos']))
    ax = FieldRadialAxial(field, g96['z_axial'][0], g96['z_axial'][-1], N=len(g96['z_axial']))
    z = g96['z_axial']
    assert_same_polynomials(ax.electrostatic_coeffs, g96['coeffs'], z[1] - z[0], 1e-11)
    res = ax.get_tracer(g96['bounds']).trace_multiple(g96['p0'], g96['v0'], atol=1e-10)
    from traceon_b200.tracing import xy_plane_intersection
    for i, (t, s) in enumerate(res):
        assert len(s) == len(g96[f'ax_s{i}'])
        assert np.max(np.abs(xy_plane_intersection(s, 9.5e-3)[:3] - g96['cross_axial'][i][:3])) < 1e-12


def test_trace_attempt_cap_and_nonfinite(cuda, g96):
    """A particle that would loop forever ends with a status (no hang)."""
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.tracing import Tracer
    from traceon_b200 import geometry as G
    field = FieldRadialBEM(EffectivePointCharges(g96['charges'], g96['jac'], g96['pos']))
    tr = Tracer(field, G.LENS_BOUNDS)
    p0, v0 = G.electron_beam(4, 1)
    plane, final, status, counters = tr.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=1e-10, max_attempts=5)
    assert np.all(status == cuda.TRACE_MAX_ATTEMPTS) and np.all(counters[:, 1] == 5)
    bad = FieldRadialBEM(EffectivePointCharges(g96['charges'] * np.nan, g96['jac'], g96['pos']))
    plane, final, status, counters = Tracer(bad, G.LENS_BOUNDS).trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=1e-10)
    assert np.all(status == cuda.TRACE_NONFINITE)


def test_solver_api_end_to_end(cuda, g96):
    """solve_direct on a Mesh/Excitation like the reference's public API."""
    from traceon_b200.excitation import Mesh, Excitation
    from traceon_b200 import solver as S
    geo = lens(96)
    mesh = Mesh.from_geometry(geo)
    exc = Excitation(mesh)
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, g96['volts'])})
    field = S.solve_direct(exc)
    q = field.electrostatic_point_charges.charges
    assert np.max(np.abs(q - g96['charges'])) / np.abs(g96['charges']).max() < 1e-10
    sup = S.solve_direct_superposition(exc)
    Q = np.array([sup[n].electrostatic_point_charges.charges for n in geo.names])
    assert np.max(np.abs(Q - g96['sup_charges'])) / np.abs(g96['sup_charges']).max() < 1e-9
    total = sup['ground_in'] + sup['lens'] + sup['ground_out']
    assert np.allclose(total.electrostatic_point_charges.charges, q, rtol=0, atol=1e-9 * np.abs(q).max())
    E = field.electrostatic_field_at_points(g96['points'])
    assert np.max(np.abs(E - g96['E_points'])) / np.abs(g96['E_points']).max() < 1e-10
    assert np.allclose(field.field_at_point(g96['points'][0]), g96['E_points'][0], rtol=1e-10,
                       atol=1e-10 * np.abs(g96['E_points']).max())


def test_autotuned_team_size(cuda, port):
    """team_warps='tune': the measured choice (one of 1, 2, 4, 8) is cached per
    device and problem size, and the traces it gives match the oracle."""
    from traceon_b200 import autotune
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.tracing import Tracer
    from traceon_b200 import geometry as G
    from oracle.oracle import EM, hermite_plane_crossing
    autotune.clear()
    q, jac, pos = _geometry_field(cuda, port)
    field = FieldRadialBEM(EffectivePointCharges(q, jac, pos))
    p0, v0 = G.electron_beam(40, 5)
    tr = Tracer(field, G.LENS_BOUNDS)
    plane, _, status, _ = tr.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=1e-10, team_warps='tune')
    assert np.all(status == cuda.TRACE_EXITED)
    tab = autotune.table()
    keys = [k for k in tab if k[0] == 'bem_team_warps' and len(k) == 4]
    assert len(keys) == 1 and tab[keys[0]] in autotune.TEAM_CANDIDATES
    timings = tab[keys[0] + ('times_ms',)]
    assert set(timings) == set(autotune.TEAM_CANDIDATES)
    tr.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=1e-10, team_warps='tune')  # served from the table
    assert autotune.table() == tab
    for i in range(0, 40, 13):
        t, s = port.trace_bem(p0[i], v0[i], EM, q, jac, pos, G.LENS_BOUNDS, 1e-10)
        h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
        assert np.max(np.abs(plane[i, 1:4] - h[:3])) < 1e-12


def test_current_rings_vs_oracle(cuda, port):
    """Current-ring field (radial.c:55-83) at many points through the device
    API and the compat entry point, and the current rings' axial derivatives
    (radial.c:85-103), against the oracle."""
    import torch
    from test_oracle import _coil_rings
    I, jac, pos = _coil_rings(5, n=40)
    rng = np.random.default_rng(6)
    M = 300
    pts = np.stack([rng.uniform(0, 2e-3, M), rng.uniform(-1e-3, 1e-3, M), rng.uniform(-8e-3, 8e-3, M)], 1)
    src = cuda.dev_pack_current_sources(cuda.to_dev(I, torch.float64), cuda.to_dev(jac, torch.float64),
                                        cuda.to_dev(pos, torch.float64))
    H = cuda.dev_current_field_points(cuda.to_dev(pts, torch.float64), src).cpu().numpy()
    H_or = np.array([port.current_field_radial(p, I, jac, pos) for p in pts])
    assert np.max(np.abs(H - H_or)) < 1e-11 * np.max(np.abs(H_or))
    for p in pts[:5]:
        h = cuda.current_field_radial(p, I, jac, pos)
        assert np.max(np.abs(h - port.current_field_radial(p, I, jac, pos))) < 1e-11 * np.max(np.abs(H_or))
    z = np.linspace(-8e-3, 8e-3, 101)
    d = cuda.dev_axial_derivatives(cuda.to_dev(z, torch.float64), src, current=True).cpu().numpy()
    d_or = port.current_axial_derivatives_radial(z, I, jac, pos)
    for c in range(d_or.shape[1]):
        assert np.max(np.abs(d[:, c] - d_or[:, c])) < 1e-10 * np.max(np.abs(d_or[:, c]))
