"""The combined electro-magnetostatic workload at reduced size: the einzel
lens inside the iron pole piece of a magnetic lens with four coils
(geometry.combined_lens).  Charges of both systems against the oracle's own
fill and LAPACK solves (the magnetizable right-hand side from the oracle's
current-ring field, solver.py:128-144), and the surrogate extended to the
magnetic field: its field H against the exact BEM field, and 5 keV electrons
traced through E + B against the oracle's FP64 BEM trace."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VOLTS = np.array([0.0, 3000.0, 0.0])


@pytest.fixture(scope='module')
def combined(cuda, port):
    from traceon_b200 import geometry as G
    from traceon_b200 import backend as B
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.field import EffectivePointCharges
    from traceon_b200.solver import ElectrostaticSolverRadial, MagnetostaticSolverRadial
    cl = G.combined_lens(3, n_elec=450, n_mag=360)
    geo = cl.geometry
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names[:3], VOLTS)})
    exc.add_magnetizable(pole=1000.0)
    I, cjac, cpos = cl.coil_sources()
    se = ElectrostaticSolverRadial(exc)
    sm = MagnetostaticSolverRadial(exc, current_point_charges=EffectivePointCharges(I, cjac, cpos))
    fe, fm = se.solve_matrix()[0], sm.solve_matrix()[0]
    # the oracle's charges
    Ae = port.matrix(se.vertices, se.excitation_types, se.excitation_values, threads=8)
    qe = np.linalg.solve(Ae, se.excitation_values)
    Am = port.matrix(sm.vertices, sm.excitation_types, sm.excitation_values, threads=8)
    Fm = np.zeros(len(sm.vertices))
    for i in range(len(Fm)):
        n = port.higher_order_normal_radial(0.0, sm.vertices[i])
        H = port.current_field_radial(sm.get_center_of_element(i), I, cjac, cpos)
        Fm[i] = -B.flux_density_to_charge_factor(1000.0) * (H[0] * n[0] + H[2] * n[1])
    qm = np.linalg.solve(Am, Fm)
    return cl, exc, se, sm, fe, fm, qe, qm, Fm, (I, cjac, cpos)


def test_combined_charges_vs_oracle(combined):
    """The device right-hand side of the magnetizable rows (one launch) and
    the charges of both systems against the oracle."""
    cl, exc, se, sm, fe, fm, qe, qm, Fm, coils = combined
    F_gpu = sm.get_right_hand_side()
    assert np.max(np.abs(F_gpu - Fm)) <= 1e-11 * np.max(np.abs(Fm))
    for got, want in ((fe.electrostatic_point_charges.charges, qe), (fm.magnetostatic_point_charges.charges, qm)):
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-10


@pytest.fixture(scope='module')
def combined_surrogate(combined):
    from traceon_b200.surrogate import SurrogateTrainer, FieldSurrogate
    cl, exc, se, sm, fe, fm, qe, qm, Fm, coils = combined
    geo = cl.geometry
    tr = SurrogateTrainer(geo, electrodes=geo.names[:3], magnetizable={'pole': 1000.0}, coils=cl)
    model, info = tr.train(n_samples=1 << 19, steps=6000, batch=8192, seed=0)
    strengths = np.concatenate([VOLTS, cl.coil_current])
    fs = FieldSurrogate(model, tr.fields, tr.z, tr.tabs, strengths, geo.segments, engine='tc')
    return tr, model, info, fs


def test_combined_surrogate_fields(combined, combined_surrogate):
    """The unit fields superposed with the excitation's strengths reproduce
    the directly solved magnetic field (linearity), and the surrogate's H is
    closer to the exact BEM H than the magnetic axial series alone, off the
    axis."""
    import torch
    from traceon_b200 import backend as B
    cl, exc, se, sm, fe, fm, qe, qm, Fm, coils = combined
    tr, model, info, fs = combined_surrogate
    assert model.n_el == 3 and model.n_coils == 4
    rng = np.random.default_rng(6)
    pts = np.stack([rng.uniform(0.2e-3, 0.8e-3, 1500), np.zeros(1500), rng.uniform(-8e-3, 8e-3, 1500)], 1)
    H_direct = fm.magnetostatic_field_at_points(pts)
    pt = B.to_dev(pts, torch.float64)
    _, H_bem = B.dev_field_points(pt, fs.mag_sources, False, True)
    H_bem = (H_bem + B.dev_current_field_points(pt, fs.cur_sources)).cpu().numpy()
    assert np.max(np.abs(H_bem - H_direct)) < 1e-9 * np.max(np.abs(H_direct))
    E, H, used = fs.kernel_field_at_points(pts, magnetic=True)
    _, H_ax = B.dev_axial_field_points(pt, fs.zt, fs.mag_table)
    H_ax = H_ax.cpu().numpy()
    ok = used == 0
    assert ok.sum() > 1000
    assert np.abs(H - H_bem)[ok].max() < 0.2 * np.abs(H_ax - H_bem)[ok].max()


def test_combined_surrogate_traces_vs_oracle(combined, combined_surrogate, port):
    """5 keV electrons (r0 <= 0.2 mm) through E + B: the surrogate tracer's
    exit-plane crossings within 1 nm of the oracle's FP64 BEM trace with the
    oracle's charges and the same coils; the magnetic lens turns the beam."""
    from traceon_b200 import geometry as G
    from oracle.oracle import EM, hermite_plane_crossing
    cl, exc, se, sm, fe, fm, qe, qm, Fm, (I, cjac, cpos) = combined
    tr, model, info, fs = combined_surrogate
    p0, v0 = G.combined_beam(8, 4)
    plane, final, status, counters = fs.trace_endpoints(p0, v0, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
    assert (status == 0).all()
    jac_e, pos_e = port.fill_jacobian_buffer_radial(se.vertices)
    jac_m, pos_m = port.fill_jacobian_buffer_radial(sm.vertices)
    err, turn = [], 0.0
    for i in range(len(p0)):
        t, s = port.trace_bem(p0[i], v0[i], EM, qe, jac_e, pos_e, G.LENS_BOUNDS, 1e-10, mag=(qm, jac_m, pos_m),
                              current=(I, cjac, cpos))
        h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
        err.append(np.max(np.abs(plane[i, 1:3] - h[:2])))
        turn = max(turn, abs(h[1]))
    assert max(err) < 1e-9
    assert turn > 1e-6
