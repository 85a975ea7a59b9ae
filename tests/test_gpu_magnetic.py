"""Tracing through combined electrostatic and magnetostatic fields: the GPU
tracer's Lorentz force (E + v x mu0 H) with the electrostatic charges, the
magnetostatic charges of a magnetizable pole piece and the current rings
that magnetise it (field_radial_traceable, traceon/backend/tracing.c:125-165;
the force, tracing.c:20-57), against the CPU oracle's trace of the same
configuration with charges from its own fill and LAPACK solves."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _combined_lens(n_lens=300, n_pole=160):
    from traceon_b200 import geometry as G
    lens = G.einzel_lens(n_lens)
    pole = G.aperture_tube(2.5e-3, 3.0e-3, -2.0e-3, 2.0e-3, n_pole)
    verts = np.concatenate([lens.vertices, pole])
    idx = np.concatenate([lens.electrode_index, np.full(len(pole), 3)])
    return G.LensGeometry(verts, idx, lens.names + ['pole'])


def test_trace_electric_and_magnetic_fields_vs_oracle(cuda, port):
    from traceon_b200 import geometry as G
    from traceon_b200 import backend as B
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.field import EffectivePointCharges
    from traceon_b200.solver import ElectrostaticSolverRadial, MagnetostaticSolverRadial
    from traceon_b200.tracing import Tracer
    from oracle.oracle import EM, hermite_plane_crossing
    from test_oracle import _coil_rings
    geo = _combined_lens()
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(ground_in=0.0, lens=1200.0, ground_out=0.0)
    exc.add_magnetizable(pole=1000.0)
    I, cjac, cpos = _coil_rings(11, n=12)
    # current densities x area weights: ~70 A-turns in all, about 0.01 T on
    # the axis -- a moderate magnetic lens for 1 keV electrons
    I = I * 2.5e6
    se = ElectrostaticSolverRadial(exc)
    sm = MagnetostaticSolverRadial(exc, current_point_charges=EffectivePointCharges(I, cjac, cpos))
    field = se.solve_matrix()[0] + sm.solve_matrix()[0]

    # oracle charges: its own fills and LAPACK; the magnetizable right-hand
    # side from its own current-ring field (solver.py:128-144)
    Ae = port.matrix(se.vertices, se.excitation_types, se.excitation_values, threads=8)
    qe = np.linalg.solve(Ae, se.excitation_values)
    Am = port.matrix(sm.vertices, sm.excitation_types, sm.excitation_values, threads=8)
    normals = np.array([port.higher_order_normal_radial(0.0, v) for v in sm.vertices])
    Fm = np.zeros(len(sm.vertices))
    for i in range(len(Fm)):
        c = sm.get_center_of_element(i)
        H = port.current_field_radial(c, I, cjac, cpos)
        Fm[i] = -B.flux_density_to_charge_factor(sm.excitation_values[i]) * (H[0] * normals[i][0] +
                                                                            H[2] * normals[i][1])
    qm_ = np.linalg.solve(Am, Fm)
    jac_e, pos_e = port.fill_jacobian_buffer_radial(se.vertices)
    jac_m, pos_m = port.fill_jacobian_buffer_radial(sm.vertices)

    p0, v0 = G.electron_beam(6, 3, r_max=0.3e-3, angle_max=10e-3)
    plane, final, status, counters = Tracer(field, G.LENS_BOUNDS).trace_endpoints(p0, v0, G.LENS_EXIT_Z,
                                                                                  atol=1e-10)
    assert (status == 0).all()
    rot = 0.0
    for i in range(len(p0)):
        t, s = port.trace_bem(p0[i], v0[i], EM, qe, jac_e, pos_e, G.LENS_BOUNDS, 1e-10,
                              mag=(qm_, jac_m, pos_m), current=(I, cjac, cpos))
        h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
        assert np.max(np.abs(plane[i, 1:3] - h[:2])) < 1e-11, i
        rot = max(rot, abs(h[1]))
    assert rot > 1e-6  # the magnetic lens turned the beam out of its start plane
