"""The C-ABI library builds, loads and exports every symbol that
include/traceon_b200.h declares (no GPU needed: nothing is computed)."""
import ctypes as C
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, 'include', 'traceon_b200.h')


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    funcs = set(re.findall(r'\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;', text))
    funcs -= {'sizeof'}
    consts = set(re.findall(r'extern\s+const\s+\w+\s+([A-Za-z_][A-Za-z0-9_]*)\s*;', text))
    return funcs, consts


def test_library_exports_header_symbols():
    from traceon_b200 import build
    lib_path = build.build()
    lib = C.CDLL(lib_path)
    funcs, consts = declared_symbols()
    assert len(funcs) > 40
    missing = [f for f in sorted(funcs | consts) if not hasattr(lib, f)]
    assert not missing, missing


def test_constants_match_reference():
    from traceon_b200 import backend as B
    # traceon/backend/__init__.py:58-66 reads these with in_dll
    assert B.TRACING_BLOCK_SIZE == 100000
    assert B.DERIV_2D_MAX == 9
    assert B.N_QUAD_2D == 16
    assert B.N_TRIANGLE_QUAD == 12
    assert (B.NU_MAX, B.M_MAX) == (4, 8)


def test_reference_table_resolves():
    """Every name in the reference's backend_functions table
    (traceon/backend/__init__.py:287-328) resolves in this library."""
    from traceon_b200 import backend as B
    names = ['kronrod_adaptive', 'ellipkm1', 'ellipk', 'ellipem1', 'ellipe', 'normal_2d',
             'higher_order_normal_radial', 'normal_3d', 'position_and_jacobian_3d', 'position_and_jacobian_radial',
             'delta_position_and_jacobian_radial', 'trace_particle', 'potential_radial_ring',
             'dr1_potential_radial_ring', 'dz1_potential_radial_ring', 'axial_derivatives_radial', 'potential_radial',
             'potential_radial_derivs', 'flux_density_to_charge_factor', 'charge_radial', 'field_radial',
             'field_radial_derivs', 'axial_coefficients_3d', 'fill_jacobian_buffer_current_three_d',
             'potential_3d_derivs', 'field_3d_derivs', 'current_potential_axial_radial_ring',
             'current_potential_axial', 'current_field_radial_ring', 'current_field_radial',
             'current_axial_derivatives_radial', 'fill_jacobian_buffer_radial', 'self_potential_radial',
             'self_field_dot_normal_radial', 'fill_matrix_radial', 'fill_jacobian_buffer_3d', 'plane_intersection',
             'triangle_areas', 'field_radial_traceable', 'field_radial_derivs_traceable']
    for n in names:
        assert hasattr(B.backend_lib, n), n


def test_host_scalars_match_oracle(port):
    """Scalar helpers evaluated on the host by the library's shared code."""
    import numpy as np
    from traceon_b200 import backend as B
    p = 10.0 ** -np.linspace(0.5, 80, 30)
    assert np.allclose(B.ellipkm1(p), port.ellipkm1(p), rtol=1e-15, atol=0)
    assert np.allclose(B.ellipem1(p), port.ellipem1(p), rtol=1e-15, atol=0)
    k = np.linspace(-1, 1, 40)[1:-1]
    assert np.allclose(B.ellipk(k), port.ellipk(k), rtol=1e-14, atol=0)
    assert np.allclose(B.ellipe(k), port.ellipe(k), rtol=1e-14, atol=0)
    rng = np.random.default_rng(0)
    for _ in range(50):
        r0, z0 = rng.uniform(1e-4, 2e-3), rng.uniform(-2e-3, 2e-3)
        dr, dz = rng.uniform(-5e-4, 5e-4), rng.uniform(-5e-4, 5e-4)
        assert np.isclose(B.potential_radial_ring(r0, z0, dr, dz), port.potential_radial_ring(r0, z0, dr, dz),
                          rtol=1e-13, atol=0)
        assert np.isclose(B.dr1_potential_radial_ring(r0, z0, dr, dz), port.dr1_potential_radial_ring(r0, z0, dr, dz),
                          rtol=1e-11, atol=0)
        assert np.isclose(B.dz1_potential_radial_ring(r0, z0, dr, dz), port.dz1_potential_radial_ring(r0, z0, dr, dz),
                          rtol=1e-11, atol=0)
    from traceon_b200.geometry import einzel_lens
    v = einzel_lens(30).vertices
    for x in v:
        assert np.allclose(B.higher_order_normal_radial(0.0, x), port.higher_order_normal_radial(0.0, x), atol=1e-15)
        assert np.isclose(B.charge_radial(x, 2.0), port.charge_radial(x, 2.0), rtol=1e-14)
        j, pos = B.position_and_jacobian_radial(0.3, x[0], x[2], x[3], x[1])
        assert np.isfinite(j) and pos.shape == (2,)


def test_plane_intersection_host():
    import numpy as np
    from traceon_b200 import backend as B
    s = np.zeros((3, 6))
    s[:, 2] = [0.0, 1.0, 2.0]
    s[:, 0] = [0.0, 1.0, 4.0]
    out = B.plane_intersection(s, np.array([0, 0, 1.5]), np.array([0, 0, 1.0]))
    assert np.isclose(out[0], 2.5) and np.isclose(out[2], 1.5)
    import pytest
    with pytest.raises(ValueError):
        B.plane_intersection(s, np.array([0, 0, 5.0]), np.array([0, 0, 1.0]))
