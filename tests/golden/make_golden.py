"""Generate the golden vectors in tests/golden/ from the reference Python package.

Run in a container that has the reference sources (default
/root/reference; override with TRACEON_REF_SRC):

    python tests/golden/make_golden.py

The script copies the reference tree to a temporary directory, compiles its C
backend there with the shipped flags (setup.py:8), stubs the two imports the
path does not use (meshio: mesher.py:10, file I/O only; matplotlib), imports
``traceon`` and records its outputs through its own public API.  Nothing here
runs on a GPU; the .npz files it writes are committed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SRC = os.environ.get('TRACEON_REF_SRC', '/root/reference')


def import_reference():
    tmp = tempfile.mkdtemp(prefix='traceon_ref_')
    dst = os.path.join(tmp, 'traceon_ref')
    shutil.copytree(os.path.join(REF_SRC, 'traceon'), os.path.join(dst, 'traceon'))
    be = os.path.join(dst, 'traceon', 'backend')
    subprocess.check_call(['gcc', '-O3', '-mavx', '-ffast-math', '-DNDEBUG', '-fPIC', '-shared', '-std=gnu99',
                           '-o', os.path.join(be, 'traceon_backend.so'), os.path.join(be, 'traceon-backend.c'),
                           '-lm'], stderr=subprocess.DEVNULL)
    for name in ('meshio', 'matplotlib', 'matplotlib.pyplot'):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, dst)
    os.environ['TRACEON_THREADS'] = '8'
    import traceon  # noqa: F401
    import traceon.logging as logging
    logging.set_log_level(logging.LogLevel.SILENT)
    return tmp


def main():
    tmp = import_reference()
    try:
        import traceon.backend as B
        import traceon.excitation as E
        import traceon.mesher as M
        import traceon.solver as S
        import traceon.tracing as T
        from traceon.field import FieldRadialAxial

        sys.path.insert(0, REPO)
        from traceon_b200 import geometry as G

        rng = np.random.default_rng(20261203)

        # ---- elliptic integrals: elliptic.c:9-75
        p = np.concatenate([10.0 ** -np.linspace(1, 100, 25), np.linspace(0, 1, 40)[1:-1]])
        k = np.linspace(-1, 1, 40)[1:-1]
        np.savez(os.path.join(HERE, 'elliptic.npz'), p=p, ellipkm1=B.ellipkm1(p), ellipem1=B.ellipem1(p),
                 k=k, ellipk=B.ellipk(k), ellipe=B.ellipe(k))

        # ---- ring kernels: radial_ring.c:21-53 at random and near-singular pairs
        n = 200
        r0 = rng.uniform(1e-4, 3e-3, n)
        z0 = rng.uniform(-5e-3, 5e-3, n)
        scale = 10.0 ** rng.uniform(-9, -3, n)
        dr = rng.uniform(-1, 1, n) * scale
        dz = rng.uniform(-1, 1, n) * scale
        dr = np.maximum(dr, -r0 + 1e-6)
        pot = np.array([B.potential_radial_ring(*a) for a in zip(r0, z0, dr, dz)])
        dr1 = np.array([B.dr1_potential_radial_ring(*a) for a in zip(r0, z0, dr, dz)])
        dz1 = np.array([B.dz1_potential_radial_ring(*a) for a in zip(r0, z0, dr, dz)])
        np.savez(os.path.join(HERE, 'rings.npz'), r0=r0, z0=z0, dr=dr, dz=dz, pot=pot, dr1=dr1, dz1=dz1)

        # ---- a small einzel lens through the public API
        geo = G.einzel_lens(96)
        volts = np.array([0.0, 1500.0, 0.0])
        verts = geo.vertices
        N = len(verts)
        points = verts.reshape(-1, 3)
        lines = np.arange(4 * N).reshape(N, 4)
        phys = {name: np.nonzero(geo.electrode_index == e)[0] for e, name in enumerate(geo.names)}
        mesh = M.Mesh(points=points, lines=lines, physical_to_lines=phys, ensure_outward_normals=False)
        exc = E.Excitation(mesh, E.Symmetry.RADIAL)
        exc.add_voltage(**{name: float(v) for name, v in zip(geo.names, volts)})
        active, _ = exc.get_electrostatic_active_elements()
        # Mesh() merges duplicate points after truncating 16 mantissa bits
        # (mesher.py:262-290); use the vertices the solver actually sees.
        assert np.array_equal(active, verts)
        verts = np.ascontiguousarray(active)

        jac, pos = B.fill_jacobian_buffer_radial(verts)
        normals = np.array([B.higher_order_normal_radial(0.0, v) for v in verts])
        types_ = np.ones(N, dtype=np.uint8)
        values = geo.voltages_to_values(volts)
        fill = np.zeros((N, N))
        B.fill_matrix_radial(fill, verts, types_, values, jac, pos, 0, N - 1)
        diag = np.array([B.self_potential_radial(v) for v in verts])

        solver = S.ElectrostaticSolverRadial(exc)
        matrix = solver.get_matrix()
        field = S.solve_direct(exc)
        charges = field.electrostatic_point_charges.charges

        sup = S.solve_direct_superposition(exc)
        sup_charges = np.array([sup[name].electrostatic_point_charges.charges for name in geo.names])

        M_pts = 64
        pts = np.stack([rng.uniform(0, 0.9e-3, M_pts) * np.cos(th := rng.uniform(0, 2 * np.pi, M_pts)),
                        rng.uniform(0, 0.9e-3, M_pts) * 0 + 0, rng.uniform(-8e-3, 8e-3, M_pts)], axis=1)
        pts[:, 1] = np.abs(pts[:, 0]) * np.sin(th)
        E_pts = np.array([field.electrostatic_field_at_point(p) for p in pts])
        V_pts = np.array([field.electrostatic_potential_at_point(p) for p in pts])

        z_ax = np.linspace(-9.95e-3, 9.95e-3, 200)
        derivs = field.get_electrostatic_axial_potential_derivatives(z_ax)
        axial = FieldRadialAxial(field, z_ax[0], z_ax[-1], N=len(z_ax))
        coeffs = axial.electrostatic_coeffs
        ax_pts = np.stack([rng.uniform(0, 0.2e-3, 32), np.zeros(32), rng.uniform(-9.9e-3, 9.9e-3, 32)], axis=1)
        E_ax = np.array([axial.electrostatic_field_at_point(p) for p in ax_pts])
        V_ax = np.array([axial.electrostatic_potential_at_point(p) for p in ax_pts])

        p0, v0 = G.electron_beam(3, 11)
        bounds = G.LENS_BOUNDS
        tracer = field.get_tracer(bounds)
        tracer_ax = axial.get_tracer(bounds)
        traces, traces_ax = {}, {}
        for i in range(3):
            t, s = tracer(p0[i], v0[i], atol=1e-10)
            traces[f'bem_t{i}'], traces[f'bem_s{i}'] = t, s
            t, s = tracer_ax(p0[i], v0[i], atol=1e-10)
            traces[f'ax_t{i}'], traces[f'ax_s{i}'] = t, s
        cross = np.array([T.xy_plane_intersection(traces[f'bem_s{i}'], G.LENS_EXIT_Z) for i in range(3)])
        cross_ax = np.array([T.xy_plane_intersection(traces[f'ax_s{i}'], G.LENS_EXIT_Z) for i in range(3)])

        np.savez(os.path.join(HERE, 'lens96.npz'), vertices=verts, volts=volts, jac=jac, pos=pos, normals=normals,
                 fill=fill, diag=diag, matrix=matrix, charges=charges, sup_charges=sup_charges, points=pts,
                 E_points=E_pts, V_points=V_pts, z_axial=z_ax, derivs=derivs, coeffs=coeffs, axial_points=ax_pts,
                 E_axial=E_ax, V_axial=V_ax, p0=p0, v0=v0, bounds=bounds, cross=cross, cross_axial=cross_ax,
                 **traces)

        # ---- a dielectric row block (DIELECTRIC rows, radial.c:287-304;
        #      diagonal solver.py:239-244)
        d_verts = verts[:24]
        d_types = np.full(24, 3, dtype=np.uint8)
        d_values = np.full(24, 4.5)
        jd, pd = B.fill_jacobian_buffer_radial(d_verts)
        d_fill = np.zeros((24, 24))
        B.fill_matrix_radial(d_fill, d_verts, d_types, d_values, jd, pd, 0, 23)
        d_diag = np.array([B.self_field_dot_normal_radial(v, 4.5) - 1 for v in d_verts])
        np.savez(os.path.join(HERE, 'dielectric24.npz'), vertices=d_verts, values=d_values, fill=d_fill, diag=d_diag)
        print('golden vectors written to', HERE)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == '__main__':
    main()
