"""The drop-in boundary exercised through the reference's own ctypes shim.

The reference loads its C backend from traceon/backend/traceon_backend.so
(traceon/backend/__init__.py:23-55), binds every entry of its
`backend_functions` table at import time (:287-353) and wraps them
(:355-780).  This test copies the reference package, unmodified, to a
temporary directory, puts libtraceon_b200.so at that path, and imports it in
a child process: the import itself resolves every table entry against this
library.  The child then calls the host-evaluated entry points through the
reference's own wrappers -- elliptic integrals, element geometry, ring
kernels, the QUADPACK self integrals over this library's exported
integrands (scipy LowLevelCallable), the axial-series lookups and the plane
crossing -- and the same child run against the reference's backend compiled
from its own sources (oracle/_ref, no fast-math) gives the expected values.
The array entry points run on the GPU and are covered by the GPU tests.

Needs the reference sources (TRACEON_REF_SRC, default /root/reference); it
is skipped where they are absent."""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = os.environ.get('TRACEON_REF_SRC', '/root/reference')
OURS = os.path.join(REPO, 'traceon_b200', 'libtraceon_b200.so')
REF_LIB = os.path.join(REPO, 'oracle', '_ref', 'libtraceon_ref_strict.so')

CHILD = r'''
import json, sys, types
import numpy as np
for name in ('meshio', 'matplotlib', 'matplotlib.pyplot'):
    sys.modules.setdefault(name, types.ModuleType(name))
sys.path.insert(0, sys.argv[1])
import traceon.backend as RB

out = {'lib': RB.backend_lib._name,
       'constants': [RB.TRACING_BLOCK_SIZE, RB.DERIV_2D_MAX, RB.N_QUAD_2D, RB.N_TRIANGLE_QUAD, RB.NU_MAX, RB.M_MAX]}
p = np.array([1e-30, 1e-12, 1e-6, 0.01, 0.3, 0.7, 0.999999])
out['ellipkm1'] = RB.ellipkm1(p).tolist()
out['ellipem1'] = RB.ellipem1(p).tolist()
out['ellipk'] = RB.ellipk(p).tolist()
out['ellipe'] = RB.ellipe(p).tolist()
line = np.array([[1.0e-3, 0.0, -1.0e-3], [1.2e-3, 0.0, -0.6e-3], [1.05e-3, 0.0, -0.87e-3], [1.12e-3, 0.0, -0.72e-3]])
out['normal_2d'] = RB.normal_2d(np.array([1.0, 2.0]), np.array([2.0, 3.5])).tolist()
out['higher_order_normal'] = [RB.higher_order_normal_radial(a, line).tolist() for a in (-0.7, 0.0, 0.4)]
out['pos_jac'] = [list(map(float, np.concatenate([np.ravel(x) for x in RB.position_and_jacobian_radial(a, line[0], line[2], line[3], line[1])])))
                  for a in (-1.0, -0.2, 0.9)]
out['delta_pos_jac'] = [list(map(float, np.concatenate([np.ravel(x) for x in RB.delta_position_and_jacobian_radial(a, line[0], line[2], line[3], line[1])])))
                        for a in (-0.5, 0.3)]
rings = [(1e-3, 0.2e-3, 0.3e-3, -0.1e-3), (0.5e-3, -1e-3, 1e-5, 2e-6), (2e-3, 0.0, -0.4e-3, 1.5e-3)]
out['ring'] = [[RB.potential_radial_ring(*r), RB.dr1_potential_radial_ring(*r), RB.dz1_potential_radial_ring(*r)]
               for r in rings]
out['charge_radial'] = RB.charge_radial(line, 2.5)
out['flux_factor'] = [RB.flux_density_to_charge_factor(K) for K in (2.0, 10.0, 1000.0)]
out['current_ring'] = RB.current_field_radial_ring(1e-3, 0.5e-3, 3e-3, 0.2e-3).tolist()
out['current_axial'] = RB.current_potential_axial_radial_ring(0.5e-3, 3e-3, 1e-3)
out['self_potential'] = RB.self_potential_radial(line)
out['self_field_dot_normal'] = RB.self_field_dot_normal_radial(line, 5.0)
rng = np.random.default_rng(0)
z = np.linspace(-1e-3, 1e-3, 11)
coeffs = rng.normal(size=(10, RB.DERIV_2D_MAX, 6))
pt = np.array([0.1e-3, 0.05e-3, 0.13e-3])
out['potential_derivs'] = RB.potential_radial_derivs(pt, z, coeffs)
out['field_derivs'] = RB.field_radial_derivs(pt, z, coeffs).tolist()
t = np.linspace(0, 1, 50)
traj = np.stack([np.sin(t), np.cos(t), t - 0.37, np.cos(t), -np.sin(t), np.ones_like(t)], 1)
out['plane'] = RB.plane_intersection(traj, np.array([0.0, 0.0, 0.2]), np.array([0.0, 0.0, 1.0])).tolist()
try:
    RB.plane_intersection(traj, np.array([0.0, 0.0, 5.0]), np.array([0.0, 0.0, 1.0]))
    out['no_crossing'] = 'found'
except ValueError:
    out['no_crossing'] = 'ValueError'
print(json.dumps(out))
'''


def _run_shim(lib, tmp):
    dst = os.path.join(tmp, os.path.basename(lib))
    shutil.copytree(os.path.join(REF_SRC, 'traceon'), os.path.join(dst, 'traceon'))
    so = os.path.join(dst, 'traceon', 'backend', 'traceon_backend.so')
    os.symlink(lib, so)  # the path the reference's loader tries first
    r = subprocess.run([sys.executable, '-c', CHILD, dst], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert os.path.realpath(out['lib']) == os.path.realpath(lib) or out['lib'] == so
    return out


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_SRC, 'traceon', 'backend')),
                    reason='reference sources not present')
def test_reference_backend_module_binds_this_library():
    if not os.path.exists(OURS):
        pytest.skip('libtraceon_b200.so not built')
    if not os.path.exists(REF_LIB):
        pytest.skip('oracle/_ref not built')
    tmp = tempfile.mkdtemp(prefix='traceon_shim_')
    try:
        ours = _run_shim(OURS, tmp)
        ref = _run_shim(REF_LIB, tmp)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    assert ours['constants'] == ref['constants'] == [100000, 9, 16, 12, 4, 8]
    assert ours['no_crossing'] == ref['no_crossing'] == 'ValueError'
    tol = {'ellipk': 1e-15, 'ellipe': 1e-15, 'self_potential': 1e-9, 'self_field_dot_normal': 1e-9}
    for key, want in ref.items():
        if key in ('lib', 'constants', 'no_crossing'):
            continue
        a, b = np.asarray(ours[key], dtype=float), np.asarray(want, dtype=float)
        scale = max(np.max(np.abs(b)), 1e-300)
        assert np.max(np.abs(a - b)) <= tol.get(key, 1e-14) * scale, (key, a, b)
