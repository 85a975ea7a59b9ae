"""Learned field surrogate for a radially symmetric lens.

The surrogate field of a lens with electrode voltages V is

    E(r, z) = E_axial(r, z; V) + sum_e V_e * C_e(r, z),
    C_e = S * rho^p * NN_e(features(r, z)),   rho = r / r_max,

where E_axial is the reference's axial series expansion (traceon/field.py,
FieldRadialAxial; radial.c:347-384) of the solved charges -- exact on the
axis, degrading away from it -- and NN is a 4 x 128 SiLU network that learns,
per electrode at 1 V, the difference between the exact BEM field
(radial.c:150-173) and that series.  The field is linear in the voltages, so
one network serves every voltage setting; the rho^p envelope makes the
correction vanish toward the axis where the series is already exact.  Near an
electrode (within `fallback_dist`) and outside the network's domain the
tracer falls back to the exact BEM sum.

Training data come from the GPU BEM evaluator itself (tb_field_radial_points)
and the GPU axial series (tb_axial_field_points); the network is trained on
the GPU by this library's BF16 / FP32-accumulate kernels (tb_mlp_*), with
Adam on FP32 master weights.  There is no reference counterpart; the
surrogate is checked against the FP64 BEM field and the FP64 BEM trace.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import backend as B

IN, H, OUT = 16, 128, 32
MAX_SOURCES = OUT // 3  # electrodes + coils, 3 outputs each
OFF = {}
_o = 0
for _name, _n in (('W1', H * IN), ('b1', H), ('W2', H * H), ('b2', H), ('W3', H * H), ('b3', H), ('W4', H * H),
                  ('b4', H), ('W5', OUT * H), ('b5', OUT)):
    OFF[_name] = (_o, _n)
    _o += _n
NPARAM = _o
LAYERS = [('W1', 'b1', IN, H), ('W2', 'b2', H, H), ('W3', 'b3', H, H), ('W4', 'b4', H, H), ('W5', 'b5', H, OUT)]

_lib = B.backend_lib
_vp, _i64, _f = C.c_void_p, C.c_int64, C.c_float
for _name, _args in {
    'tb_mlp_gemm': (_vp, _i64, C.c_int, _vp, _i64, C.c_int, _vp, _i64, _i64, _i64, _i64, C.c_int, _vp),
    'tb_mlp_bias_silu': (_vp, _vp, _vp, _vp, _i64, _i64, _vp),
    'tb_mlp_bias_out': (_vp, _vp, _vp, _i64, _i64, _vp),
    'tb_mlp_mse_grad': (_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _vp),
    'tb_mlp_silu_back': (_vp, _vp, _vp, _i64, _vp),
    'tb_mlp_colsum': (_vp, _vp, _i64, _i64, _vp),
    'tb_mlp_adam': (_vp, _vp, _vp, _vp, _vp, _i64, _f, _f, _f, _f, _i64, _vp),
    'tb_mlp_features': (_vp, _i64, C.c_double, C.c_double, C.c_double, _vp, _vp),
}.items():
    getattr(_lib, _name).argtypes = list(_args)
    getattr(_lib, _name).restype = C.c_int


class TbSurrogate(C.Structure):
    """tb_surrogate_t of include/traceon_b200.h"""
    _fields_ = [('weights_bf16', _vp), ('params_f32', _vp), ('r_max', C.c_double), ('z_c', C.c_double),
                ('z_half', C.c_double), ('z_lo', C.c_double), ('z_hi', C.c_double), ('n_electrodes', C.c_int),
                ('n_coils', C.c_int), ('strengths', C.c_double * MAX_SOURCES), ('scale', C.c_float * OUT),
                ('env_power', C.c_int), ('segments', _vp), ('n_segments', C.c_int), ('fallback_dist', C.c_double),
                ('engine', C.c_int)]


def _call(name, *args):
    r = getattr(_lib, name)(*args)
    if r != B.TB_OK:
        raise B.BackendError(f'{name} failed with status {r}')


def _s():
    return B._stream()


class MLP:
    """The network's parameters (FP32 master + BF16 copy) and Adam state on
    the device, with forward / backward passes built from tb_mlp_* kernels."""

    def __init__(self, seed=0, params=None):
        torch = B._torch()
        dev = B.device()
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(NPARAM, dtype=np.float32)
            for W, b, fan_in, fan_out in LAYERS:
                o, n = OFF[W]
                lim = math.sqrt(6.0 / fan_in) * (0.5 if W == 'W5' else 1.0)
                p[o:o + n] = rng.uniform(-lim, lim, n)
            params = p
        self.p = torch.as_tensor(np.asarray(params, dtype=np.float32), device=dev).contiguous()
        self.pb = self.p.to(torch.bfloat16)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_count = 0

    def _w(self, t, name):
        o, n = OFF[name]
        return t[o:o + n]

    def forward(self, X, keep=False):
        """X (M, 16) bf16 features -> (M, 32) fp32 outputs; with keep, also
        the pre-activations Z_l (fp32) and activations Y_l (bf16)."""
        torch = B._torch()
        M = X.shape[0]
        acts, pre = [X], []
        cur = X
        for W, b, fin, fout in LAYERS:
            Cm = torch.empty((M, fout), dtype=torch.float32, device=X.device)
            _call('tb_mlp_gemm', cur.data_ptr(), fin, 0, self._w(self.pb, W).data_ptr(), fin, 0, Cm.data_ptr(), fout,
                  M, fout, fin, 0, _s())
            if W != 'W5':
                Z = torch.empty_like(Cm) if keep else None
                Y = torch.empty((M, fout), dtype=torch.bfloat16, device=X.device)
                _call('tb_mlp_bias_silu', Cm.data_ptr(), self._w(self.p, b).data_ptr(), B._ptr(Z), Y.data_ptr(), M,
                      fout, _s())
                pre.append(Z)
                acts.append(Y)
                cur = Y
            else:
                out = torch.empty_like(Cm)
                _call('tb_mlp_bias_out', Cm.data_ptr(), self._w(self.p, b).data_ptr(), out.data_ptr(), M, fout, _s())
        return (out, pre, acts) if keep else out

    def loss_and_grad(self, X, T, n_out, w=None):
        """MSE over the first n_out outputs (rows weighted by w (M) if given);
        fills self.g, returns the loss (device scalar)."""
        torch = B._torch()
        M = X.shape[0]
        out, pre, acts = self.forward(X, keep=True)
        dY = torch.empty((M, OUT), dtype=torch.bfloat16, device=X.device)
        nblk = (M * OUT + 255) // 256
        part = torch.empty(nblk, dtype=torch.float32, device=X.device)
        _call('tb_mlp_mse_grad', out.data_ptr(), T.data_ptr(), B._ptr(w), dY.data_ptr(), part.data_ptr(), M, OUT,
              n_out, _s())
        g = dY
        for li in range(len(LAYERS) - 1, -1, -1):
            W, b, fin, fout = LAYERS[li]
            Xin = acts[li]
            # dW = g^T . Xin  (fout x fin), db = column sums of g
            _call('tb_mlp_gemm', g.data_ptr(), fout, 1, Xin.data_ptr(), fin, 1, self._w(self.g, W).data_ptr(), fin,
                  fout, fin, M, 0, _s())
            _call('tb_mlp_colsum', g.data_ptr(), self._w(self.g, b).data_ptr(), M, fout, _s())
            if li == 0:
                break
            # dA = g . W  (M x fin), then through SiLU of layer li-1
            dA = torch.empty((M, fin), dtype=torch.float32, device=X.device)
            _call('tb_mlp_gemm', g.data_ptr(), fout, 0, self._w(self.pb, W).data_ptr(), fin, 1, dA.data_ptr(), fin,
                  M, fin, fout, 0, _s())
            gz = torch.empty((M, fin), dtype=torch.bfloat16, device=X.device)
            _call('tb_mlp_silu_back', dA.data_ptr(), pre[li - 1].data_ptr(), gz.data_ptr(), M * fin, _s())
            g = gz
        return part.sum() / (M * n_out)

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        _call('tb_mlp_adam', self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
              self.pb.data_ptr(), NPARAM, lr, b1, b2, eps, self.step_count, _s())


def features(points_t, r_max, z_c, z_half):
    torch = B._torch()
    X = torch.empty((points_t.shape[0], IN), dtype=torch.bfloat16, device=points_t.device)
    _call('tb_mlp_features', points_t.data_ptr(), points_t.shape[0], r_max, z_c, z_half, X.data_ptr(), _s())
    return X


class SurrogateModel:
    """Network + normalisation of a surrogate for one lens geometry.  Its
    field sources are n_electrodes electrodes (per unit voltage; outputs
    (phi, E_r, E_z)) followed by n_coils current coils (per unit current;
    outputs (magnetostatic potential, H_r, H_z))."""

    def __init__(self, n_electrodes, r_max, z_lo, z_hi, scale, env_power=8, params=None, seed=0, n_coils=0):
        self.n_el = int(n_electrodes)
        self.n_coils = int(n_coils)
        if not 1 <= self.n_el + self.n_coils <= MAX_SOURCES:
            raise ValueError(f'1 to {MAX_SOURCES} field sources (electrodes + coils)')
        self.r_max, self.z_lo, self.z_hi = float(r_max), float(z_lo), float(z_hi)
        self.z_c, self.z_half = 0.5 * (z_lo + z_hi), 0.5 * (z_hi - z_lo)
        self.scale = np.asarray(scale, dtype=np.float32)
        self.env_power = int(env_power)
        self.mlp = MLP(seed=seed, params=params)

    @property
    def n_src(self):
        return self.n_el + self.n_coils

    def n_out(self):
        return 3 * self.n_src

    def envelope(self, r):
        """(M, n_out) envelope: rho^p for the potential and the axial
        component, rho^(p+1) for the radial component."""
        rho = np.asarray(r) / self.r_max
        e = rho ** self.env_power
        cols = [e, e * rho, e] * self.n_src
        return np.stack(cols, axis=1)

    def state(self):
        return {'params': self.mlp.p.cpu().numpy(), 'n_el': self.n_el, 'n_coils': self.n_coils, 'r_max': self.r_max,
                'z_lo': self.z_lo, 'z_hi': self.z_hi, 'scale': self.scale, 'env_power': self.env_power}

    def save(self, path):
        np.savez(path, **self.state())

    @staticmethod
    def load(path):
        d = np.load(path)
        return SurrogateModel(int(d['n_el']), float(d['r_max']), float(d['z_lo']), float(d['z_hi']), d['scale'],
                              int(d['env_power']), params=d['params'], n_coils=int(d['n_coils']))

    def predict_residual(self, points):
        """Per-source corrections (M, n_src, 3) at unit strength: (phi, E_r,
        E_z) of the electrodes, then (potential, H_r, H_z) of the coils."""
        torch = B._torch()
        pts = B.to_dev(np.asarray(points, dtype=np.float64).reshape(-1, 3), torch.float64)
        y = self.mlp.forward(features(pts, self.r_max, self.z_c, self.z_half)).cpu().numpy()[:, :self.n_out()]
        r = np.hypot(points[:, 0], points[:, 1])
        return (y * self.scale[:self.n_out()] * self.envelope(r)).reshape(-1, self.n_src, 3)


# ---------------------------------------------------------------- data
def unit_fields(geo, electrodes=None):
    """FieldRadialBEM of every electrode (default: all names of geo) at 1 V,
    the others at 0 V, from one factorisation (the superposition solve of
    traceon/solver.py:364-400)."""
    from .excitation import Excitation, Mesh
    from .solver import ElectrostaticSolverRadial
    names = list(geo.names) if electrodes is None else list(electrodes)
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: 1.0 for n in names})
    solver = ElectrostaticSolverRadial(exc)
    F = np.zeros((len(names), len(solver.vertices)))
    for k, n in enumerate(names):
        F[k, solver.names[n]] = 1.0
    return solver.solve_matrix(F)


def unit_coil_fields(geo, magnetizable, coils):
    """FieldRadialBEM of every coil at 1 A-turn, the others off: the current
    ring plus the magnetostatic charges it induces on the magnetizable
    electrodes (`magnetizable`: {name: mu_r}), all right-hand sides solved
    with one factorisation (MagnetostaticSolverRadial, solver.py:267-353).
    coils: an object with coil_sources(currents) -> (current densities,
    jac (N, 12), pos (N, 12, 3)) (geometry.CombinedLens)."""
    from .excitation import Excitation, Mesh
    from .field import EffectivePointCharges, FieldRadialBEM
    from .solver import MagnetostaticSolverRadial
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_magnetizable(**magnetizable)
    n = len(coils.coil_r)
    rings = []
    F = []
    for c in range(n):
        cur = np.zeros(n)
        cur[c] = 1.0
        I, jac, pos = coils.coil_sources(cur)
        one = EffectivePointCharges(I[c:c + 1], jac[c:c + 1], pos[c:c + 1])
        rings.append(one)
        F.append(MagnetostaticSolverRadial(exc, current_point_charges=one).get_right_hand_side())
    solver = MagnetostaticSolverRadial(exc)
    X = solver.solve_charges_device(np.array(F)).cpu().numpy()
    jac, pos = solver.jacobians_and_positions()
    return [FieldRadialBEM(magnetostatic_point_charges=EffectivePointCharges(x, jac, pos), current_point_charges=r)
            for x, r in zip(X, rings)]


def _field_table(f, zt, dz):
    """Axial coefficient table (nz-1, 9, 6) of a unit field: its electrostatic
    charges, or for a coil its magnetostatic charges plus its current ring
    (FieldRadialAxial's magnetostatic table, traceon/field.py:971-991)."""
    if len(f.electrostatic_point_charges):
        d = B.dev_axial_derivatives(zt, f.electrostatic_point_charges.device_sources())
    else:
        d = B.dev_axial_derivatives(zt, f.magnetostatic_point_charges.device_sources())
        d = d + B.dev_axial_derivatives(zt, f.current_point_charges.device_sources(), current=True)
    return B.dev_axial_coefficients(d, dz)


def axial_tables(fields, z_lo, z_hi, nz):
    """Axial coefficient tables (nz-1, 9, 6) of each unit field on the grid."""
    torch = B._torch()
    z = np.linspace(z_lo, z_hi, nz)
    zt = B.to_dev(z, torch.float64)
    return z, zt, [_field_table(f, zt, z[1] - z[0]) for f in fields]


def _segment_distance(points_rz, segs):
    d = np.full(len(points_rz), np.inf)
    for r0, z0, r1, z1 in segs:
        a = np.array([r0, z0])
        u = np.array([r1 - r0, z1 - z0])
        L2 = u @ u
        t = np.clip(((points_rz - a) @ u) / L2, 0, 1) if L2 > 0 else np.zeros(len(points_rz))
        q = a + t[:, None] * u
        d = np.minimum(d, np.linalg.norm(points_rz - q, axis=1))
    return d


def sample_points(n, seed, r_min, r_max, z_lo, z_hi, segs, exclude):
    """n points uniform in r in [r_min, r_max], z in [z_lo, z_hi], at azimuth
    0, farther than `exclude` from every electrode segment."""
    rng = np.random.default_rng(seed)
    out = []
    got = 0
    while got < n:
        m = int((n - got) * 1.3) + 1024
        r = rng.uniform(r_min, r_max, m)
        z = rng.uniform(z_lo, z_hi, m)
        keep = _segment_distance(np.stack([r, z], 1), segs) > exclude
        out.append(np.stack([r[keep], np.zeros(keep.sum()), z[keep]], 1))
        got += keep.sum()
    return np.concatenate(out)[:n]


def residual_targets(points, fields, zt, tabs, chunk=1 << 20):
    """(M, n_src, 3) BEM minus axial series of each unit field at points with
    y = 0 (so the x component is the radial one): (phi, E_r, E_z) of an
    electrode; (magnetostatic potential of the induced charges, H_r, H_z) of
    a coil, H being the induced charges' field plus the ring's own."""
    torch = B._torch()
    M = len(points)
    out = np.zeros((M, len(fields), 3))
    for s in range(0, M, chunk):
        pts = B.to_dev(points[s:s + chunk], torch.float64)
        for e, (f, c) in enumerate(zip(fields, tabs)):
            if len(f.electrostatic_point_charges):
                pb, fb = B.dev_field_points(pts, f.electrostatic_point_charges.device_sources())
            else:
                pb, fb = B.dev_field_points(pts, f.magnetostatic_point_charges.device_sources())
                fb = fb + B.dev_current_field_points(pts, f.current_point_charges.device_sources())
            pa, fa = B.dev_axial_field_points(pts, zt, c)
            out[s:s + chunk, e, 0] = (pb - pa).cpu().numpy()
            out[s:s + chunk, e, 1] = (fb[:, 0] - fa[:, 0]).cpu().numpy()
            out[s:s + chunk, e, 2] = (fb[:, 2] - fa[:, 2]).cpu().numpy()
    return out


class SurrogateTrainer:
    """Builds the data set of a geometry and trains a SurrogateModel.  Field
    sources: the electrodes `electrodes` (default: every name of geo) and,
    when `coils` is given, its current coils magnetising the `magnetizable`
    electrodes ({name: mu_r})."""

    def __init__(self, geo, r_min=0.1e-3, r_max=0.75e-3, z_lo=-11.5e-3, z_hi=11.5e-3, nz=4601, exclude=50e-6,
                 env_power=8, electrodes=None, magnetizable=None, coils=None):
        self.geo = geo
        self.r_min, self.r_max, self.z_lo, self.z_hi = r_min, r_max, z_lo, z_hi
        self.exclude, self.env_power = exclude, env_power
        self.fields = unit_fields(geo, electrodes)
        self.n_el = len(self.fields)
        if coils is not None:
            self.fields = self.fields + unit_coil_fields(geo, magnetizable or {}, coils)
        self.n_coils = len(self.fields) - self.n_el
        self.z, self.zt, self.tabs = axial_tables(self.fields, z_lo, z_hi, nz)

    def dataset(self, n, seed=0):
        pts = sample_points(n, seed, self.r_min, self.r_max, self.z_lo, self.z_hi, self.geo.segments, self.exclude)
        R = residual_targets(pts, self.fields, self.zt, self.tabs).reshape(len(pts), -1)
        return pts, R

    def train(self, n_samples=1 << 22, steps=80000, batch=8192, lr=2e-3, lr_end=2e-5, seed=0, holdout=0.01,
              log_every=0, weighting='radial', bins=16):
        """Adam on the MSE of the normalised residuals.  weighting 'radial'
        weights every sample by the inverse mean square of the targets in
        its band of rho (`bins` bands), so that the network is fitted to the
        same relative accuracy at every radius instead of being dominated by
        the largest residuals near the electrodes; 'uniform' weights all
        samples alike."""
        torch = B._torch()
        pts, R = self.dataset(n_samples, seed)
        n_el = len(self.fields)  # field sources: electrodes and coils, 3 outputs each
        tmp = SurrogateModel(self.n_el, self.r_max, self.z_lo, self.z_hi, np.ones(OUT), self.env_power, seed=seed,
                             n_coils=self.n_coils)
        env = tmp.envelope(np.hypot(pts[:, 0], pts[:, 1]))
        Y = R / env
        scale = np.ones(OUT, dtype=np.float32)
        scale[:3 * n_el] = np.sqrt(np.mean(Y ** 2, axis=0)) + 1e-300
        T = (Y / scale[:3 * n_el]).astype(np.float32)
        model = SurrogateModel(self.n_el, self.r_max, self.z_lo, self.z_hi, scale, self.env_power, seed=seed,
                               n_coils=self.n_coils)
        n_hold = max(1, int(len(pts) * holdout))
        dev = B.device()
        pts_t = torch.as_tensor(pts, device=dev)
        X = features(pts_t, model.r_max, model.z_c, model.z_half)
        Tt = torch.as_tensor(T, device=dev)
        if weighting == 'radial':
            rho = np.hypot(pts[:, 0], pts[:, 1]) / model.r_max
            band = np.minimum((rho * bins).astype(int), bins - 1)
            ms = np.array([np.mean(T[band == b] ** 2) if np.any(band == b) else 1.0 for b in range(bins)])
            wts = 1.0 / np.maximum(ms[band], 1e-30)
            wts = (wts / wts.mean()).astype(np.float32)
        elif weighting == 'uniform':
            wts = None
        else:
            raise ValueError(f'unknown weighting {weighting!r}')
        Wt = None if wts is None else torch.as_tensor(wts, device=dev)
        Xtr, Ttr = X[n_hold:], Tt[n_hold:]
        Wtr = None if Wt is None else Wt[n_hold:]
        Xho, Tho = X[:n_hold], Tt[:n_hold]
        ntr = Xtr.shape[0]
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        hist = []
        for step in range(steps):
            idx = torch.randint(0, ntr, (batch,), device=dev, generator=gen)
            loss = model.mlp.loss_and_grad(Xtr[idx].contiguous(), Ttr[idx].contiguous(), 3 * n_el,
                                           None if Wtr is None else Wtr[idx].contiguous())
            frac = step / max(1, steps - 1)
            cur = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * frac))
            model.mlp.adam(cur)
            if log_every and step % log_every == 0:
                hist.append((step, float(loss)))
        out = model.mlp.forward(Xho)[:, :3 * n_el]
        ho = float(((out - Tho) ** 2).mean())
        self.holdout_points = pts[:n_hold]
        self.holdout_residual = R[:n_hold]
        return model, {'holdout_mse': ho, 'history': hist, 'scale': scale[:3 * n_el].tolist()}


class FieldSurrogate:
    """A traceable surrogate field for given source strengths: the axial
    series of sum_s V_s (unit table s) plus the network's correction, with the
    exact BEM field of the same charges as fallback.  `strengths` lists the
    electrode voltages, then (for a model with coils) the coil currents in
    A-turns; the magnetic part is the axial series of sum_c I_c (coil table c)
    plus the coils' corrections, its fallback the induced magnetostatic
    charges and the current rings."""

    ENGINES = {'tc': 0, 'warp': 1}

    def __init__(self, model, fields, z, tabs, strengths, segments, fallback_dist=50e-6, engine='tc'):
        """engine: 'tc' evaluates the network with tcgen05 MMAs (groups of 128
        particles, accumulators in tensor memory); 'warp' with warp-level
        mma.sync (32 particles per warp)."""
        torch = B._torch()
        if engine not in self.ENGINES:
            raise ValueError(f'unknown engine {engine!r}; expected one of {sorted(self.ENGINES)}')
        self.engine = engine
        self.model = model
        self.strengths = np.asarray(strengths, dtype=np.float64)
        assert len(self.strengths) == model.n_src == len(fields) == len(tabs)
        ne = model.n_el
        self.volts, self.currents = self.strengths[:ne], self.strengths[ne:]
        self.z = z
        self.zt = B.to_dev(z, torch.float64)
        self.table = sum(float(v) * t for v, t in zip(self.volts, tabs[:ne])).contiguous()
        self.mag_table = sum(float(c) * t for c, t in zip(self.currents, tabs[ne:])).contiguous() \
            if model.n_coils else None
        bem = fields[0] * float(self.strengths[0])
        for f, v in zip(fields[1:], self.strengths[1:]):
            bem = bem + f * float(v)
        self.bem = bem
        self.sources = bem.electrostatic_point_charges.device_sources()
        self.mag_sources = bem.magnetostatic_point_charges.device_sources() if model.n_coils else None
        self.cur_sources = bem.current_point_charges.device_sources() if model.n_coils else None
        self.segments = B.to_dev(np.asarray(segments, dtype=np.float64).reshape(-1, 4), torch.float64)
        self.fallback_dist = float(fallback_dist)
        self.field_bounds = None

    def _tb_field(self):
        def src(t):
            return (t.data_ptr() if t is not None and t.numel() else None), (t.shape[1] if t is not None else 0)
        e, ne = src(self.sources)
        m, nm = src(self.mag_sources)
        c, nc = src(self.cur_sources)
        return B.TbField(e, ne, m, nm, c, nc, None, self.zt.data_ptr(), self.table.data_ptr(),
                         B._ptr(self.mag_table), len(self.z))

    def _descriptor(self):
        m = self.model
        s = TbSurrogate()
        s.weights_bf16 = m.mlp.pb.data_ptr()
        s.params_f32 = m.mlp.p.data_ptr()
        s.r_max, s.z_c, s.z_half, s.z_lo, s.z_hi = m.r_max, m.z_c, m.z_half, m.z_lo, m.z_hi
        s.n_electrodes = m.n_el
        s.n_coils = m.n_coils
        for i, v in enumerate(self.strengths):
            s.strengths[i] = float(v)
        for i, v in enumerate(m.scale):
            s.scale[i] = float(v)
        s.env_power = m.env_power
        s.segments = self.segments.data_ptr()
        s.n_segments = self.segments.shape[0]
        s.fallback_dist = self.fallback_dist
        s.engine = self.ENGINES[self.engine]
        return self._tb_field(), s

    def trace_device(self, start, qm, bounds, atol, plane_z=None, max_attempts=100_000, stream=None):
        torch = B._torch()
        n = start.shape[0]
        dev = start.device
        f, s = self._descriptor()
        o = B.TbTraceOpts()
        for i, v in enumerate(np.asarray(bounds, dtype=np.float64).reshape(-1)):
            o.bounds[i] = float(v)
        o.atol = float(atol)
        o.plane_z = 0.0 if plane_z is None else float(plane_z)
        o.record_plane = 0 if plane_z is None else 1
        o.max_attempts = int(max_attempts)
        o.max_rows = 0
        o.team_warps = 0
        status = torch.empty(n, dtype=torch.int32, device=dev)
        final = torch.empty((n, 7), dtype=torch.float64, device=dev)
        plane = torch.empty((n, 7), dtype=torch.float64, device=dev) if plane_z is not None else None
        counters = torch.empty((n, 3), dtype=torch.int64, device=dev)
        work = torch.empty(1, dtype=torch.int32, device=dev)
        r = _lib.tb_trace_surrogate(start.data_ptr(), None, qm.data_ptr(), n, C.byref(f), C.byref(s), C.byref(o),
                                    status.data_ptr(), final.data_ptr(), B._ptr(plane), counters.data_ptr(),
                                    work.data_ptr(), B._stream() if stream is None else stream)
        if r != B.TB_OK:
            raise B.BackendError(f'tb_trace_surrogate failed with status {r}')
        from .tracing import TraceResult
        res = TraceResult(status, final, plane, counters)
        res._keep = (start, qm, work, self)
        return res

    def trace_axial_device(self, start, qm, bounds, atol, plane_z=None, max_attempts=100_000, stream=None):
        """The same particles through the axial series of this field's
        coefficient tables alone (FieldRadialAxial's field, radial.c:347-384;
        the tracer's k_trace_axial), without the network and without the BEM
        fallback: the method the learned correction improves on.  Returns a
        TraceResult of device tensors (counters (n, 2))."""
        from .tracing import TraceResult
        torch = B._torch()
        n = start.shape[0]
        dev = start.device
        f = B.TbField(None, 0, None, 0, None, 0, None, self.zt.data_ptr(), self.table.data_ptr(),
                      B._ptr(self.mag_table), len(self.z))
        o = B.TbTraceOpts()
        for i, v in enumerate(np.asarray(bounds, dtype=np.float64).reshape(-1)):
            o.bounds[i] = float(v)
        o.atol = float(atol)
        o.plane_z = 0.0 if plane_z is None else float(plane_z)
        o.record_plane = 0 if plane_z is None else 1
        o.max_attempts = int(max_attempts)
        o.max_rows = 0
        o.team_warps = 0
        status = torch.empty(n, dtype=torch.int32, device=dev)
        final = torch.empty((n, 7), dtype=torch.float64, device=dev)
        plane = torch.empty((n, 7), dtype=torch.float64, device=dev) if plane_z is not None else None
        counters = torch.empty((n, 2), dtype=torch.int64, device=dev)
        work = torch.empty(1, dtype=torch.int32, device=dev)
        B._call('tb_trace_rk45', start.data_ptr(), None, qm.data_ptr(), n, C.byref(f), C.byref(o), None, None,
                status.data_ptr(), final.data_ptr(), B._ptr(plane), counters.data_ptr(), work.data_ptr(),
                B._stream() if stream is None else stream)
        res = TraceResult(status, final, plane, counters)
        res._keep = (start, qm, work, self)
        return res

    def trace_endpoints(self, position, velocity, bounds, plane_z, mass=None, charge=None, atol=1e-8,
                        max_attempts=100_000):
        """Batched endpoint tracing with host arrays in and out (the public
        form of trace_device): returns (plane (n,7), final (n,7), status (n,),
        counters (n,3))."""
        from scipy.constants import e as qe, m_e
        torch = B._torch()
        mass = m_e if mass is None else mass
        charge = -qe if charge is None else charge
        pos = np.atleast_2d(np.asarray(position, dtype=np.float64))
        vel = np.atleast_2d(np.asarray(velocity, dtype=np.float64))
        n = len(pos)
        start = B.to_dev(np.concatenate([pos, vel], 1), torch.float64)
        qm = B.to_dev(np.broadcast_to(np.asarray(charge, dtype=np.float64) / mass, (n,)).copy(), torch.float64)
        res = self.trace_device(start, qm, bounds, atol, plane_z=plane_z, max_attempts=max_attempts)
        return (res.plane.cpu().numpy(), res.final.cpu().numpy(), res.status.cpu().numpy(),
                res.counters.cpu().numpy())

    def trace_session(self, n, bounds, plane_z, mass=None, charge=None, atol=1e-8, max_attempts=100_000):
        """A TraceSession for repeated batches of n particles (see there)."""
        return TraceSession(self, n, bounds, plane_z, mass, charge, atol, max_attempts)

    def kernel_field_at_points(self, points, magnetic=False):
        """Surrogate E at points (M, 3) as the tracer's kernel evaluates it
        (electrode fallback included); returns (E, used_bem), or with
        magnetic=True (E, H, used_bem)."""
        torch = B._torch()
        pts = B.to_dev(np.asarray(points, dtype=np.float64).reshape(-1, 3), torch.float64)
        M = pts.shape[0]
        out = torch.empty((M, 3), dtype=torch.float64, device=pts.device)
        out_h = torch.empty((M, 3), dtype=torch.float64, device=pts.device) if magnetic else None
        ub = torch.empty(M, dtype=torch.int32, device=pts.device)
        f, s = self._descriptor()
        r = _lib.tb_surrogate_field_points(pts.data_ptr(), M, C.byref(f), C.byref(s), out.data_ptr(),
                                           B._ptr(out_h), ub.data_ptr(), B._stream())
        if r != B.TB_OK:
            raise B.BackendError(f'tb_surrogate_field_points failed with status {r}')
        if magnetic:
            return out.cpu().numpy(), out_h.cpu().numpy(), ub.cpu().numpy()
        return out.cpu().numpy(), ub.cpu().numpy()

    def field_at_points(self, points):
        """Surrogate E at points (M, 3) (without the electrode fallback)."""
        torch = B._torch()
        pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
        _, fa = B.dev_axial_field_points(B.to_dev(pts, torch.float64), self.zt, self.table)
        E = fa.cpu().numpy()
        corr = self.model.predict_residual(pts)[:, :self.model.n_el]  # (M, n_el, 3): the electrodes
        r = np.hypot(pts[:, 0], pts[:, 1])
        er = np.einsum('e,me->m', self.volts, corr[:, :, 1])
        ez = np.einsum('e,me->m', self.volts, corr[:, :, 2])
        with np.errstate(invalid='ignore', divide='ignore'):
            cx = np.where(r > 0, pts[:, 0] / r, 0.0)
            cy = np.where(r > 0, pts[:, 1] / r, 0.0)
        E[:, 0] += er * cx
        E[:, 1] += er * cy
        E[:, 2] += ez
        return E


_tb_trace_surrogate_args = [_vp, _vp, _vp, _i64, C.POINTER(B.TbField), C.POINTER(TbSurrogate),
                            C.POINTER(B.TbTraceOpts), _vp, _vp, _vp, _vp, _vp, _vp]
_lib.tb_trace_surrogate.argtypes = _tb_trace_surrogate_args
_lib.tb_surrogate_field_points.argtypes = [_vp, _i64, C.POINTER(B.TbField), C.POINTER(TbSurrogate), _vp, _vp, _vp,
                                           _vp]
_lib.tb_surrogate_field_points.restype = C.c_int
_lib.tb_trace_surrogate.restype = C.c_int


class TraceSession:
    """Repeated endpoint tracing of batches of n particles through one
    surrogate field, for callers that trace many batches: pinned host staging
    buffers, static device buffers, and the whole step -- host-to-device copy
    of the start states, the tracer launch (work-queue reset + kernel),
    device-to-host copies of the endpoints -- captured once in a CUDA graph.
    Each run() is one graph replay and one stream synchronisation.

    run(position, velocity) returns views of the pinned output buffers
    (plane (n,7), final (n,7), status (n,), counters (n,3)), valid until the
    next run(); copy them to keep them.  run_many(batches) traces a sequence
    of batches with two buffer sets in flight, so that one batch's copies and
    host staging overlap the next batch's trace.  replay_device() replays
    only the device part (start states already in `start`), for timing.
    A session's buffers are shared by its calls: use it from one host thread
    at a time."""

    def __init__(self, field, n, bounds, plane_z, mass=None, charge=None, atol=1e-8, max_attempts=100_000):
        from scipy.constants import e as qe, m_e
        torch = B._torch()
        dev = B.device()
        self._args = (bounds, plane_z, mass, charge, atol, max_attempts)
        self._peer = None  # the second buffer set of run_many, made on first use
        self._streams = None
        mass = m_e if mass is None else mass
        charge = -qe if charge is None else charge
        self.n = int(n)
        self.field = field
        self.start_h = torch.empty((n, 6), dtype=torch.float64).pin_memory()
        self.plane_h = torch.empty((n, 7), dtype=torch.float64).pin_memory()
        self.final_h = torch.empty((n, 7), dtype=torch.float64).pin_memory()
        self.status_h = torch.empty(n, dtype=torch.int32).pin_memory()
        self.counters_h = torch.empty((n, 3), dtype=torch.int64).pin_memory()
        self.start = torch.zeros((n, 6), dtype=torch.float64, device=dev)
        self.qm = torch.full((n,), float(charge) / float(mass), dtype=torch.float64, device=dev)
        self.status = torch.empty(n, dtype=torch.int32, device=dev)
        self.final = torch.empty((n, 7), dtype=torch.float64, device=dev)
        self.plane = torch.empty((n, 7), dtype=torch.float64, device=dev)
        self.counters = torch.empty((n, 3), dtype=torch.int64, device=dev)
        self.work = torch.empty(1, dtype=torch.int32, device=dev)
        self.f, self.s = field._descriptor()
        o = B.TbTraceOpts()
        for i, v in enumerate(np.asarray(bounds, dtype=np.float64).reshape(-1)):
            o.bounds[i] = float(v)
        o.atol = float(atol)
        o.plane_z = float(plane_z)
        o.record_plane = 1
        o.max_attempts = int(max_attempts)
        o.max_rows = 0
        o.team_warps = 0
        self.o = o
        # one eager single-particle launch first, so that the kernel
        # attributes and the library's lazy set-up happen outside the capture
        self.start[0, 5] = 1.0
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._launch(side.cuda_stream, n=1)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph_device = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph_device):
            self._launch(torch.cuda.current_stream().cuda_stream)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.start.copy_(self.start_h, non_blocking=True)
            self._launch(torch.cuda.current_stream().cuda_stream)
            self.plane_h.copy_(self.plane, non_blocking=True)
            self.final_h.copy_(self.final, non_blocking=True)
            self.status_h.copy_(self.status, non_blocking=True)
            self.counters_h.copy_(self.counters, non_blocking=True)

    def _launch(self, stream, n=None):
        n = self.n if n is None else n
        r = _lib.tb_trace_surrogate(self.start.data_ptr(), None, self.qm.data_ptr(), n, C.byref(self.f),
                                    C.byref(self.s), C.byref(self.o), self.status.data_ptr(), self.final.data_ptr(),
                                    self.plane.data_ptr(), self.counters.data_ptr(), self.work.data_ptr(), stream)
        if r != B.TB_OK:
            raise B.BackendError(f'tb_trace_surrogate failed with status {r}')

    @property
    def h2d_bytes(self):
        return self.n * 6 * 8

    @property
    def d2h_bytes(self):
        return self.n * (7 + 7) * 8 + self.n * 4 + self.n * 3 * 8

    def run(self, position, velocity):
        torch = B._torch()
        sh = self.start_h.numpy()
        sh[:, :3] = position
        sh[:, 3:] = velocity
        self.graph.replay()
        torch.cuda.current_stream().synchronize()
        return self.plane_h.numpy(), self.final_h.numpy(), self.status_h.numpy(), self.counters_h.numpy()

    def run_many(self, batches, before=None):
        """Traces batches [(position (n,3), velocity (n,3)), ...] with two
        buffer sets (this session's and a second one, made on the first call)
        replayed alternately on two streams: while batch i traces, batch i - 1's
        endpoints come back and batch i + 1's start states are staged in pinned
        memory.  Returns one (plane, final, status, counters) tuple of host
        copies per batch, in order.  before: optional callable run on a
        batch's stream just before its replay (cache control in measurements).
        Work already queued on the current stream completes first; the current
        stream waits for all batches on return."""
        torch = B._torch()
        if self._peer is None:
            self._peer = TraceSession(self.field, self.n, *self._args)
            self._streams = (torch.cuda.Stream(device=self.start.device), torch.cuda.Stream(device=self.start.device))
        sets = (self, self._peer)
        cur = torch.cuda.current_stream()
        for st in self._streams:
            st.wait_stream(cur)
        events = [None, None]
        out = [None] * len(batches)

        def collect(i):
            k = i % 2
            events[k].synchronize()
            t = sets[k]
            out[i] = (t.plane_h.numpy().copy(), t.final_h.numpy().copy(), t.status_h.numpy().copy(),
                      t.counters_h.numpy().copy())

        for i, (position, velocity) in enumerate(batches):
            k = i % 2
            if i >= 2:
                collect(i - 2)  # frees set k: its outputs are read and its staging is no longer in use
            t = sets[k]
            sh = t.start_h.numpy()
            sh[:, :3] = position
            sh[:, 3:] = velocity
            with torch.cuda.stream(self._streams[k]):
                if before is not None:
                    before()
                t.graph.replay()
                ev = torch.cuda.Event()
                ev.record()
            events[k] = ev
        for i in range(max(0, len(batches) - 2), len(batches)):
            collect(i)
        for st in self._streams:
            cur.wait_stream(st)
        return out

    def replay_device(self):
        self.graph_device.replay()
