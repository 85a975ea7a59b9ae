"""Benchmark: traced electrons per second at <= 1 nm endpoint error through
the einzel-lens workload, learned surrogate vs plain BEM field.

Workload: the three-tube einzel lens of 1,000 cubic line elements graded
toward the tube edges (0 V / V_mid / 0 V, V_mid from the seed), solved once on
the GPU.  A step traces a batch of electrons (default 262,144) at 1 keV +-5 %,
angles +-20 mrad, start radius up to the beam's r_max at z = -9.5 mm, with
adaptive RKF45 at atol = 1e-10 m until they leave the bounds (|x|,|y| <= 2 mm,
|z| <= 10 mm), recording each electron's crossing of the exit plane
z = +9.5 mm.  Two beams: `wide` (r0 <= 0.35 mm, the headline: the axial
series alone misses 1 nm there, the learned correction holds it) and `narrow`
(r0 <= 0.2 mm, the plain-method workload's beam).  Synthetic inputs; no
dataset.

On each beam three arms: the surrogate (axial series + BF16 MLP correction
trained on the GPU from BEM samples in the setup phase, BEM fallback near
electrodes), the axial series alone (the same table, no network), and the
plain FP64 BEM tracer on a 16,384-electron slice.  Endpoint errors of the
surrogate and of the axial series against the CPU oracle on a held-out
sample of each beam (1 % of the headline beam), traced in spawned processes
while the GPU works; CPU baselines: the reference C backend's plain-BEM
tracer and its axial-series tracer on all host threads.

  --field bem: the plain FP64 BEM field only.
  --impl reference: the reference C backend's plain BEM tracer on host cores.
  --workload solve: only the precision workload's solve (the lens at
      --precision-n elements, 8 right-hand sides): GPU FP64 fill, FP64
      pivoted LU and the mixed tensor-core solve (also reported, as
      `precision_solve`, beside the tracer in the default run).
  --workload combined: the combined electro-magnetostatic workload.
  --workload batch: the batching workload (64 mirror lenses filled, solved
      and traced with the direct BEM field, one CUDA graph per step).

`value` is whole-job electrons/s with the start states resident in HBM;
`e2e` is the same through the public API with host arrays over a stream of
batches (two in flight), host<->device copies inside the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_ELEMENTS = 1000
SEED = 1
ATOL = 1e-10
METRIC = 'traced electrons/s at <=1 nm endpoint error, surrogate vs plain BEM field'

# Start-radius range of the two beams (1 keV +-5 %, +-20 mrad, z0 = -9.5 mm).
# narrow: the plain-method workload's r0 <= 0.2 mm, where the axial series
# alone already traces within 1 nm.  wide: start radii out to where the axial
# series alone misses 1 nm and the learned correction is what holds it.
BEAMS = {'narrow': {'r_max': 0.2e-3}, 'wide': {'r_max': 0.35e-3}}


def workload_config(electrons, field, beam):
    desc = {'surrogate': 'learned surrogate field (axial series + BF16 MLP correction, BEM fallback)',
            'bem': 'plain BEM field (FP64)'}[field]
    r_mm = BEAMS[beam]['r_max'] * 1e3
    return {'workload': f'einzel lens, {N_ELEMENTS} cubic elements, {desc}, {electrons} electrons/step at '
                        f'1 keV +-5%, +-20 mrad, r0<={r_mm:g} mm ({beam} beam), RKF45 atol=1e-10 m, '
                        f'exit plane z=+9.5 mm',
            'elements': N_ELEMENTS, 'electrons_per_step': electrons, 'atol_m': ATOL, 'seed': SEED,
            'field': field, 'beam': beam, 'beam_r0_max_m': BEAMS[beam]['r_max'],
            'l2': 'L2 flushed (256 MiB write, inside the step time) before every timed step'}


def dist_info():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f'traceon_b200_clocks_gpu{index}_', suffix='.csv')
        os.close(fd)

    def __enter__(self):
        q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(',') for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace('.', '').isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace('.', '').isdigit()]
        reasons = set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip() == 'Active':
                    reasons.add(n)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': sorted(reasons), 'samples': len(rows)}


# ---------------------------------------------------------------- workload
def lens_inputs(electrons, beam='wide', seed=SEED):
    """The lens (1,000 elements), its voltages and `electrons` start states
    of the named beam."""
    from traceon_b200 import geometry as G
    geo = G.einzel_lens(N_ELEMENTS)
    volts = G.einzel_lens_voltages(SEED)
    p0, v0 = G.surrogate_beam(electrons, seed + 100, r_max=BEAMS[beam]['r_max'])
    return geo, volts, p0, v0


def oracle_charges(geo, volts, threads):
    """FP64 oracle: CPU fill, converged QUADPACK self terms, LAPACK solve."""
    from oracle.oracle import Oracle, solve
    port = Oracle('port')
    values = geo.voltages_to_values(volts)
    A = port.matrix(geo.vertices, np.ones(len(geo), np.uint8), values, threads=threads)
    q = solve(A, values)[0]
    jac, pos = port.fill_jacobian_buffer_radial(geo.vertices)
    return q, jac, pos


# Endpoints traced by the CPU oracle: its FP64 BEM trace of each checked
# electron and its cubic-Hermite crossing of the exit plane, in a pool of
# spawned processes (no CUDA in them) that runs while the GPU work proceeds.
_ORACLE = {}


def _oracle_init(q, jac, pos):
    try:
        os.nice(10)  # below the bench's own host thread
    except OSError:
        pass
    from oracle.oracle import Oracle
    _ORACLE.update(oracle=Oracle('port'), q=q, jac=jac, pos=pos)


def _oracle_trace_one(state):
    from oracle.oracle import EM, hermite_plane_crossing
    from traceon_b200 import geometry as G
    t, s = _ORACLE['oracle'].trace_bem(state[:3], state[3:], EM, _ORACLE['q'], _ORACLE['jac'], _ORACLE['pos'],
                                      G.LENS_BOUNDS, ATOL)
    h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
    return (np.nan, np.nan) if h is None else (float(h[0]), float(h[1]))


class OracleTraces:
    """Exit-plane crossings of electrons traced by the CPU oracle, computed
    asynchronously in `workers` spawned processes."""

    def __init__(self, q, jac, pos, workers):
        import multiprocessing as mp
        self.workers = workers
        self.pool = mp.get_context('spawn').Pool(workers, _oracle_init, (q, jac, pos))
        self.jobs = {}
        self.t0 = time.perf_counter()

    def submit(self, name, p0, v0):
        states = [np.concatenate([a, b]) for a, b in zip(p0, v0)]
        self.jobs[name] = self.pool.map_async(_oracle_trace_one, states, chunksize=4)

    def result(self, name):
        return np.array(self.jobs[name].get(), dtype=np.float64).reshape(-1, 2)

    def close(self):
        self.pool.close()
        self.pool.join()
        return time.perf_counter() - self.t0


def endpoint_errors_nm(plane, ref_xy):
    """Max and p99 over electrons of max(|dx|, |dy|) at the exit plane, nm;
    electrons without a crossing on either side count as infinite."""
    d = np.max(np.abs(plane[:, 1:3] - ref_xy), axis=1) * 1e9
    finite = np.isfinite(d)
    d = np.where(finite, d, np.inf)
    # with missing crossings, the nearest-rank percentile (interpolating
    # between infinities would give NaN)
    p99 = np.percentile(d, 99) if finite.all() else np.percentile(d, 99, method='higher')
    return {'max_nm': float(np.max(d)), 'p99_nm': float(p99), 'n': int(len(d)),
            'within_1nm': int(np.sum(d <= 1.0))}


def cpu_reference_rate(q, jac, pos, p0, v0, threads, seconds, kind='ref', axial=None):
    """The reference's own CPU tracer (oracle/_ref: trace_particle with its
    field_radial_traceable callback, or with field_radial_derivs_traceable
    when `axial` = (z, coefficients) is given) on `threads` host threads for
    about `seconds`; returns (electrons/s, electrons traced, kind)."""
    from oracle.oracle import Oracle, EM, available
    from traceon_b200 import geometry as G
    if kind == 'ref' and not available('ref'):
        kind = 'port'
    o = Oracle(kind)
    done = []
    lock = threading.Lock()
    stop = time.perf_counter() + seconds
    counter = iter(range(len(p0)))
    zero_mag = None if axial is None else np.zeros_like(axial[1])

    def worker():
        while time.perf_counter() < stop:
            with lock:
                i = next(counter, None)
            if i is None:
                return
            if axial is None:
                o.trace_bem(p0[i], v0[i], EM, q, jac, pos, G.LENS_BOUNDS, ATOL)
            else:
                o.trace_axial(p0[i], v0[i], EM, axial[0], axial[1], zero_mag, G.LENS_BOUNDS, ATOL)
            with lock:
                done.append(i)

    t0 = time.perf_counter()
    ts = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    el = time.perf_counter() - t0
    return len(done) / el, len(done), kind


def reference_axial_table(q, jac, pos, z):
    """The reference's FieldRadialAxial table of the oracle charges on the
    grid z: its C axial-derivative sums (oracle/_ref) and its SciPy spline
    coefficients (traceon/field.py:971-991)."""
    from oracle.oracle import Oracle, available, axial_coefficients
    o = Oracle('ref' if available('ref') else 'port')
    return axial_coefficients(z, o.axial_derivatives_radial(z, q, jac, pos))


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return
    cores = host_cores()
    geo, volts, p0, v0 = lens_inputs(4096, args.beam)
    q, jac, pos = oracle_charges(geo, volts, cores)
    for _ in range(args.warmup):
        cpu_reference_rate(q, jac, pos, p0, v0, cores, 2.0)
    rates, n_total, t_total = [], 0, 0.0
    # each step a bounded sample: about two minutes of CPU work in total
    step_s = min(args.ref_seconds, max(2.0, 120.0 / max(args.steps, 1)))
    for s in range(args.steps):
        sl = slice((s * cores * 4) % len(p0), None)
        r, n, kind = cpu_reference_rate(q, jac, pos, p0[sl], v0[sl], cores, step_s)
        rates.append(r)
        n_total += n
        t_total += n / r if r else 0
    value = n_total / t_total if t_total else 0.0
    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t_total / max(args.steps, 1), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': workload_config(args.electrons, args.field, args.beam),
            'reference_field': 'plain BEM (the reference has no learned surrogate)',
            'cpu_baseline': {'value': value, 'unit': 'electrons/s', 'cores': cores,
                             'kind': 'reference' if kind == 'ref' else 'port',
                             'sample': f'{n_total} electrons of this beam over {args.steps} steps of ~{step_s:.0f} s '
                                       f'(reference C backend trace_particle + field_radial_traceable, '
                                       f'{cores} threads)'},
            'e2e': {'value': value, 'unit': 'electrons/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- precision solve
def precision_solve(n, nrhs=8, seed=2, field_points=1 << 20, fp64_lu=True, fp64_peak=None, check=4096,
                    keep_state=False):
    """The precision workload's charge solve: the three-electrode lens meshed
    to n cubic elements, nrhs right-hand sides with every electrode voltage
    ~U[-3, 3] kV.  GPU FP64 fill (+ singular self terms), then (a) the FP64
    LU with partial pivoting (numpy.linalg.solve's factorisation) and (b) the
    mixed solve (FP32 tensor-core LU of the equilibrated matrix, FP64
    iterative refinement; its lookahead width tuned first by
    autotune.tune_solve_lookahead, then the median of three solves).
    CUDA-event times; charges of (b) against (a).
    Then potential and field of the first right-hand side's charges at
    `field_points` points, and the axial derivatives of the same charges on
    2,000 z-points; FP64 rooflines of the fill, field and axial kernels
    against `fp64_peak` (TFLOP/s) with the algorithmic flop counts of their
    formulas.  `check` points of the field are re-evaluated by the CPU oracle
    here; with keep_state the inputs and outputs stay in out['_field_state']
    for the caller's own precision_field_check instead."""
    import torch
    from traceon_b200 import backend as B
    from traceon_b200.geometry import einzel_lens

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    geo = einzel_lens(n)
    v = B.to_dev(geo.vertices, torch.float64)
    t = B.to_dev(np.ones(n, np.uint8), torch.uint8)
    val = B.to_dev(np.zeros(n), torch.float64)
    A = torch.empty((n, n), dtype=torch.float64, device='cuda')
    jac, pos = B.dev_jacobian_buffer(v)

    def fill_offdiag():
        B.dev_fill_matrix(A, v, t, val, jac, pos)

    def self_terms():
        B.dev_self_integrals(v, t, val, A)

    fill_offdiag()
    self_terms()  # warm-up
    fill_ms, _ = timed(fill_offdiag)
    self_ms, _ = timed(self_terms)
    rng = np.random.default_rng(seed)
    F = torch.as_tensor(geo.voltages_to_values(rng.uniform(-3000, 3000, (nrhs, 3)).T).T.copy(), device='cuda')

    def lu64():
        LU = A.clone()
        _, perm = B.dev_lu_factor(LU)
        return B.dev_lu_solve(LU, perm, F)

    from traceon_b200 import autotune
    lookahead = autotune.tune_solve_lookahead(A, F)  # warms the solve up too
    runs = [timed(lambda: B.dev_solve_mixed(A, F)) for _ in range(3)]
    mixed_ms = float(np.median([r[0] for r in runs]))
    Xm, iters, rel = runs[-1][1]
    lib_ms = None
    if fp64_lu:
        lu64()
        lu_ms, X64 = timed(lu64)
        err = float(((Xm - X64).abs().amax(1) / X64.abs().amax(1)).max())
        # context only: the vendor library's FP64 LU (getrf + getrs through
        # torch.linalg.solve), not a path of this library
        torch.linalg.solve(A, F.T)
        lib_ms, _ = timed(lambda: torch.linalg.solve(A, F.T))
    else:  # profiling the mixed solve alone
        lu_ms, err = None, None
    fill_ms_total = fill_ms + self_ms
    out = {'workload': f'einzel lens, {n} cubic elements, {nrhs} right-hand sides (electrode voltages U[-3,3] kV)',
           'fill_fp64_ms': fill_ms_total, 'fill_offdiagonal_ms': fill_ms, 'self_integrals_ms': self_ms,
           'solve_fp64_lu_ms': lu_ms, 'solve_mixed_ms': mixed_ms,
           'solve_mixed_ms_runs': [r[0] for r in runs],
           'lookahead_reserve_sms': lookahead['reserve_sms'],
           'lookahead_tuning_ms': {str(k): v for k, v in lookahead['times_ms'].items()},
           'mixed_iterations': iters, 'mixed_last_correction': rel, 'charges_rel_err_vs_fp64': err,
           'solve_fp64_vendor_lu_ms': lib_ms,
           'speedup_vs_vendor_fp64_lu': lib_ms / mixed_ms if lib_ms else None,
           'speedup_solve': lu_ms / mixed_ms if lu_ms else None,
           'speedup_fill_plus_solve': (fill_ms_total + lu_ms) / (fill_ms_total + mixed_ms) if lu_ms else None,
           'fill_plus_mixed_solve_ms': fill_ms_total + mixed_ms,
           'speedup_fill_plus_solve_vs_vendor': (fill_ms_total + lib_ms) / (fill_ms_total + mixed_ms)
           if lib_ms else None,
           'lu_flop': 2.0 / 3.0 * n ** 3}
    # fill roofline: N^2 entries x 16 ring potentials (the diagonal's Gauss
    # terms are computed and overwritten, as in the reference)
    pots = float(n) * n * 16
    out['fill_roofline'] = fp64_roofline(pots, FLOP_RING_POT, fill_ms, fp64_peak, 'k_fill_matrix',
                                         'ring-potential evaluations (+ 1 log, 1 rsqrt each)')
    del A
    torch.cuda.empty_cache()
    if field_points:
        out.update(precision_fields(geo, Xm[0], field_points, seed, fp64_peak))
        if not keep_state:
            state = out.pop('_field_state')
            if check:
                out.update(precision_field_check(state, check, host_cores()))
    out.update(axial_roofline(geo, Xm[0], fp64_peak))
    return out


def fp64_roofline(units, flop_per_unit, ms, peak, kernel, unit_desc):
    achieved = units * flop_per_unit / (ms * 1e-3) / 1e12
    return {'bound': 'fp64', 'kernel': kernel, 'units': units, 'flop_per_unit': flop_per_unit,
            'unit_desc': unit_desc, 'achieved': achieved, 'unit': 'TFLOP/s', 'peak': peak,
            'frac': achieved / peak if peak else None,
            'peak_source': 'FP64 FMA throughput measured in this run (tests/probe tb_probe_fp64_fma)'}


def precision_fields(geo, charges_t, m, seed, fp64_peak=None):
    """Potential and field of the charges at m points (x = r ~ U[0, 0.9] mm,
    y = 0, z ~ U[-8, 8] mm), FP64 ring sums on the GPU; the inputs and
    outputs are kept in '_field_state' for precision_field_check."""
    import torch
    from traceon_b200 import backend as B
    rng = np.random.default_rng(seed + 1)
    pts = np.zeros((m, 3))
    pts[:, 0] = rng.uniform(0.0, 0.9e-3, m)
    pts[:, 2] = rng.uniform(-8e-3, 8e-3, m)
    pts_t = B.to_dev(pts, torch.float64)
    v = B.to_dev(geo.vertices, torch.float64)
    jac, pos = B.dev_jacobian_buffer(v)
    src = B.dev_pack_sources(charges_t.contiguous(), jac, pos)
    B.dev_field_points(pts_t[:1024], src)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    pot, fld = B.dev_field_points(pts_t, src)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    pairs = float(m) * src.shape[1]
    return {'field_points': m, 'field_ms': ms, 'field_ring_pairs_per_s': pairs / (ms * 1e-3),
            'field_roofline': fp64_roofline(pairs, FLOP_FIELD_PAIR_POT, ms, fp64_peak, 'k_field_points',
                                            'ring-pair potential + field evaluations (+ 1 log, 1 rsqrt, '
                                            '1 reciprocal each)'),
            '_field_state': (geo.vertices, charges_t.cpu().numpy(), pts, pot.cpu().numpy(), fld.cpu().numpy(), seed)}


def precision_field_check(state, check, threads):
    """`check` of the field points re-evaluated by the CPU oracle (its own
    element quadrature and the same charges) on `threads` host threads."""
    from oracle.oracle import Oracle
    vertices, q, pts, pot, fld, seed = state
    rng = np.random.default_rng(seed + 2)
    sample = rng.choice(len(pts), min(check, len(pts)), replace=False)
    port = Oracle('port')
    jac_o, pos_o = port.fill_jacobian_buffer_radial(vertices)
    t0 = time.perf_counter()
    f_or = port.field_radial_many(pts[sample], q, jac_o, pos_o, threads=threads)
    p_or = port.potential_radial_many(pts[sample], q, jac_o, pos_o, threads=threads)
    f_gpu, p_gpu = fld[sample], pot[sample]
    # relative to the largest value of the sample (E_r vanishes on the axis)
    ferr = float(np.max(np.abs(f_gpu - f_or)) / np.max(np.abs(f_or)))
    perr = float(np.max(np.abs(p_gpu - p_or)) / np.max(np.abs(p_or)))
    return {'field_rel_err_vs_oracle': ferr, 'potential_rel_err_vs_oracle': perr, 'field_checked_points': len(sample),
            'field_check_s': time.perf_counter() - t0}


def axial_roofline(geo, charges_t, fp64_peak, nz=2000):
    """Axial derivatives (9 per z) of the charges on nz z-points over the
    lens: nz x 16 N ring recurrences."""
    import torch
    from traceon_b200 import backend as B
    v = B.to_dev(geo.vertices, torch.float64)
    jac, pos = B.dev_jacobian_buffer(v)
    src = B.dev_pack_sources(charges_t.contiguous(), jac, pos)
    z = B.to_dev(np.linspace(-9.95e-3, 9.95e-3, nz), torch.float64)
    B.dev_axial_derivatives(z, src)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    B.dev_axial_derivatives(z, src)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    units = float(nz) * src.shape[1]
    return {'axial_ms': ms, 'axial_z_points': nz,
            'axial_roofline': fp64_roofline(units, FLOP_AXIAL_RING, ms, fp64_peak, 'k_axial_derivs',
                                            'ring recurrences of 9 axial derivatives (+ 1 sqrt, 2 divisions each)')}


# ---------------------------------------------------------------- GPU arm
def load_probe():
    """libtb_probe.so (tests/probe): the FP64 FMA throughput probe, a
    measurement helper kept out of the product library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location('tb_probe_loader', os.path.join(HERE, 'tests', 'probe', 'loader.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load()


def measure_fp64_peak(B, torch):
    """FP64 FMA throughput (TFLOP/s) of this GPU, measured in this run: the
    denominator of the FP64-bound kernels' rooflines (MEASURED_PEAKS.json
    covers HBM and bf16 only)."""
    probe = load_probe()
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    sms = B.num_sms()
    blocks = sms * 8
    iters = 4096
    s = torch.cuda.current_stream().cuda_stream
    probe.tb_probe_fp64_fma(blocks, iters, out.data_ptr(), s)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        probe.tb_probe_fp64_fma(blocks, iters, out.data_ptr(), s)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = max(best, blocks * 256 * iters * 16 / (ms * 1e-3) / 1e12)
    return best


def read_peaks():
    try:
        return json.load(open(os.path.join(HERE, 'MEASURED_PEAKS.json')))
    except Exception:
        return {}


MLP_FLOP_PER_EVAL = 2 * (16 * 128 + 3 * 128 * 128 + 128 * 32)  # dense BF16 flops of one network evaluation
# Algorithmic FP64 flops of one ring pair, counted on the formulas (FMA = 2;
# the Cody polynomials of K and E: 4 polynomials of degree 7, 14 flops each;
# the transcendental steps listed separately):
#   field pair (E_r, E_z sums):           87 flops + 1 log + 1 rsqrt + 1 reciprocal
#   potential + field pair:               90 flops + the same
#   ring potential term of the fill:      46 flops + 1 log + 1 rsqrt
#   axial derivative recurrence (9 terms): 54 flops + 1 sqrt + 2 divisions
FLOP_FIELD_PAIR = 87
FLOP_FIELD_PAIR_POT = 90
FLOP_RING_POT = 46
FLOP_AXIAL_RING = 54
FALLBACK_BF16_TFLOPS = 1590.0  # dense bf16 burst of a cuBLAS GEMM on this pool's B200s, used without MEASURED_PEAKS.json


def time_steps(fn, steps, flush):
    """Device time of `steps` calls of fn, enqueued back to back between CUDA
    events on the launching stream (the host runs ahead of the GPU, so a host
    pause -- garbage collection, the OS -- does not enter the measurement).
    L2 is flushed (a 256 MiB write, ~0.04 ms) before every step; that write
    is inside the step's time."""
    import torch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    results = []
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push('timed_steps')  # lets a profiler select the timed launches
    ev[0].record()
    for i in range(steps):
        flush.fill_(1.0)
        results.append(fn())
        ev[i + 1].record()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    return ms, results


def timed_launches(fn, steps, flush):
    """Device time (ms) of `steps` launches of fn, each after an L2 flush:
    one eager call, then fn captured as a CUDA graph whose replays are timed
    (so the host's launch overhead stays out of the short launches); returns
    (ms list, the captured call's result, refreshed by every replay)."""
    import torch
    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode='thread_local'):
        res = fn()
    ms, _ = time_steps(g.replay, steps, flush)
    res._graph = g  # the outputs live in the graph's memory pool
    return ms, res


def run_gpu(args):
    import torch
    ws, rank, local = dist_info()
    cores = host_cores()
    E = args.electrons
    beam = args.beam
    other = 'narrow' if beam == 'wide' else 'wide'
    geo, volts, p0, v0 = lens_inputs(E, beam, SEED + rank)
    _, _, p0o, v0o = lens_inputs(E, other, SEED + rank + 1000)
    # ---- the CPU oracle starts first and overlaps the GPU work (rank 0)
    oracle_pool = None
    n_check = min(args.check, E) if rank == 0 else 0
    n_check_o = min(args.check_other, E) if rank == 0 else 0
    t_or = time.perf_counter()
    q_or = jac_or = pos_or = None
    if n_check or n_check_o or (ws == 1 and args.cpu_seconds > 0):
        q_or, jac_or, pos_or = oracle_charges(geo, volts, cores)
    if n_check or n_check_o:
        oracle_pool = OracleTraces(q_or, jac_or, pos_or, max(1, cores - 1))
        oracle_pool.submit(beam, p0[:n_check], v0[:n_check])
        oracle_pool.submit(other, p0o[:n_check_o], v0o[:n_check_o])
    oracle_setup_s = time.perf_counter() - t_or

    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=300))
    from traceon_b200 import backend as B
    from traceon_b200 import geometry as G
    from traceon_b200.solver import ElectrostaticSolverRadial
    from traceon_b200.excitation import Mesh, Excitation
    from traceon_b200.tracing import Tracer
    from scipy.constants import e as qe, m_e

    # ---- setup (timed separately, not part of a step): GPU solve
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, volts)})
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    field = ElectrostaticSolverRadial(exc).solve_matrix()[0]
    torch.cuda.synchronize()
    setup = {'solve_s': time.perf_counter() - t0, 'oracle_charges_s': oracle_setup_s}
    bem_tracer = Tracer(field, G.LENS_BOUNDS)
    Nq = len(field.electrostatic_point_charges) * B.N_QUAD_2D
    sur = None
    if args.field == 'surrogate':
        from traceon_b200.surrogate import SurrogateTrainer, FieldSurrogate
        t0 = time.perf_counter()
        trainer = SurrogateTrainer(geo)
        model, info = trainer.train(n_samples=args.train_samples, steps=args.train_steps, batch=8192, seed=0)
        torch.cuda.synchronize()
        setup['surrogate_train_s'] = time.perf_counter() - t0
        setup['surrogate_holdout_mse'] = info['holdout_mse']
        setup['surrogate_train'] = (f'{args.train_samples} BEM samples of the unit-voltage fields, '
                                    f'{args.train_steps} Adam steps of 8192 (one network for every voltage setting '
                                    f'of this lens)')
        sur = FieldSurrogate(model, trainer.fields, trainer.z, trainer.tabs, volts, geo.segments, engine=args.engine)

    def start_of(p, v):
        return torch.as_tensor(np.concatenate([p, v], 1), device='cuda', dtype=torch.float64).contiguous()

    start, start_o = start_of(p0, v0), start_of(p0o, v0o)
    qm = torch.full((E,), -qe / m_e, device='cuda', dtype=torch.float64)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')
    MAXA = 20000

    def step_bem(st, q=qm):
        return bem_tracer.trace_device(st, q, atol=ATOL, plane_z=G.LENS_EXIT_Z, team_warps=args.team_warps,
                                       max_attempts=MAXA)

    sess = None
    if sur is not None:
        # the public batched API: static buffers, the step captured as a CUDA graph
        sess = sur.trace_session(E, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=ATOL, max_attempts=MAXA)
        sess.start.copy_(start)  # start states resident in HBM for `value`

    def step_sur():
        sess.replay_device()
        return sess

    step = step_sur if sur is not None else (lambda: step_bem(start))
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ms_list, results = time_steps(step, args.steps, flush)
    total_ms = float(np.sum(ms_list))
    if ws > 1:
        from traceon_b200.parallel import max_over_ranks
        total_ms = max_over_ranks(total_ms, device='cuda')
    res = results[-1]
    status = res.status.cpu().numpy()
    plane = res.plane.cpu().numpy()
    counters = res.counters.cpu().numpy()
    attempts = float(counters[:, 1].sum())
    value = ws * E * args.steps / (total_ms * 1e-3)

    # ---- e2e through the public API with host arrays: every step copies the
    # start states in (pinned staging, H2D) and the endpoints out (D2H)
    e2e_ms = []
    if sess is not None:
        # a stream of batches, each copied in from host arrays and its
        # endpoints copied out, two batches in flight; L2 flushed on each
        # batch's stream before its replay
        n_e2e = max(3, min(args.steps, 10))
        flush_l2 = lambda: flush.fill_(1.0)  # noqa: E731
        sess.run_many([(p0, v0)] * 2, before=flush_l2)  # warm-up: builds the second buffer set
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        outs = sess.run_many([(p0, v0)] * n_e2e, before=flush_l2)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t1) * 1e3 / n_e2e)
        h2d, d2h = sess.h2d_bytes, sess.d2h_bytes
        e2e_api = ('FieldSurrogate.trace_session(...).run_many([(positions, velocities), ...]): pinned staging, '
                   f'two CUDA-graph buffer sets in flight, {n_e2e} batches')
        # the session's outputs against the device-resident run
        assert np.array_equal(np.nan_to_num(outs[-1][0]), np.nan_to_num(plane)), \
            'session outputs differ from the device run'
    else:
        for _ in range(max(1, min(args.steps, 5))):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            bem_tracer.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=ATOL, team_warps=args.team_warps,
                                       max_attempts=MAXA)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t1) * 1e3)
        h2d, d2h = E * 6 * 8 + E * 8, E * (7 + 7) * 8 + E * 4 + E * 2 * 8
        e2e_api = 'Tracer.trace_endpoints(positions, velocities, ...)'
    e2e_value = ws * E / (np.median(e2e_ms) * 1e-3)

    # ---- the arms on both beams: surrogate, axial series alone, plain BEM
    # (a 16,384-electron slice); their exit-plane crossings for the errors
    arms = {}
    if sur is not None:
        m = min(E, args.bem_electrons)
        for name, st, pl_sur in ((beam, start, plane), (other, start_o, None)):
            row = {}
            if pl_sur is None:
                ms_s, r_s = timed_launches(
                    lambda: sur.trace_device(st, qm, G.LENS_BOUNDS, ATOL, plane_z=G.LENS_EXIT_Z, max_attempts=MAXA),
                    3, flush)
                pl_sur = r_s.plane.cpu().numpy()
                row['surrogate'] = {'value': E / (np.mean(ms_s) * 1e-3), 'ms_per_step': float(np.mean(ms_s)),
                                    'attempts_mean': float(r_s.counters[:, 1].double().mean()),
                                    'bem_fallback_evals': int(r_s.counters[:, 2].sum().item()),
                                    'status_exited': int((r_s.status == 0).sum().item())}
            else:
                row['surrogate'] = {'value': value, 'ms_per_step': total_ms / args.steps,
                                    'attempts_mean': attempts / E,
                                    'bem_fallback_evals': int(counters[:, 2].sum()),
                                    'status_exited': int((status == 0).sum())}
            ms_a, r_a = timed_launches(
                lambda: sur.trace_axial_device(st, qm, G.LENS_BOUNDS, ATOL, plane_z=G.LENS_EXIT_Z,
                                               max_attempts=MAXA), 3, flush)
            pl_ax = r_a.plane.cpu().numpy()
            row['axial_only'] = {'value': E / (np.mean(ms_a) * 1e-3), 'ms_per_step': float(np.mean(ms_a)),
                                 'attempts_mean': float(r_a.counters[:, 1].double().mean()),
                                 'status_exited': int((r_a.status == 0).sum().item()),
                                 'kernel': 'k_trace_axial'}
            st_m, qm_m = st[:m].contiguous(), qm[:m].contiguous()
            ms_b, r_b = timed_launches(lambda: step_bem(st_m, qm_m), 2, flush)
            pl_bem = r_b.plane.cpu().numpy()
            pairs = float(r_b.counters[:, 1].sum().item()) * 6 * Nq
            launch_s = np.mean(ms_b) * 1e-3
            row['plain_bem'] = {'value': ws * m / launch_s, 'electrons': m, 'ms_per_step': float(np.mean(ms_b)),
                                'kernel': 'k_trace_bem',
                                'roofline': {'bound': 'fp64', 'unit': 'TFLOP/s', 'flop_per_pair': FLOP_FIELD_PAIR,
                                             'achieved': pairs * FLOP_FIELD_PAIR / launch_s / 1e12,
                                             'unit_desc': 'ring-pair field evaluations, algorithmic FP64 flops '
                                                          '(+ 1 log, 1 rsqrt, 1 reciprocal per pair)'}}
            row['speedup_surrogate_vs_plain_bem'] = row['surrogate']['value'] / row['plain_bem']['value']
            row['speedup_axial_only_vs_plain_bem'] = row['axial_only']['value'] / row['plain_bem']['value']
            # errors against the GPU FP64 BEM trace of the slice (itself
            # pinned to the CPU oracle by the parity tests)
            row['err_vs_gpu_bem'] = {'surrogate': endpoint_errors_nm(pl_sur[:m], pl_bem[:, 1:3]),
                                     'axial_only': endpoint_errors_nm(pl_ax[:m], pl_bem[:, 1:3])}
            row['_planes'] = (pl_sur, pl_ax)
            arms[name] = row

    if rank != 0:
        if oracle_pool is not None:
            oracle_pool.close()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel
    peaks = read_peaks()
    fp64_peak = measure_fp64_peak(B, torch)
    launch_s = total_ms / args.steps * 1e-3
    if sur is not None:
        evals = attempts * 6
        achieved = evals * MLP_FLOP_PER_EVAL / launch_s / 1e12
        peak = peaks.get('bf16_tflops')
        peak_source = 'MEASURED_PEAKS.json bf16_tflops (burst)'
        if not peak:  # no measurement on this pool: the earlier burst figure of a cuBLAS bf16 GEMM here
            peak, peak_source = FALLBACK_BF16_TFLOPS, 'fallback: 1,590 TFLOP/s bf16 burst measured earlier on this pool'
        roof = {'bound': 'tensor', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                'frac': achieved / peak if peak else None,
                'traffic': args.traffic if args.engine == 'tc' else None, 'traffic_unit': 'bytes per launch (ncu)',
                'kernel': 'k_trace_surrogate_tc' if args.engine == 'tc' else 'k_trace_surrogate',
                'flop_per_unit': MLP_FLOP_PER_EVAL, 'units_per_launch': evals,
                'unit_desc': 'network evaluations (dense BF16 flops of the 16-128x4-32 MLP)',
                'peak_source': peak_source}
        for row in arms.values():
            rf = row['plain_bem']['roofline']
            rf['peak'] = fp64_peak
            rf['frac'] = rf['achieved'] / fp64_peak
            rf['peak_source'] = 'FP64 FMA throughput measured in this run (tests/probe tb_probe_fp64_fma)'
    else:
        pairs_per_launch = attempts * 6 * Nq
        achieved = pairs_per_launch * FLOP_FIELD_PAIR / launch_s / 1e12
        roof = {'bound': 'fp64', 'achieved': achieved, 'peak': fp64_peak, 'unit': 'TFLOP/s',
                'frac': achieved / fp64_peak if fp64_peak else None, 'traffic': None, 'kernel': 'k_trace_bem',
                'flop_per_unit': FLOP_FIELD_PAIR, 'units_per_launch': pairs_per_launch,
                'unit_desc': 'ring-pair field evaluations, algorithmic FP64 flops (+ 1 log, 1 rsqrt, '
                             '1 reciprocal per pair)',
                'peak_source': 'FP64 FMA throughput measured in this run (tests/probe tb_probe_fp64_fma)'}

    precision = precision_solve(args.precision_n, fp64_peak=fp64_peak, field_points=args.field_points,
                                keep_state=True) if args.precision_n > 0 else None

    # ---- accuracy against the CPU oracle (the held-out sample of each beam)
    accuracy = {'checked_against': 'CPU oracle: FP64 fill + QUADPACK diagonal + LAPACK solve on the host, FP64 BEM '
                                   'RKF45 trace, cubic-Hermite crossing of the exit plane'}
    if oracle_pool is not None:
        for name, n_c in ((beam, n_check), (other, n_check_o)):
            if not n_c:
                continue
            ref_xy = oracle_pool.result(name)
            row = arms.get(name)
            if row is not None:
                pl_sur, pl_ax = row['_planes']
                row['err_vs_oracle'] = {'surrogate': endpoint_errors_nm(pl_sur[:n_c], ref_xy),
                                        'axial_only': endpoint_errors_nm(pl_ax[:n_c], ref_xy)}
            elif name == beam:
                accuracy[name] = endpoint_errors_nm(plane[:n_c], ref_xy)
        accuracy['oracle_wall_s'] = oracle_pool.close()
        accuracy['oracle_workers'] = oracle_pool.workers
    if q_or is not None:
        q_gpu = field.electrostatic_point_charges.charges
        accuracy['charges_rel_err'] = float(np.max(np.abs(q_gpu - q_or)) / np.abs(q_or).max())
    if beam in arms and 'err_vs_oracle' in arms[beam]:
        eh = arms[beam]['err_vs_oracle']['surrogate']
        accuracy.update({'endpoint_err_max_nm': eh['max_nm'], 'endpoint_err_p99_nm': eh['p99_nm'],
                         'checked_electrons': eh['n'], 'checked_fraction': eh['n'] / E})
    for row in arms.values():
        row.pop('_planes', None)
    if precision is not None and args.field_check > 0:
        precision.update(precision_field_check(precision.pop('_field_state'), args.field_check, cores))
    elif precision is not None:
        precision.pop('_field_state', None)

    # ---- CPU baselines (rank 0, N = 1): the reference's plain-BEM tracer and
    # its axial-series tracer on this beam, all host threads, bounded samples
    cpu = cpu_axial = None
    if ws == 1 and args.cpu_seconds > 0 and q_or is not None:
        rate, n, kind = cpu_reference_rate(q_or, jac_or, pos_or, p0, v0, cores, args.cpu_seconds)
        cpu = {'value': rate, 'unit': 'electrons/s', 'cores': cores, 'kind': 'reference' if kind == 'ref' else 'port',
               'sample': f'{n} electrons of this beam traced by the reference C backend (trace_particle + '
                         f'field_radial_traceable, plain BEM; the reference has no surrogate) on {cores} threads '
                         f'for ~{args.cpu_seconds:.0f} s'}
        if sur is not None:
            coeffs = reference_axial_table(q_or, jac_or, pos_or, sur.z)
            rate, n, kind = cpu_reference_rate(q_or, jac_or, pos_or, p0, v0, cores, args.cpu_seconds / 2,
                                               axial=(sur.z, coeffs))
            cpu_axial = {'value': rate, 'unit': 'electrons/s', 'cores': cores,
                         'kind': 'reference' if kind == 'ref' else 'port',
                         'sample': f'{n} electrons of this beam traced by the reference C backend through its axial '
                                   f'series (trace_particle + field_radial_derivs_traceable, FieldRadialAxial '
                                   f'table of {len(sur.z)} z-points) on {cores} threads for '
                                   f'~{args.cpu_seconds / 2:.0f} s'}

    if sur is not None and beam in arms:
        sp = arms[beam]['plain_bem']['value']
        # electrons after which training + surrogate tracing beats the plain BEM tracer
        setup['break_even_electrons'] = setup['surrogate_train_s'] / max(1.0 / sp - 1.0 / value, 1e-30)
    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
            'step_ms': {'min': float(np.min(ms_list)), 'median': float(np.median(ms_list)),
                        'max': float(np.max(ms_list))},
            'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'bf16+f64' if sur is not None else 'f64',
            'data': 'synthetic', 'config': workload_config(E, args.field, beam),
            'e2e': {'value': e2e_value, 'unit': 'electrons/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                    'api': e2e_api},
            'gpu_launches': args.steps, 'roofline': roof,
            'speedup_vs_plain_bem': arms[beam]['speedup_surrogate_vs_plain_bem'] if beam in arms else None,
            'beams': arms or None,
            'cpu_baseline': cpu, 'cpu_baseline_axial': cpu_axial, 'clocks': clk.summary(),
            'accuracy': accuracy,
            'trace_stats': {'status_exited': int((status == 0).sum()),
                            'accepted_steps_mean': float(counters[:, 0].mean()),
                            'attempts_mean': float(counters[:, 1].mean()),
                            'bem_fallback_evals': int(counters[:, 2].sum()) if counters.shape[1] > 2 else None},
            'setup': setup, 'precision_solve': precision}
    print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_solve(args):
    """--workload solve: only the precision workload's fill and solves (one
    JSON line; used for the solver's profiles)."""
    import torch
    torch.cuda.set_device(dist_info()[2])
    from traceon_b200 import backend as B
    p = precision_solve(args.precision_n, fp64_lu=not args.skip_fp64_lu, fp64_peak=measure_fp64_peak(B, torch),
                        check=args.field_check, field_points=args.field_points)
    line = {'metric': 'mixed-precision charge solve time (precision workload)', 'value': p['solve_mixed_ms'],
            'unit': 'ms', 'higher_is_better': False, 'n_gpus': 1, 'dtype': 'f32 tensor-core LU + f64 refinement',
            'data': 'synthetic', 'config': {'workload': p['workload'], 'elements': args.precision_n},
            'precision_solve': p}
    print(json.dumps(line), flush=True)


COMBINED_VOLTS = (0.0, 3000.0, 0.0)


def _log(t0, msg):
    """A progress line on stderr (seconds since t0), for the long workloads."""
    sys.stderr.write(f'[{time.perf_counter() - t0:8.1f} s] {msg}\n')
    sys.stderr.flush()


def run_combined(args):
    """--workload combined: the combined electro-magnetostatic workload.  The
    einzel lens meshed to 16,384 elements inside an iron pole piece
    (mu_r = 1000) of 16,384 magnetizable elements magnetised by 4 coils (r ~
    U[3, 6] mm, U[0.5, 5] kA-turns): both systems filled on the GPU and solved
    by the mixed solve (beside the vendor FP64 LU), the surrogate trained on
    (phi, E, H) of the 3 electrodes and 4 coils at unit strength, then
    1,048,576 electrons at 5 keV (lognormal 2 %) traced through E + B by the
    tensor-core surrogate tracer; the plain BEM tracer on a slice for the
    comparison and as the reference for the slice's endpoints; a sample re-traced
    by the CPU oracle."""
    import torch
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    from traceon_b200 import backend as B
    from traceon_b200 import geometry as G
    from traceon_b200.excitation import Excitation, Mesh
    from traceon_b200.field import EffectivePointCharges
    from traceon_b200.solver import ElectrostaticSolverRadial, MagnetostaticSolverRadial
    from traceon_b200.surrogate import SurrogateTrainer, FieldSurrogate
    from traceon_b200.tracing import Tracer
    from scipy.constants import e as qe, m_e

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    T0 = time.perf_counter()
    cl = G.combined_lens(SEED, n_elec=args.combined_n, n_mag=args.combined_n)
    geo = cl.geometry
    _log(T0, f'combined lens: {len(geo)} elements')
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: v for n, v in zip(geo.names[:3], COMBINED_VOLTS)})
    exc.add_magnetizable(pole=1000.0)
    coils = EffectivePointCharges(*cl.coil_sources())
    se = ElectrostaticSolverRadial(exc)
    sm = MagnetostaticSolverRadial(exc, current_point_charges=coils)
    solve = {}
    fields = []
    for name, sv in (('electrostatic', se), ('magnetostatic', sm)):
        A = sv.get_matrix_device()
        F = sv.get_right_hand_side_device()[None].contiguous()
        B.dev_solve_mixed(A, F)
        fill_ms, _ = timed(sv.get_matrix_device)
        rhs_ms, _ = timed(sv.get_right_hand_side_device)
        mixed_ms, (X, iters, rel) = timed(lambda: B.dev_solve_mixed(A, F))
        torch.linalg.solve(A, F.T)
        vendor_ms, X64 = timed(lambda: torch.linalg.solve(A, F.T))
        err = float(((X[0] - X64[:, 0]).abs().max() / X64.abs().max()).item())
        solve[name] = {'elements': len(sv.vertices), 'fill_fp64_ms': fill_ms, 'rhs_ms': rhs_ms,
                       'solve_mixed_ms': mixed_ms, 'mixed_iterations': iters,
                       'solve_fp64_vendor_lu_ms': vendor_ms, 'speedup_vs_vendor_fp64_lu': vendor_ms / mixed_ms,
                       'charges_rel_err_vs_fp64': err}
        jac, pos = sv.jacobians_and_positions()
        fields.append(sv.charges_to_field(EffectivePointCharges(X[0].cpu().numpy(), jac, pos)))
        del A
        torch.cuda.empty_cache()
        _log(T0, f'{name} system filled and solved: {solve[name]}')
    field = fields[0] + fields[1]
    t0 = time.perf_counter()
    tr = SurrogateTrainer(geo, r_max=args.combined_r_max, electrodes=geo.names[:3], magnetizable={'pole': 1000.0},
                          coils=cl)
    _log(T0, 'unit fields and axial tables of the 7 sources')
    model, info = tr.train(n_samples=args.train_samples, steps=args.train_steps, batch=8192, seed=0)
    _log(T0, f'surrogate trained: holdout mse {info["holdout_mse"]:.3g}')
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    strengths = np.concatenate([COMBINED_VOLTS, cl.coil_current])
    fs = FieldSurrogate(model, tr.fields, tr.z, tr.tabs, strengths, geo.segments, engine=args.engine)
    E = args.combined_electrons
    p0, v0 = G.combined_beam(E, SEED + 200)
    start = torch.as_tensor(np.concatenate([p0, v0], 1), device='cuda')
    qm = torch.full((E,), -qe / m_e, device='cuda', dtype=torch.float64)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')

    def run():
        return fs.trace_device(start, qm, G.LENS_BOUNDS, ATOL, plane_z=G.LENS_EXIT_Z, max_attempts=50000)

    run()
    torch.cuda.synchronize()
    _log(T0, 'first surrogate trace done')
    with Clocks(local) as clk:
        ms, res = time_steps(run, args.steps, flush)
    _log(T0, f'timed surrogate traces: {np.mean(ms):.1f} ms per step')
    res = res[-1]
    plane = res.plane.cpu().numpy()
    status = res.status.cpu().numpy()
    counters = res.counters.cpu().numpy()
    value = E / (np.mean(ms) * 1e-3)
    m = min(E, args.combined_bem_electrons)
    bem = Tracer(field, G.LENS_BOUNDS)
    st_m, qm_m = start[:m].contiguous(), qm[:m].contiguous()
    ms_b, r_b = timed_launches(lambda: bem.trace_device(st_m, qm_m, atol=ATOL, plane_z=G.LENS_EXIT_Z,
                                                        max_attempts=50000), 1, flush)
    pl_b = r_b.plane.cpu().numpy()
    plain = {'value': m / (np.mean(ms_b) * 1e-3), 'electrons': m, 'ms_per_step': float(np.mean(ms_b))}
    _log(T0, f'plain BEM slice: {plain}')
    acc = {'vs_gpu_bem': endpoint_errors_nm(plane[:m], pl_b[:, 1:3])}
    evals = float(counters[:, 1].sum()) * 6
    peak = read_peaks().get('bf16_tflops') or FALLBACK_BF16_TFLOPS
    achieved = evals * MLP_FLOP_PER_EVAL / (np.mean(ms) * 1e-3) / 1e12
    # the exact sums of the fallback points: every point sums the
    # electrostatic and the magnetizable rings (16 per element), FP64
    fallback_pairs = float(counters[:, 2].sum()) * 16.0 * (len(se.vertices) + len(sm.vertices))
    fp64_peak = measure_fp64_peak(B, torch)
    fallback_roofline = fp64_roofline(fallback_pairs, FLOP_FIELD_PAIR, float(np.mean(ms)), fp64_peak,
                                      'k_trace_surrogate_tc<MAG> (group BEM sums of the fallback points)',
                                      'ring-pair field evaluations (+ 1 log, 1 rsqrt, 1 reciprocal each); '
                                      'the current rings are not counted')
    if args.combined_check > 0:
        from oracle.oracle import Oracle, EM, hermite_plane_crossing
        from concurrent.futures import ThreadPoolExecutor
        port = Oracle('port')
        qe_, qm_ = fields[0].electrostatic_point_charges, fields[1].magnetostatic_point_charges
        cur = cl.coil_sources()
        n_c = min(args.combined_check, m)

        def one(i):
            t, s_ = port.trace_bem(p0[i], v0[i], EM, qe_.charges, qe_.jacobians, qe_.positions, G.LENS_BOUNDS, ATOL,
                                   mag=(qm_.charges, qm_.jacobians, qm_.positions), current=cur)
            h = hermite_plane_crossing(t, s_, G.LENS_EXIT_Z)
            return (np.nan, np.nan) if h is None else (h[0], h[1])

        with ThreadPoolExecutor(host_cores()) as ex:
            ref = np.array(list(ex.map(one, range(n_c))))
        acc['vs_cpu_oracle'] = endpoint_errors_nm(plane[:n_c], ref)
        _log(T0, f'oracle traces: {acc["vs_cpu_oracle"]}')
        acc['vs_cpu_oracle_note'] = 'the GPU solve\'s charges traced by the oracle (FP64 BEM, E + B)'
    line = {'metric': 'traced electrons/s at <=1 nm endpoint error, combined electro-magnetostatic lens, '
                      'surrogate (phi, E, B) vs plain BEM field', 'value': value, 'unit': 'electrons/s',
            'n_gpus': 1, 'steps': args.steps, 'ms_per_step': float(np.mean(ms)), 'higher_is_better': True,
            'dtype': 'bf16+f64', 'data': 'synthetic',
            'config': {'workload': f'combined electro-magnetostatic lens: einzel lens of {args.combined_n} elements '
                                   f'(0 / 3 kV / 0) in an iron pole piece (mu_r 1000) of {args.combined_n} elements, '
                                   f'4 coils {np.round(cl.coil_current).tolist()} A-turns; {E} electrons at 5 keV '
                                   f'(lognormal 2 %), r0 <= 0.2 mm, +-10 mrad, RKF45 atol 1e-10 m',
                       'electrons_per_step': E, 'surrogate_r_max_m': args.combined_r_max},
            'solve': solve, 'surrogate_train_s': train_s, 'surrogate_holdout_mse': info['holdout_mse'],
            'plain_bem': plain, 'speedup_vs_plain_bem': value / plain['value'],
            'roofline': {'bound': 'tensor', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                         'frac': achieved / peak, 'kernel': 'k_trace_surrogate_tc<MAG>',
                         'flop_per_unit': MLP_FLOP_PER_EVAL, 'units_per_launch': evals},
            'roofline_fallback_fp64': fallback_roofline,
            'trace_stats': {'status_exited': int((status == 0).sum()), 'attempts_mean': float(counters[:, 1].mean()),
                            'bem_fallback_evals': int(counters[:, 2].sum())},
            'accuracy': acc, 'clocks': clk.summary()}
    print(json.dumps(line), flush=True)


def _batch_oracle_init(items):
    try:
        os.nice(10)
    except OSError:
        pass
    from oracle.oracle import Oracle
    _ORACLE.update(oracle=Oracle('port'), items=items)


def _batch_oracle_one(job):
    """The oracle's FP64 BEM trace of one particle of geometry g (the GPU
    solve's charges): its final state (t, x, y, z) and its position at the
    GPU trace's final time t_gpu (cubic Hermite between accepted states)."""
    g, state, atol, t_gpu = job
    from oracle.oracle import EM, hermite_position_at
    q, jac, pos, bounds = _ORACLE['items'][g]
    t, s = _ORACLE['oracle'].trace_bem(state[:3], state[3:], EM, q, jac, pos, bounds, atol, max_attempts=20000)
    p = hermite_position_at(t, s, t_gpu)
    return (float(t[-1]), float(s[-1, 0]), float(s[-1, 1]), float(s[-1, 2]), float(p[0]), float(p[1]), float(p[2]),
            len(t))


def run_batch(args):
    """--workload batch: the batching workload.  64 mirror lenses (a
    random_lens stack of 2-5 tubes, radii U[0.5, 3] mm, gaps U[0.2, 1] mm,
    electrodes U[-5, 5] kV, followed by an aperture-plate mirror at -1.1 kV;
    N ~ U[500, 6000] elements each) filled, factored and solved in one
    persistent launch, then 65,536 electrons per lens (lognormal energies,
    median 1 keV, sigma 1, clipped to [100 eV, 10 keV]; angles U[-50, 50]
    mrad) traced through the direct BEM field in one more; the two captured as
    one CUDA graph with launch shapes picked by the autotuner.  A step is one
    replay of the graph.  Oracle checks: the charges of the smallest lenses
    against its own fill and LAPACK solve, and a seeded subsample of every
    lens's electrons traced by the oracle through the GPU charges."""
    import torch
    torch.cuda.set_device(dist_info()[2])
    from traceon_b200 import backend as B
    from traceon_b200 import geometry as G
    from traceon_b200 import autotune
    from traceon_b200.batch import BatchPipeline
    from traceon_b200.excitation import Excitation, Mesh
    cores = host_cores()
    ng, ne = args.batch_geometries, args.batch_electrons
    lenses = [G.mirror_lens(SEED * 1000 + g) for g in range(ng)]
    excs, starts = [], []
    for g, m in enumerate(lenses):
        exc = Excitation(Mesh.from_geometry(m.geometry))
        exc.add_voltage(**{n: float(v) for n, v in zip(m.geometry.names, m.voltages)})
        excs.append(exc)
        starts.append(G.mirror_beam(ne, SEED * 1000 + 500 + g, m.z_start))
    Ns = np.array([len(m.geometry) for m in lenses])
    t0 = time.perf_counter()
    pipe = BatchPipeline(excs, [s_[0] for s_ in starts], [s_[1] for s_ in starts], [m.bounds for m in lenses],
                         atol=args.batch_atol, max_attempts=20000)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    tuned = autotune.tune_batch_pipeline(pipe)
    pipe.batch.launch()
    pipe.batch.check()  # every lens solved without falling back
    status_solve = pipe.batch.status.cpu().numpy()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    solve_ms = [timed(pipe.batch.launch) for _ in range(2)]
    pipe.capture()
    for _ in range(args.warmup):
        pipe.replay()
    torch.cuda.synchronize()
    with Clocks(0) as clk:
        ms_list = [timed(pipe.replay) for _ in range(args.steps)]
    final = pipe.final.cpu().numpy()
    status = pipe.status.cpu().numpy()
    counters = pipe.counters.cpu().numpy()
    value = pipe.n / (np.mean(ms_list) * 1e-3)
    # how the electrons ended: back out of the entrance (reflected), through
    # the mirror bore, or out of the side of the box
    gid = np.repeat(np.arange(ng), pipe.counts)
    zlo = np.array([m.bounds[2, 0] for m in lenses])[gid]
    zhi = np.array([m.bounds[2, 1] for m in lenses])[gid]
    reflected = float(np.mean(final[:, 3] < zlo))
    through = float(np.mean(final[:, 3] > zhi))
    # the FP64 rooflines: ring-pair evaluations of the trace, ring potentials of the fill
    rings = 16 * Ns[gid]
    pairs = float(np.sum(counters[:, 1] * 6.0 * rings))
    fp64_peak = measure_fp64_peak(B, torch)
    trace_ms = float(np.mean(ms_list)) - float(np.mean(solve_ms))
    acc = {}
    # charges of the smallest lenses against the oracle's own fill + LAPACK
    from oracle.oracle import Oracle
    port = Oracle('port')
    err = []
    for g in np.argsort(Ns)[:args.batch_charge_check]:
        geo = lenses[g].geometry
        vals = geo.voltages_to_values(lenses[g].voltages)
        A = port.matrix(geo.vertices, np.ones(len(geo), np.uint8), vals, threads=cores)
        x = np.linalg.solve(A, vals)
        got = pipe.batch.charges[g].cpu().numpy()
        err.append(float(np.max(np.abs(got - x)) / np.max(np.abs(x))))
    acc['charges_rel_err_vs_oracle'] = {'max': max(err) if err else None, 'lenses': len(err),
                                        'elements': [int(Ns[g]) for g in np.argsort(Ns)[:args.batch_charge_check]]}
    if args.batch_check > 0:
        import multiprocessing as mp
        items = []
        for g, s_ in enumerate(pipe.batch.solvers):
            jac, pos = port.fill_jacobian_buffer_radial(s_.vertices)
            items.append((pipe.batch.charges[g].cpu().numpy(), jac, pos, lenses[g].bounds))
        rng = np.random.default_rng(SEED + 77)
        jobs, where = [], []
        offs = np.concatenate([[0], np.cumsum(pipe.counts)])
        start_h = pipe.start.cpu().numpy()
        for g in range(ng):
            pick = np.sort(rng.choice(pipe.counts[g], min(args.batch_check, pipe.counts[g]), replace=False))
            for i in pick:
                jobs.append((g, start_h[offs[g] + i], args.batch_atol, float(final[offs[g] + i, 0])))
                where.append(offs[g] + i)
        t1 = time.perf_counter()
        with mp.get_context('spawn').Pool(max(1, cores), _batch_oracle_init, (items,)) as pool:
            ref = np.array(pool.map(_batch_oracle_one, jobs, chunksize=4))
        got = final[where][:, :4]
        d_pos = np.max(np.abs(got[:, 1:] - ref[:, 1:4]), axis=1) * 1e9
        d_at = np.max(np.abs(got[:, 1:] - ref[:, 4:7]), axis=1) * 1e9
        d_t = np.abs(got[:, 0] - ref[:, 0]) / np.abs(ref[:, 0])
        worst = np.argsort(-d_at)[:5]
        acc['endpoints_vs_oracle'] = {
            'particles': len(jobs), 'per_lens': args.batch_check,
            'final_state_max_nm': float(d_pos.max()), 'final_state_p99_nm': float(np.percentile(d_pos, 99)),
            'final_state_within_1nm': int(np.sum(d_pos <= 1.0)), 'time_rel_max': float(d_t.max()),
            'at_gpu_time_max_nm': float(d_at.max()), 'at_gpu_time_p99_nm': float(np.percentile(d_at, 99)),
            'at_gpu_time_within_1nm': int(np.sum(d_at <= 1.0)),
            'worst': [{'lens': int(jobs[k][0]), 'status': int(status[where[k]]),
                       'attempts': int(counters[where[k], 1]), 'oracle_states': int(ref[k, 7]),
                       'time_rel': float(d_t[k]), 'final_state_nm': float(d_pos[k]), 'at_gpu_time_nm': float(d_at[k])}
                      for k in worst],
            'oracle_s': time.perf_counter() - t1, 'oracle_workers': max(1, cores),
            'note': 'the oracle\'s FP64 RKF45 through the GPU solve\'s charges: its final state (first point outside '
                    'the lens box) and its position at the GPU trace\'s final time'}
    line = {'metric': 'traced electrons/s, batching workload (fill + solve + trace of 64 lenses, one CUDA graph)',
            'value': value, 'unit': 'electrons/s', 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': float(np.mean(ms_list)), 'higher_is_better': True, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': f'{ng} mirror lenses, N ~ U[500, 6000] (sum {int(Ns.sum())}), {ne} electrons '
                                   f'each (lognormal energies median 1 keV, sigma 1, clipped 100 eV-10 keV; '
                                   f'+-50 mrad), direct BEM field, RKF45 atol {args.batch_atol:g} m',
                       'geometries': ng, 'electrons_per_geometry': ne, 'elements_total': int(Ns.sum()),
                       'elements_min_max': [int(Ns.min()), int(Ns.max())]},
            'graph': {'launches_per_replay': 2, 'kernels': ['k_batch_solve', 'k_trace_bem'],
                      'memset_nodes_per_replay': 3},
            'solve_ms': float(np.mean(solve_ms)), 'trace_ms': trace_ms,
            'solve_status': {'ok': int(np.sum(status_solve == 0)), 'fallback_lu': int(np.sum(status_solve == 5))},
            'autotune': tuned,
            'trace_stats': {'status_exited': int(np.sum(status == 0)), 'max_attempts': int(np.sum(status == 1)),
                            'reflected_fraction': reflected, 'through_mirror_fraction': through,
                            'side_exit_fraction': 1.0 - reflected - through,
                            'attempts_mean': float(counters[:, 1].mean()),
                            'attempts_p50_p99_max': [float(np.percentile(counters[:, 1], 50)),
                                                     float(np.percentile(counters[:, 1], 99)),
                                                     int(counters[:, 1].max())]},
            'trace_roofline': fp64_roofline(pairs, FLOP_FIELD_PAIR, trace_ms, fp64_peak, 'k_trace_bem',
                                            'ring-pair field evaluations (+ 1 log, 1 rsqrt, 1 reciprocal each)'),
            'setup_s': setup_s, 'accuracy': acc, 'clocks': clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='tracer', choices=['tracer', 'solve', 'combined', 'batch'],
                    help='tracer: the headline metric (default); solve: only the precision-workload solve; '
                         'combined: the combined electro-magnetostatic workload')
    ap.add_argument('--combined-n', type=int, default=16384, help='elements of each part of the combined lens')
    ap.add_argument('--combined-electrons', type=int, default=1 << 20)
    ap.add_argument('--combined-r-max', type=float, default=0.95e-3,
                    help='radius of the combined surrogate\'s domain (m); points beyond it use the exact BEM sums')
    ap.add_argument('--combined-bem-electrons', type=int, default=2048)
    ap.add_argument('--combined-check', type=int, default=16,
                    help='electrons of the combined workload re-traced by the CPU oracle (~1.5 min each per core)')
    ap.add_argument('--batch-geometries', type=int, default=64)
    ap.add_argument('--batch-electrons', type=int, default=65536, help='electrons per lens of the batching workload')
    ap.add_argument('--batch-atol', type=float, default=1e-8)
    ap.add_argument('--batch-check', type=int, default=32, help='electrons per lens re-traced by the CPU oracle')
    ap.add_argument('--batch-charge-check', type=int, default=4, help='smallest lenses solved by the CPU oracle')
    ap.add_argument('--electrons', type=int, default=262144)
    ap.add_argument('--field', default='surrogate', choices=['surrogate', 'bem'])
    ap.add_argument('--bem-electrons', type=int, default=16384, help='slice traced with the plain BEM field')
    ap.add_argument('--train-samples', type=int, default=1 << 22)
    ap.add_argument('--train-steps', type=int, default=80000)
    ap.add_argument('--team-warps', type=int, default=0)
    ap.add_argument('--engine', default='tc', choices=['tc', 'warp'],
                    help='surrogate network engine: tcgen05 (tc) or warp-level mma.sync (warp)')
    ap.add_argument('--beam', default='wide', choices=sorted(BEAMS),
                    help='beam of the headline number (the other beam is measured beside it)')
    ap.add_argument('--check', type=int, default=2621,
                    help='electrons of the headline beam re-traced by the CPU oracle (default: 1 %% of 262,144)')
    ap.add_argument('--check-other', type=int, default=256,
                    help='electrons of the other beam re-traced by the CPU oracle')
    ap.add_argument('--field-points', type=int, default=1 << 20,
                    help='points of the precision workload field evaluation')
    ap.add_argument('--field-check', type=int, default=4096,
                    help='points of the precision workload field re-evaluated by the CPU oracle')
    ap.add_argument('--cpu-seconds', type=float, default=15.0)
    ap.add_argument('--skip-fp64-lu', action='store_true',
                    help='--workload solve: time only the mixed solve (for profiles)')
    ap.add_argument('--precision-n', type=int, default=16384,
                    help='elements of the precision-workload solve measured beside the tracer (0: skip)')
    ap.add_argument('--ref-seconds', type=float, default=20.0)
    # DRAM bytes (read + write) of one full-size launch of the dominant kernel
    # from an ncu capture of this workload (k_trace_surrogate_tc, wide beam:
    # 17.06 MB read + 2.80 MB written; see the profile summary of that kernel)
    ap.add_argument('--traffic', type=float, default=19.86e6)
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'solve':
        run_solve(args)
    elif args.workload == 'combined':
        run_combined(args)
    elif args.workload == 'batch':
        run_batch(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
