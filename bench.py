"""Benchmark: traced electrons per second at <= 1 nm endpoint error through
the einzel-lens workload, learned surrogate vs plain BEM field.

Workload: the three-tube einzel lens of 1,000 cubic line elements graded
toward the tube edges (0 V / V_mid / 0 V, V_mid from the seed), solved once on
the GPU (FP64 fill, singular self terms, FP64 LU).  A step traces a batch of
electrons (default 262,144) at 1 keV +-5 %, angles +-20 mrad, start radius
<= 0.2 mm at z = -9.5 mm, with adaptive RKF45 at atol = 1e-10 m until they
leave the bounds (|x|,|y| <= 2 mm, |z| <= 10 mm), recording each electron's
crossing of the exit plane z = +9.5 mm.  Synthetic inputs; no dataset.

  --field surrogate (default): the surrogate field (axial series + BF16 MLP
      correction trained on the GPU from BEM samples in the setup phase, BEM
      fallback near electrodes); the plain BEM tracer is measured beside it
      on a 16,384-electron slice of the same beam (`plain_bem`).
  --field bem: the plain FP64 BEM field only.
  --impl reference: the reference C backend's plain BEM tracer on host cores.
  --workload solve: only the precision workload's solve (the lens at
      --precision-n elements, 8 right-hand sides): GPU FP64 fill, FP64
      pivoted LU and the mixed tensor-core solve (also reported, as
      `precision_solve`, beside the tracer in the default run).

`value` is whole-job electrons/s with the start states resident in HBM;
`e2e` is the same through the public API with host arrays over a stream of
batches (two in flight), host<->device copies inside the timed region.  Endpoints of a sample of electrons are
checked every run against the full CPU oracle (oracle charges, FP64 BEM
trace): `accuracy.endpoint_err_max_nm` must stay <= 1.
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


def workload_config(electrons, field):
    desc = {'surrogate': 'learned surrogate field (axial series + BF16 MLP correction, BEM fallback)',
            'bem': 'plain BEM field (FP64)'}[field]
    return {'workload': f'einzel lens, {N_ELEMENTS} cubic elements, {desc}, {electrons} electrons/step at '
                        f'1 keV +-5%, +-20 mrad, r0<=0.2 mm, RKF45 atol=1e-10 m, exit plane z=+9.5 mm',
            'elements': N_ELEMENTS, 'electrons_per_step': electrons, 'atol_m': ATOL, 'seed': SEED,
            'field': field, 'l2': 'L2 flushed (256 MiB write, inside the step time) before every timed step'}


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
def lens_inputs(electrons, seed=SEED):
    from traceon_b200 import geometry as G
    geo = G.einzel_lens(N_ELEMENTS)
    volts = G.einzel_lens_voltages(SEED)
    p0, v0 = G.surrogate_beam(electrons, seed + 100)
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


def check_endpoints(plane_gpu, p0, v0, q, jac, pos, sample, threads):
    """Max |(x, y)| difference (nm) at the exit plane between the GPU and the
    CPU oracle (both cubic-Hermite crossings) on `sample` electrons."""
    from oracle.oracle import Oracle, EM, hermite_plane_crossing
    from traceon_b200 import geometry as G
    from concurrent.futures import ThreadPoolExecutor
    port = Oracle('port')

    def one(i):
        t, s = port.trace_bem(p0[i], v0[i], EM, q, jac, pos, G.LENS_BOUNDS, ATOL)
        h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
        return np.max(np.abs(plane_gpu[i, 1:3] - h[:2]))

    with ThreadPoolExecutor(threads) as ex:
        errs = list(ex.map(one, sample))
    return float(max(errs)) * 1e9, float(np.percentile(errs, 99)) * 1e9


def cpu_reference_rate(geo, q, jac, pos, p0, v0, threads, seconds, kind='ref'):
    """The reference's own CPU tracer (oracle/_ref: trace_particle with its
    field_radial_traceable callback) on `threads` host threads for about
    `seconds`; returns (electrons/s, electrons traced)."""
    from oracle.oracle import Oracle, EM, available
    from traceon_b200 import geometry as G
    if kind == 'ref' and not available('ref'):
        kind = 'port'
    o = Oracle(kind)
    done = []
    lock = threading.Lock()
    stop = time.perf_counter() + seconds
    counter = iter(range(len(p0)))

    def worker():
        while time.perf_counter() < stop:
            with lock:
                i = next(counter, None)
            if i is None:
                return
            o.trace_bem(p0[i], v0[i], EM, q, jac, pos, G.LENS_BOUNDS, ATOL)
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
    geo, volts, p0, v0 = lens_inputs(4096)
    q, jac, pos = oracle_charges(geo, volts, cores)
    for _ in range(args.warmup):
        cpu_reference_rate(geo, q, jac, pos, p0, v0, cores, 2.0)
    rates, n_total, t_total = [], 0, 0.0
    # each step a bounded sample: about two minutes of CPU work in total
    step_s = min(args.ref_seconds, max(2.0, 120.0 / max(args.steps, 1)))
    for s in range(args.steps):
        sl = slice((s * cores * 4) % len(p0), None)
        r, n, kind = cpu_reference_rate(geo, q, jac, pos, p0[sl], v0[sl], cores, step_s)
        rates.append(r)
        n_total += n
        t_total += n / r if r else 0
    value = n_total / t_total if t_total else 0.0
    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t_total / max(args.steps, 1), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': workload_config(args.electrons, args.field),
            'reference_field': 'plain BEM (the reference has no learned surrogate)',
            'cpu_baseline': {'value': value, 'unit': 'electrons/s', 'cores': cores,
                             'kind': 'reference' if kind == 'ref' else 'port',
                             'sample': f'{n_total} electrons over {args.steps} steps of ~{step_s:.0f} s '
                                       f'(reference C backend trace_particle + field_radial_traceable, '
                                       f'{cores} threads)'},
            'e2e': {'value': value, 'unit': 'electrons/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- precision solve
def precision_solve(n, nrhs=8, seed=2, field_points=1 << 20, fp64_lu=True):
    """The precision workload's charge solve: the three-electrode lens meshed
    to n cubic elements, nrhs right-hand sides with every electrode voltage
    ~U[-3, 3] kV.  GPU FP64 fill (+ singular self terms), then (a) the FP64
    LU with partial pivoting (numpy.linalg.solve's factorisation) and (b) the
    mixed solve (FP32 tensor-core LU of the equilibrated matrix, FP64
    iterative refinement).  CUDA-event times; charges of (b) against (a)."""
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

    def fill():
        jac, pos = B.dev_jacobian_buffer(v)
        B.dev_fill_matrix(A, v, t, val, jac, pos)
        B.dev_self_integrals(v, t, val, A)

    fill()  # warm-up
    fill_ms, _ = timed(fill)
    rng = np.random.default_rng(seed)
    F = torch.as_tensor(geo.voltages_to_values(rng.uniform(-3000, 3000, (nrhs, 3)).T).T.copy(), device='cuda')

    def lu64():
        LU = A.clone()
        _, perm = B.dev_lu_factor(LU)
        return B.dev_lu_solve(LU, perm, F)

    B.dev_solve_mixed(A, F)
    mixed_ms, (Xm, iters, rel) = timed(lambda: B.dev_solve_mixed(A, F))
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
    out = {'workload': f'einzel lens, {n} cubic elements, {nrhs} right-hand sides (electrode voltages U[-3,3] kV)',
           'fill_fp64_ms': fill_ms, 'solve_fp64_lu_ms': lu_ms, 'solve_mixed_ms': mixed_ms,
           'mixed_iterations': iters, 'mixed_last_correction': rel, 'charges_rel_err_vs_fp64': err,
           'solve_fp64_vendor_lu_ms': lib_ms,
           'speedup_vs_vendor_fp64_lu': lib_ms / mixed_ms if lib_ms else None,
           'speedup_solve': lu_ms / mixed_ms if lu_ms else None,
           'speedup_fill_plus_solve': (fill_ms + lu_ms) / (fill_ms + mixed_ms) if lu_ms else None,
           'lu_flop': 2.0 / 3.0 * n ** 3}
    del A
    torch.cuda.empty_cache()
    if field_points:
        out.update(precision_fields(geo, Xm[0], field_points, seed))
    return out


def precision_fields(geo, charges_t, m, seed, check=64):
    """Potential and field of the first right-hand side's charges at m points
    (x = r ~ U[0, 0.9] mm, y = 0, z ~ U[-8, 8] mm), FP64 ring sums on the GPU;
    `check` of them re-evaluated by the CPU oracle (its own element
    quadrature and the same charges) as the check."""
    import torch
    from traceon_b200 import backend as B
    from oracle.oracle import Oracle
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
    sample = rng.choice(m, check, replace=False)
    port = Oracle('port')
    q = charges_t.cpu().numpy()
    jac_o, pos_o = port.fill_jacobian_buffer_radial(geo.vertices)
    f_or = port.field_radial_many(pts[sample], q, jac_o, pos_o)
    p_or = port.potential_radial_many(pts[sample], q, jac_o, pos_o)
    f_gpu, p_gpu = fld.cpu().numpy()[sample], pot.cpu().numpy()[sample]
    ferr = float(np.max(np.abs(f_gpu - f_or)) / np.max(np.abs(f_or)))
    perr = float(np.max(np.abs(p_gpu - p_or)) / np.max(np.abs(p_or)))
    pairs = m * src.shape[1]
    return {'field_points': m, 'field_ms': ms, 'field_ring_pairs_per_s': pairs / (ms * 1e-3),
            'field_rel_err_vs_oracle': ferr, 'potential_rel_err_vs_oracle': perr, 'field_checked_points': check}


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
    denominator of the FP64-bound kernels' rooflines (the driver's measured
    peaks cover HBM and bf16 only)."""
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


MLP_FLOP_PER_EVAL = 2 * (16 * 128 + 3 * 128 * 128 + 128 * 16)  # dense BF16 flops of one network evaluation
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


def run_gpu(args):
    import torch
    ws, rank, local = dist_info()
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

    E = args.electrons
    geo, volts, p0, v0 = lens_inputs(E, SEED + rank)
    # ---- setup (timed separately, not part of a step): GPU solve
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, volts)})
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    field = ElectrostaticSolverRadial(exc).solve_matrix()[0]
    torch.cuda.synchronize()
    setup = {'solve_s': time.perf_counter() - t0}
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
        setup['surrogate_train'] = f'{args.train_samples} BEM samples, {args.train_steps} Adam steps of 8192'
        sur = FieldSurrogate(model, trainer.fields, trainer.z, trainer.tabs, volts, geo.segments, engine=args.engine)

    start = torch.as_tensor(np.concatenate([p0, v0], 1), device='cuda', dtype=torch.float64).contiguous()
    qm = torch.full((E,), -qe / m_e, device='cuda', dtype=torch.float64)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')

    def step_bem(st=start, q=qm):
        return bem_tracer.trace_device(st, q, atol=ATOL, plane_z=G.LENS_EXIT_Z, team_warps=args.team_warps,
                                       max_attempts=20000)

    sess = None
    if sur is not None:
        # the public batched API: static buffers, the step captured as a CUDA graph
        sess = sur.trace_session(E, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=ATOL, max_attempts=20000)
        sess.start.copy_(start)  # start states resident in HBM for `value`

    def step_sur():
        sess.replay_device()
        return sess

    step = step_sur if sur is not None else step_bem
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
    attempts = [int(counters[:, 1].sum())] * args.steps if sess is not None else \
        [int(r.counters[:, 1].sum().item()) for r in results]
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
                                       max_attempts=20000)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t1) * 1e3)
        h2d, d2h = E * 6 * 8 + E * 8, E * (7 + 7) * 8 + E * 4 + E * 2 * 8
        e2e_api = 'Tracer.trace_endpoints(positions, velocities, ...)'
    e2e_value = ws * E / (np.median(e2e_ms) * 1e-3)


    # ---- plain BEM tracer on a slice of the same beam (for the comparison)
    plain = None
    if sur is not None:
        m = min(E, args.bem_electrons)
        st_m, qm_m = start[:m].contiguous(), qm[:m].contiguous()
        step_bem(st_m, qm_m)
        ms_b, res_b = time_steps(lambda: step_bem(st_m, qm_m), 2, flush)
        pairs = np.mean([int(r.counters[:, 1].sum().item()) for r in res_b]) * 6 * Nq
        launch_s = np.mean(ms_b) * 1e-3
        plain = {'value': ws * m / launch_s, 'unit': 'electrons/s', 'electrons': m,
                 'ms_per_step': float(np.mean(ms_b)),
                 'roofline': {'bound': 'fp64', 'achieved': pairs * args.flop_per_pair / launch_s / 1e12,
                              'unit': 'TFLOP/s', 'kernel': 'k_trace_bem', 'flop_per_pair': args.flop_per_pair}}

    if rank != 0:
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
        evals = np.mean(attempts) * 6
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
                'unit_desc': 'network evaluations (dense BF16 flops of the 16-128x4-16 MLP)',
                'peak_source': peak_source}
        if plain is not None:
            plain['roofline']['peak'] = fp64_peak
            plain['roofline']['frac'] = plain['roofline']['achieved'] / fp64_peak
    else:
        pairs_per_launch = np.mean(attempts) * 6 * Nq
        achieved = pairs_per_launch * args.flop_per_pair / launch_s / 1e12
        roof = {'bound': 'fp64', 'achieved': achieved, 'peak': fp64_peak, 'unit': 'TFLOP/s',
                'frac': achieved / fp64_peak if fp64_peak else None, 'traffic': None, 'kernel': 'k_trace_bem',
                'flop_per_unit': args.flop_per_pair, 'units_per_launch': pairs_per_launch,
                'unit_desc': 'ring-pair field evaluations (executed FP64 flops per pair, ncu)',
                'peak_source': 'measured FP64 FMA probe (tb_probe_fp64_fma) in this run'}

    precision = precision_solve(args.precision_n) if args.precision_n > 0 else None

    # ---- accuracy vs the CPU oracle and the CPU baseline (rank 0, N = 1)
    cores = host_cores()
    q_or, jac_or, pos_or = oracle_charges(geo, volts, cores)
    q_gpu = field.electrostatic_point_charges.charges
    charge_err = float(np.max(np.abs(q_gpu - q_or)) / np.abs(q_or).max())
    rng = np.random.default_rng(7)
    sample = rng.choice(E, min(args.check, E), replace=False)
    err_max_nm = err_p99_nm = None
    if len(sample):
        err_max_nm, err_p99_nm = check_endpoints(plane, p0, v0, q_or, jac_or, pos_or, sample, cores)
    cpu = None
    if ws == 1 and args.cpu_seconds > 0:
        rate, n, kind = cpu_reference_rate(geo, q_or, jac_or, pos_or, p0, v0, cores, args.cpu_seconds)
        cpu = {'value': rate, 'unit': 'electrons/s', 'cores': cores, 'kind': 'reference' if kind == 'ref' else 'port',
               'sample': f'{n} electrons of this beam traced by the reference C backend (trace_particle + '
                         f'field_radial_traceable, plain BEM; the reference has no surrogate) on {cores} threads '
                         f'for ~{args.cpu_seconds:.0f} s'}

    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
            'step_ms': {'min': float(np.min(ms_list)), 'median': float(np.median(ms_list)),
                        'max': float(np.max(ms_list))},
            'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'bf16+f64' if sur is not None else 'f64',
            'data': 'synthetic', 'config': workload_config(E, args.field),
            'e2e': {'value': e2e_value, 'unit': 'electrons/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                    'api': e2e_api},
            'gpu_launches': args.steps, 'roofline': roof, 'plain_bem': plain,
            'speedup_vs_plain_bem': (value / plain['value']) if plain else None,
            'cpu_baseline': cpu, 'clocks': clk.summary(),
            'accuracy': {'endpoint_err_max_nm': err_max_nm, 'endpoint_err_p99_nm': err_p99_nm,
                         'checked_electrons': int(len(sample)), 'checked_against': 'CPU oracle FP64 BEM trace, Hermite crossing',
                         'charges_rel_err': charge_err},
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
    p = precision_solve(args.precision_n, fp64_lu=not args.skip_fp64_lu)
    line = {'metric': 'mixed-precision charge solve time (precision workload)', 'value': p['solve_mixed_ms'],
            'unit': 'ms', 'higher_is_better': False, 'n_gpus': 1, 'dtype': 'f32 tensor-core LU + f64 refinement',
            'data': 'synthetic', 'config': {'workload': p['workload'], 'elements': args.precision_n},
            'precision_solve': p}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='tracer', choices=['tracer', 'solve'],
                    help='tracer: the headline metric (default); solve: only the precision-workload solve')
    ap.add_argument('--electrons', type=int, default=262144)
    ap.add_argument('--field', default='surrogate', choices=['surrogate', 'bem'])
    ap.add_argument('--bem-electrons', type=int, default=16384, help='slice traced with the plain BEM field')
    ap.add_argument('--train-samples', type=int, default=1 << 22)
    ap.add_argument('--train-steps', type=int, default=40000)
    ap.add_argument('--team-warps', type=int, default=0)
    ap.add_argument('--engine', default='tc', choices=['tc', 'warp'],
                    help='surrogate network engine: tcgen05 (tc) or warp-level mma.sync (warp)')
    ap.add_argument('--check', type=int, default=16, help='electrons checked against the CPU oracle')
    ap.add_argument('--cpu-seconds', type=float, default=15.0)
    ap.add_argument('--skip-fp64-lu', action='store_true',
                    help='--workload solve: time only the mixed solve (for profiles)')
    ap.add_argument('--precision-n', type=int, default=16384,
                    help='elements of the precision-workload solve measured beside the tracer (0: skip)')
    ap.add_argument('--ref-seconds', type=float, default=20.0)
    # executed FP64 flops per ring-pair evaluation of the tracer's field sum
    # (dadd + dmul + 2 dfma per pair, from the ncu instruction counts)
    ap.add_argument('--flop-per-pair', type=float, default=162.0)
    # DRAM bytes (read + write) of one full-size launch of the dominant kernel
    # from an ncu capture of this workload (k_trace_surrogate_tc: 18.67 MB read
    # + 4.96 MB written; see the profile summary of that kernel)
    ap.add_argument('--traffic', type=float, default=23.63e6)
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'solve':
        run_solve(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
