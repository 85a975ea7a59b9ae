"""Benchmark: traced electrons per second through the einzel-lens workload.

Workload (one step): the three-tube einzel lens of 1,000 cubic line elements
graded toward the tube edges (0 V / V_mid / 0 V, V_mid from the seed), solved
once on the GPU (FP64 fill, singular self terms, FP64 LU); each step traces a
batch of 1 keV electrons (start r in [0, 0.2] mm, angle in [-5, 5] mrad,
z = -9.5 mm) with adaptive RKF45 at atol = 1e-10 m through the plain BEM
field until they leave the bounds (|x|,|y| <= 2 mm, |z| <= 10 mm), recording
each electron's crossing of the exit plane z = +9.5 mm.  Synthetic inputs;
no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--electrons E]
  python bench.py --impl reference ...   # the reference C backend on host cores

`value` is whole-job electrons/s with the start states resident in HBM;
`e2e` is the same through the public API (Tracer.trace_endpoints) with host
arrays, host<->device copies inside the timed region.  Endpoint accuracy is
checked every run against the CPU oracle on a sample of electrons.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_ELEMENTS = 1000
SEED = 1
ATOL = 1e-10
METRIC = 'traced electrons/s at <=1 nm endpoint error, plain BEM field'


def workload_config(electrons):
    return {'workload': f'einzel lens, {N_ELEMENTS} cubic elements, plain BEM field (FP64), '
                        f'{electrons} electrons/step at 1 keV, RKF45 atol=1e-10 m, exit plane z=+9.5 mm',
            'elements': N_ELEMENTS, 'electrons_per_step': electrons, 'atol_m': ATOL, 'seed': SEED,
            'field': 'plain BEM', 'l2': 'L2 flushed (256 MiB write) between timed steps'}


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
        self.path = os.path.join(HERE, 'gpurun_out', f'clocks_gpu{index}.csv')

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
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
    volts = G.einzel_lens_voltages(seed)
    p0, v0 = G.electron_beam(electrons, seed + 100)
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
    geo, volts, p0, v0 = lens_inputs(max(4096, args.electrons))
    q, jac, pos = oracle_charges(geo, volts, cores)
    for _ in range(args.warmup):
        cpu_reference_rate(geo, q, jac, pos, p0, v0, cores, 2.0)
    rates, n_total, t_total = [], 0, 0.0
    for s in range(args.steps):
        sl = slice((s * cores * 4) % len(p0), None)
        r, n, kind = cpu_reference_rate(geo, q, jac, pos, p0[sl], v0[sl], cores, args.ref_seconds)
        rates.append(r)
        n_total += n
        t_total += n / r if r else 0
    value = n_total / t_total if t_total else 0.0
    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t_total / max(args.steps, 1), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': workload_config(args.electrons),
            'cpu_baseline': {'value': value, 'unit': 'electrons/s', 'cores': cores,
                             'kind': 'reference' if kind == 'ref' else 'port',
                             'sample': f'{n_total} electrons over {args.steps} steps of ~{args.ref_seconds:.0f} s '
                                       f'(reference C backend trace_particle + field_radial_traceable, '
                                       f'{cores} threads)'},
            'e2e': {'value': value, 'unit': 'electrons/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def measure_fp64_peak(B, torch):
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    sms = B.num_sms()
    blocks = sms * 8
    iters = 4096
    s = torch.cuda.current_stream().cuda_stream
    B.backend_lib.tb_probe_fp64_fma(blocks, iters, out.data_ptr(), s)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.backend_lib.tb_probe_fp64_fma(blocks, iters, out.data_ptr(), s)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = max(best, blocks * 256 * iters * 16 / (ms * 1e-3) / 1e12)
    return best


def run_gpu(args):
    import torch
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
    from traceon_b200 import backend as B
    from traceon_b200 import geometry as G
    from traceon_b200.field import EffectivePointCharges, FieldRadialBEM
    from traceon_b200.solver import ElectrostaticSolverRadial
    from traceon_b200.excitation import Mesh, Excitation
    from traceon_b200.tracing import Tracer

    E = args.electrons
    geo, volts, p0, v0 = lens_inputs(E, SEED + rank)
    # ---- setup: GPU solve (timed separately, not part of a step)
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, volts)})
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solver = ElectrostaticSolverRadial(exc)
    field = solver.solve_matrix()[0]
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    tracer = Tracer(field, G.LENS_BOUNDS)
    Nq = len(field.electrostatic_point_charges) * B.N_QUAD_2D

    from scipy.constants import e as qe, m_e
    start = torch.as_tensor(np.concatenate([p0, v0], 1), device='cuda', dtype=torch.float64).contiguous()
    qm = torch.full((E,), -qe / m_e, device='cuda', dtype=torch.float64)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')

    def step_dev():
        return tracer.trace_device(start, qm, atol=ATOL, plane_z=G.LENS_EXIT_Z, team_warps=args.team_warps,
                                   max_attempts=20000)

    for _ in range(args.warmup):
        res = step_dev()
    torch.cuda.synchronize()

    # ---- timed device steps
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ms_list, attempts, launches = [], 0, 0
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = step_dev()
            e1.record()
            launches += 1
            torch.cuda.synchronize()
            ms_list.append(e0.elapsed_time(e1))
            attempts += int(res.counters[:, 1].sum().item())
        total_ms = float(np.sum(ms_list))
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    status = res.status.cpu().numpy()
    plane = res.plane.cpu().numpy()
    counters = res.counters.cpu().numpy()
    value = ws * E * args.steps / (total_ms * 1e-3)

    # ---- e2e through the public API with host arrays
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        out_plane, out_final, out_status, out_counters = tracer.trace_endpoints(p0, v0, G.LENS_EXIT_Z, atol=ATOL,
                                                                                team_warps=args.team_warps,
                                                                                max_attempts=20000)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_value = ws * E / (np.mean(e2e_ms) * 1e-3)
    h2d = E * 6 * 8 + E * 8
    d2h = E * (7 + 7) * 8 + E * 4 + E * 2 * 8

    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel (k_trace_bem): FP64 pipe
    pairs_per_launch = attempts / args.steps * 6 * Nq
    launch_s = total_ms / args.steps * 1e-3
    flop_per_pair = args.flop_per_pair
    achieved = pairs_per_launch * flop_per_pair / launch_s / 1e12
    peak = measure_fp64_peak(B, torch)

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
               'sample': f'{n} electrons of this workload traced by the reference C backend '
                         f'(trace_particle + field_radial_traceable) on {cores} threads for ~{args.cpu_seconds:.0f} s'}

    clocks = clk.summary()
    line = {'metric': METRIC, 'value': value, 'unit': 'electrons/s', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': total_ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': workload_config(E),
            'e2e': {'value': e2e_value, 'unit': 'electrons/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h},
            'gpu_launches': launches,
            'roofline': {'bound': 'fp64', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                         'frac': achieved / peak if peak else None, 'traffic': args.traffic,
                         'kernel': 'k_trace_bem', 'flop_per_pair': flop_per_pair,
                         'pairs_per_launch': pairs_per_launch,
                         'peak_source': 'measured FP64 FMA probe (tb_probe_fp64_fma) on this GPU'},
            'cpu_baseline': cpu,
            'clocks': clocks,
            'accuracy': {'endpoint_err_max_nm': err_max_nm, 'endpoint_err_p99_nm': err_p99_nm,
                         'checked_electrons': int(len(sample)), 'charges_rel_err': charge_err},
            'trace_stats': {'status_exited': int((status == 0).sum()),
                            'accepted_steps_mean': float(counters[:, 0].mean()),
                            'attempts_mean': float(counters[:, 1].mean())},
            'setup_solve_s': setup_s}
    print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--electrons', type=int, default=16384)
    ap.add_argument('--team-warps', type=int, default=0)
    ap.add_argument('--check', type=int, default=16, help='electrons checked against the CPU oracle')
    ap.add_argument('--cpu-seconds', type=float, default=15.0)
    ap.add_argument('--ref-seconds', type=float, default=20.0)
    # executed FP64 flops per ring-pair evaluation of the tracer's field sum
    # (dadd + dmul + 2 dfma per pair, from the ncu instruction counts)
    ap.add_argument('--flop-per-pair', type=float, default=162.0)
    ap.add_argument('--traffic', type=float, default=None)
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
