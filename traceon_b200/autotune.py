"""Measured choice of launch parameters.

The tracers' launch shapes depend on the workload: the plain BEM tracer
splits every field sum over a team of 1, 2, 4 or 8 warps, and the best team
size depends on how many particles there are per SM and how many rings each
field evaluation sums.  Instead of a fixed rule, `best_team_warps` times
every candidate on a bounded sample of the actual workload (CUDA events on
the launching stream) and keeps the fastest in a process-wide table keyed by
device and problem size, guarded by a lock (entry points may be called from
several host threads).

`tune_batch_pipeline` does the same for the batching workload's pipeline:
the CTAs per SM of the persistent tile-task solve (1 or 2; each CTA holds
two 64 x 64 FP64 tiles of shared memory) and the BEM team size of the
multi-geometry trace (on a sample of the batch's particles).

`tune_solve_lookahead` times the mixed solve at several lookahead widths
(the SMs left to the next panel's factorisation while a second stream runs
the rest of each trailing update; 0 = no lookahead) and sets the fastest.

The table is the library's only mutable global state; `clear()` empties it.
"""
from __future__ import annotations

import math
import threading

from . import backend as B

_lock = threading.Lock()
_table: dict = {}

TEAM_CANDIDATES = (1, 2, 4, 8)


def _bucket(x: int) -> int:
    """Power-of-two bucket of a size (the tuned choice is reused within it)."""
    return 0 if x <= 0 else 1 << int(math.ceil(math.log2(x)))


def clear() -> None:
    with _lock:
        _table.clear()


def table() -> dict:
    with _lock:
        return dict(_table)


def _time_ms(fn, reps: int = 2) -> float:
    torch = B._torch()
    fn()  # warm-up (also loads the kernel)
    best = float('inf')
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def best_team_warps(tracer, start, qm, atol: float, max_attempts: int, rings: int, sample: int = 4096) -> int:
    """Fastest team size of the plain BEM tracer for this field and particle
    count.  The sample keeps the particle count of the real launch up to
    `sample` particles (so occupancy is the same); larger launches are tuned on
    `sample` particles spread over the batch and reuse the choice per size
    bucket.  `rings`: ring sources summed per field evaluation."""
    torch = B._torch()
    n = start.shape[0]
    key = ('bem_team_warps', torch.cuda.get_device_name(start.device), _bucket(rings), _bucket(n))
    with _lock:
        if key in _table:
            return _table[key]
    if n > sample:
        idx = torch.linspace(0, n - 1, sample, device=start.device).long()
        st, q = start[idx].contiguous(), qm[idx].contiguous()
    else:
        st, q = start, qm
    times = {}
    for tw in TEAM_CANDIDATES:
        times[tw] = _time_ms(lambda tw=tw: tracer.trace_device(st, q, atol=atol, team_warps=tw,
                                                               max_attempts=max_attempts))
    best = min(times, key=times.get)
    with _lock:
        _table[key] = best
        _table[key + ('times_ms',)] = times
    return best


BATCH_BLOCK_CANDIDATES = (1, 2)


def tune_batch_pipeline(pipe, sample: int = 4096) -> dict:
    """Measured launch shape of a traceon_b200.batch.BatchPipeline: the
    solve launch timed with every CTAs-per-SM candidate, the trace timed with
    every team size on `sample` of its particles spread over the batch (at
    most 2,000 attempts each); the fastest of each is set on `pipe` (before
    its graph is captured) and kept per device and size bucket (total tiles,
    rings, particles).  Returns
    {'blocks_per_sm': b, 'team_warps': tw, 'times_ms': {...}}."""
    torch = B._torch()
    bs = pipe.batch
    tiles = int(sum(p[0] * p[0] for p in bs.plan))
    key = ('batch_pipeline', torch.cuda.get_device_name(bs.work.device), _bucket(tiles), _bucket(bs.rings),
           _bucket(pipe.n))
    with _lock:
        hit = _table.get(key)
    if hit is None:
        t_solve = {}
        for b in BATCH_BLOCK_CANDIDATES:
            bs.blocks_per_sm = b
            t_solve[b] = _time_ms(bs.launch, reps=1)
        best_b = min(t_solve, key=t_solve.get)
        bs.blocks_per_sm = best_b
        bs.launch()  # the sources the trace samples read
        m = min(sample, pipe.n)
        idx = torch.linspace(0, pipe.n - 1, m, device=bs.work.device).long()
        t_trace = {}
        for tw in TEAM_CANDIDATES:
            t_trace[tw] = _time_ms(lambda tw=tw: pipe.trace_subset(idx, tw), reps=1)
        best_tw = min(t_trace, key=t_trace.get)
        hit = {'blocks_per_sm': best_b, 'team_warps': best_tw,
               'times_ms': {'solve_by_blocks_per_sm': t_solve, 'trace_sample_by_team_warps': t_trace,
                            'trace_sample_particles': m}}
        with _lock:
            _table[key] = hit
    bs.blocks_per_sm = hit['blocks_per_sm']
    pipe.opts.team_warps = hit['team_warps']
    return hit


LOOKAHEAD_FRACTIONS = (0.0, 1 / 10, 1 / 5, 3 / 10)


def tune_solve_lookahead(A, F) -> dict:
    """Measured lookahead width of the mixed solve (backend.dev_solve_mixed)
    for the size of A (n x n, FP64, on the device) and the right-hand sides F:
    one timed solve per candidate (each fraction of the SMs in
    LOOKAHEAD_FRACTIONS, after one warm-up solve), the fastest set with
    backend.set_solve_lookahead and kept per device and size bucket.  Returns
    {'reserve_sms': r, 'times_ms': {r: ms}}."""
    torch = B._torch()
    n = A.shape[0]
    key = ('solve_lookahead', torch.cuda.get_device_name(A.device), _bucket(n))
    with _lock:
        hit = _table.get(key)
    if hit is None:
        sms = B.num_sms()
        cands = sorted({int(round(f * sms)) for f in LOOKAHEAD_FRACTIONS})
        prev = B.set_solve_lookahead(-1)
        times = {}
        try:
            for r in cands:
                B.set_solve_lookahead(r)
                times[r] = _time_ms(lambda: B.dev_solve_mixed(A, F), reps=1)
        finally:
            B.set_solve_lookahead(prev)
        hit = {'reserve_sms': min(times, key=times.get), 'times_ms': times}
        with _lock:
            _table[key] = hit
    B.set_solve_lookahead(hit['reserve_sms'])
    return hit
