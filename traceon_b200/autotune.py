"""Measured choice of launch parameters.

The tracers' launch shapes depend on the workload: the plain BEM tracer
splits every field sum over a team of 1, 2, 4 or 8 warps, and the best team
size depends on how many particles there are per SM and how many rings each
field evaluation sums.  Instead of a fixed rule, `best_team_warps` times
every candidate on a bounded sample of the actual workload (CUDA events on
the launching stream) and keeps the fastest in a process-wide table keyed by
device and problem size, guarded by a lock (entry points may be called from
several host threads).

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
