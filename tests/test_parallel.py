"""Replica-parallel tracing logic on CPU: two gloo ranks shard a beam, each
"traces" its shard with a stand-in per-electron function, and the gathered
result equals the single-process result; the job time is the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from traceon_b200.parallel import shard


def test_shard_partition():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            parts = [shard(n, r, world) for r in range(world)]
            assert parts[0].start == 0 and parts[-1].stop == n
            assert all(a.stop == b.start for a, b in zip(parts, parts[1:]))
            sizes = [p.stop - p.start for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _fake_trace(start, qm):
    # stands in for a tracer: a deterministic per-electron result row
    return torch.stack([start[:, 0] * 2 + qm, start[:, 2] - 1.0, start.sum(1)], dim=1)


def _worker(rank, world, port, n, out_path):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from traceon_b200.parallel import trace_sharded, max_over_ranks
        rng = np.random.default_rng(0)
        start = torch.as_tensor(rng.normal(size=(n, 6)))
        qm = torch.as_tensor(rng.normal(size=n))
        full = trace_sharded(_fake_trace, start, qm)
        t = max_over_ranks(1.0 + rank)
        if rank == 0:
            torch.save({'full': full, 'ref': _fake_trace(start, qm), 't': t}, out_path)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


@pytest.mark.parametrize('n', [9, 64])
def test_two_rank_gather(tmp_path, n):
    out = str(tmp_path / 'res.pt')
    mp.spawn(_worker, args=(2, _free_port(), n, out), nprocs=2, join=True)
    r = torch.load(out)
    assert torch.equal(r['full'], r['ref'])
    assert r['t'] == 2.0
