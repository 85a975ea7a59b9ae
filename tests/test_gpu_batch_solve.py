"""The batching workload's single-launch solve and its CUDA-graph pipeline:
tb_batch_solve fills, factors and solves mirror lenses of uneven N (ragged
last tiles, a geometry smaller than one tile) in one persistent launch,
giving the oracle's LAPACK charges; its packed sources equal
tb_pack_sources of those charges; a launch whose bounded waits run out
leaves status -1 and the next launch recovers; the fill -> solve -> trace
pipeline replays as a CUDA graph with the eager run's endpoints, which equal
the one-geometry tracer's and the oracle's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _excitation(m):
    from traceon_b200.excitation import Excitation, Mesh
    geo = m.geometry
    exc = Excitation(Mesh.from_geometry(geo))
    exc.add_voltage(**{n: float(v) for n, v in zip(geo.names, m.voltages)})
    return exc


@pytest.fixture(scope='module')
def lenses():
    from traceon_b200 import geometry as G
    return [G.mirror_lens(0, n_range=(40, 40))] + [G.mirror_lens(s, n_range=(65, 900)) for s in range(1, 6)]


def test_batch_solve_vs_oracle(cuda, port, lenses):
    import torch
    from traceon_b200.batch import BatchSolve
    bs = BatchSolve([_excitation(m) for m in lenses])
    assert min(len(s.vertices) for s in bs.solvers) < 64
    q = bs.solve()
    assert (bs.status.cpu().numpy() == 0).all()
    for m, got in zip(lenses, q):
        geo = m.geometry
        vals = geo.voltages_to_values(m.voltages)
        A = port.matrix(geo.vertices, np.ones(len(geo), np.uint8), vals, threads=8)
        x = np.linalg.solve(A, vals)
        assert np.max(np.abs(got - x)) / np.max(np.abs(x)) < 1e-10
    for g, s_ in enumerate(bs.solvers):
        _, _, _, jac, pos = s_.device()
        N = len(s_.vertices)
        want = cuda.dev_pack_sources(bs.charges[g], jac, pos)
        o = bs.plan[g][5]
        got = bs.sources[:, o:o + 16 * N]
        assert torch.equal(got, want)
    # a second launch gives the same charges bit for bit
    first = [c.clone() for c in bs.charges]
    bs.solve()
    assert all(torch.equal(a, b) for a, b in zip(first, bs.charges))


def test_batch_solve_wait_timeout(cuda, lenses):
    """Waits cut to one cycle: the launch gives up (status -1 for unfinished
    geometries, check() raises TB_TIMEOUT) without faulting; with the default
    bound restored the next launch on the same context solves."""
    import torch
    from traceon_b200.batch import BatchSolve
    bs = BatchSolve([_excitation(m) for m in lenses[:4]])
    old = cuda.set_wait_limit(1)
    try:
        bs.launch()
        torch.cuda.synchronize()
    finally:
        cuda.set_wait_limit(old)
    st = bs.status.cpu().numpy()
    assert (st == -1).any()
    with pytest.raises(cuda.BackendError):
        bs.check()
    bs.solve()
    assert (bs.status.cpu().numpy() == 0).all()


def test_batch_pipeline_graph(cuda, port, lenses):
    import torch
    from traceon_b200 import geometry as G
    from traceon_b200.batch import BatchPipeline
    from traceon_b200.tracing import Tracer
    from oracle.oracle import EM
    ms = lenses[1:4]
    starts = [G.mirror_beam(40, 30 + k, m.z_start) for k, m in enumerate(ms)]
    p = BatchPipeline([_excitation(m) for m in ms], [s[0] for s in starts], [s[1] for s in starts],
                      [m.bounds for m in ms], atol=1e-9, team_warps=2)
    p.enqueue()
    eager = [tuple(np.copy(a) for a in r) for r in p.results()]
    p.capture()
    for a in (p.final, p.status, p.counters):
        a.fill_(0)
    p.replay()
    torch.cuda.synchronize()
    for r0, r1 in zip(eager, p.results()):
        for a, b in zip(r0, r1):
            assert np.array_equal(a, b)
    fields = p.batch.fields()
    for k, (m, (pos, vel)) in enumerate(zip(ms, starts)):
        final, status, counters = eager[k]
        assert (status == 0).all()
        # the one-geometry tracer through the same charges, same team size
        tr = Tracer(fields[k], m.bounds)
        n = len(pos)
        st = cuda.to_dev(np.concatenate([pos, vel], 1), torch.float64)
        qm = p.qm[:n].clone()
        res = tr.trace_device(st, qm, atol=1e-9, team_warps=2)
        assert np.array_equal(res.final.cpu().numpy(), final)
    # the oracle (its own fill and LAPACK charges) on a few particles of the first lens
    m, (pos, vel) = ms[0], starts[0]
    geo = m.geometry
    vals = geo.voltages_to_values(m.voltages)
    A = port.matrix(geo.vertices, np.ones(len(geo), np.uint8), vals, threads=8)
    q = np.linalg.solve(A, vals)
    jac, pos_r = port.fill_jacobian_buffer_radial(geo.vertices)
    final = eager[0][0]
    for i in range(8):
        t, s = port.trace_bem(pos[i], vel[i], EM, q, jac, pos_r, m.bounds, 1e-9)
        assert abs(t[-1] - final[i, 0]) <= 1e-9 * abs(t[-1])
        assert np.max(np.abs(s[-1, :3] - final[i, 1:4])) < 1e-9
