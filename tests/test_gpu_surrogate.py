"""The learned surrogate: BF16 / FP32-accumulate kernels against the float64
NumPy oracle (oracle/mlp_oracle.py), and the trained surrogate's traces
against the exact BEM trace of the CPU oracle -- including what the network
gains over the axial series alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_gemm_layouts(cuda):
    """tb_mlp_gemm in all four operand layouts, incl. split-K, vs float64."""
    import torch
    from traceon_b200 import surrogate as SG
    from oracle.mlp_oracle import bf16
    rng = np.random.default_rng(0)
    for (M, N, K) in ((70, 130, 48), (128, 16, 4096), (256, 128, 128)):
        A = bf16(rng.normal(size=(M, K)))
        Bm = bf16(rng.normal(size=(N, K)))
        ref = A @ Bm.T
        for at in (0, 1):
            for bt in (0, 1):
                a = torch.as_tensor(A.T.copy() if at else A, dtype=torch.float32).to('cuda', torch.bfloat16)
                b = torch.as_tensor(Bm.T.copy() if bt else Bm, dtype=torch.float32).to('cuda', torch.bfloat16)
                Cm = torch.zeros((M, N), dtype=torch.float32, device='cuda')
                SG._call('tb_mlp_gemm', a.data_ptr(), M if at else K, at, b.data_ptr(), N if bt else K, bt,
                         Cm.data_ptr(), N, M, N, K, 0, SG._s())
                assert _rel(Cm.cpu().numpy(), ref) < 1e-6, (M, N, K, at, bt)


def test_forward_and_gradients_vs_oracle(cuda):
    import torch
    from traceon_b200 import surrogate as SG
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(1)
    mlp = SG.MLP(seed=3)
    M, n_out = 96, 9
    X = rng.uniform(-1, 1, (M, 16))
    T = rng.normal(size=(M, n_out)).astype(np.float32)
    Xt = torch.as_tensor(X, dtype=torch.float32).to('cuda', torch.bfloat16)
    out = mlp.forward(Xt).cpu().numpy()
    params = mlp.p.cpu().numpy().astype(np.float64)
    out_ref, _, _ = MO.forward(params, X)
    assert _rel(out, out_ref) < 2e-3
    loss = float(mlp.loss_and_grad(Xt, torch.as_tensor(T, device='cuda'), n_out))
    loss_ref, g_ref = MO.loss_and_grad(params, X, T.astype(np.float64), n_out)
    assert abs(loss - loss_ref) / loss_ref < 2e-3
    g = mlp.g.cpu().numpy()
    off, _ = MO.offsets()
    for name, (o, n) in off.items():
        assert _rel(g[o:o + n], g_ref[o:o + n]) < 2e-2, name


def test_adam_reduces_loss(cuda):
    import torch
    from traceon_b200 import surrogate as SG
    rng = np.random.default_rng(2)
    mlp = SG.MLP(seed=1)
    X = torch.as_tensor(rng.uniform(-1, 1, (4096, 16)), dtype=torch.float32).to('cuda', torch.bfloat16)
    T = torch.as_tensor(np.sin(3 * rng.uniform(-1, 1, (4096, 3))), dtype=torch.float32, device='cuda')
    Xf = X.float()
    T = torch.stack([torch.sin(2 * Xf[:, 0]) * Xf[:, 1], Xf[:, 2] ** 2, torch.cos(Xf[:, 3])], 1).contiguous()
    l0 = float(mlp.loss_and_grad(X, T, 3))
    for _ in range(300):
        mlp.loss_and_grad(X, T, 3)
        mlp.adam(3e-3)
    l1 = float(mlp.loss_and_grad(X, T, 3))
    assert l1 < 0.05 * l0


@pytest.fixture(scope='module')
def trained():
    from traceon_b200 import geometry as G
    from traceon_b200.surrogate import SurrogateTrainer
    geo = G.einzel_lens(300)
    tr = SurrogateTrainer(geo)
    model, info = tr.train(n_samples=1 << 20, steps=8000, batch=8192, seed=0)
    return geo, tr, model, info


def _fields(trained, volts, engine='warp'):
    from traceon_b200.surrogate import FieldSurrogate, SurrogateModel
    geo, tr, model, info = trained
    fs = FieldSurrogate(model, tr.fields, tr.z, tr.tabs, volts, geo.segments, engine=engine)
    axial_only = FieldSurrogate(model, tr.fields, tr.z, tr.tabs, volts, geo.segments)
    axial_only.model = SurrogateModel(model.n_el, model.r_max, model.z_lo, model.z_hi, model.scale * 0,
                                      model.env_power, params=model.mlp.p.cpu().numpy())
    return fs, axial_only


def test_network_gain_on_field(cuda, trained):
    """Held-out points off the axis: the learned correction makes the field
    far closer to the exact BEM field than the axial series alone."""
    import torch
    from traceon_b200 import backend as B
    fs, axial_only = _fields(trained, np.array([0.0, 1500.0, 0.0]))
    geo, tr, model, info = trained
    assert info['holdout_mse'] < 2e-3
    rng = np.random.default_rng(4)
    pts = np.stack([rng.uniform(0.3e-3, 0.8e-3, 2000), np.zeros(2000), rng.uniform(-9.5e-3, 9.5e-3, 2000)], 1)
    E_sur, used = fs.kernel_field_at_points(pts)
    E_ax, _ = axial_only.kernel_field_at_points(pts)
    _, E_bem = B.dev_field_points(B.to_dev(pts, torch.float64), fs.sources)
    E_bem = E_bem.cpu().numpy()
    ok = used == 0
    err_sur = np.abs(E_sur - E_bem)[ok].max()
    err_ax = np.abs(E_ax - E_bem)[ok].max()
    assert err_sur < err_ax / 20
    # The kernel's field matches the batched host evaluation of the same model.
    # They differ in the FP32 accumulation order inside the network, which can
    # flip BF16 roundings of hidden activations: compare against the size of
    # the learned correction itself.
    E_host = fs.field_at_points(pts)
    assert np.abs(E_host - E_sur)[ok].max() < 0.05 * np.abs(E_sur - E_ax)[ok].max()


def _endpoint_errors(port, field, p0, v0):
    import torch
    from traceon_b200 import geometry as G
    from oracle.oracle import EM, hermite_plane_crossing
    n = len(p0)
    start = torch.as_tensor(np.concatenate([p0, v0], 1), device='cuda')
    qm = torch.full((n,), EM, device='cuda', dtype=torch.float64)
    res = field.trace_device(start, qm, G.LENS_BOUNDS, 1e-10, plane_z=G.LENS_EXIT_Z)
    assert (res.status.cpu().numpy() == 0).all()
    plane = res.plane.cpu().numpy()
    q = field.bem.electrostatic_point_charges
    err = []
    for i in range(n):
        t, s = port.trace_bem(p0[i], v0[i], EM, q.charges, q.jacobians, q.positions, G.LENS_BOUNDS, 1e-10)
        h = hermite_plane_crossing(t, s, G.LENS_EXIT_Z)
        err.append(np.abs(plane[i, 1:3] - h[:2]).max())
    return np.array(err), res.counters.cpu().numpy()


def test_surrogate_traces_vs_bem_oracle(cuda, port, trained):
    """The surrogate workload's beam (1 keV +-5 %, +-20 mrad, r0 <= 0.2 mm):
    exit-plane positions within 1 nm of the exact FP64 BEM trace of the
    oracle; and on a wider beam (r0 <= 0.4 mm) the network lowers the error of
    the axial series it corrects."""
    from traceon_b200 import geometry as G
    fs, axial_only = _fields(trained, np.array([0.0, 1500.0, 0.0]))
    p0, v0 = G.surrogate_beam(16, 21)
    err, counters = _endpoint_errors(port, fs, p0, v0)
    assert err.max() < 1e-9
    assert counters[:, 2].sum() == 0  # no BEM fallback needed on this beam
    p0, v0 = G.electron_beam(16, 22, r_max=0.4e-3, angle_max=20e-3)
    err_s, _ = _endpoint_errors(port, fs, p0, v0)
    err_a, _ = _endpoint_errors(port, axial_only, p0, v0)
    assert err_s.max() < err_a.max()


def test_surrogate_fallback_near_electrodes(cuda, trained):
    """Within 50 um of an electrode the tracer's field is the exact BEM field."""
    import torch
    from traceon_b200 import backend as B
    fs, _ = _fields(trained, np.array([0.0, 1500.0, 0.0]))
    pts = np.array([[0.97e-3, 0.0, -3e-3], [0.98e-3, 0.0, 0.0], [0.5e-3, 0.0, -11.8e-3]])
    E, used = fs.kernel_field_at_points(pts)
    assert used.tolist() == [1, 1, 1]
    _, E_bem = B.dev_field_points(B.to_dev(pts, torch.float64), fs.sources)
    E_bem = E_bem.cpu().numpy()
    assert np.all(np.linalg.norm(E - E_bem, axis=1) < 1e-12 * np.linalg.norm(E_bem, axis=1))


def test_tc_engine_matches_warp_engine(cuda, trained):
    """The tcgen05 engine (128-particle groups, accumulators in tensor
    memory) evaluates the same network as the warp-level mma.sync engine:
    the same fallback decisions, and fields that differ only by FP32
    accumulation order (which can flip BF16 roundings of hidden activations),
    far below the learned correction itself.  At the fallback points the
    exact BEM sums agree to rounding: the tcgen05 engine sums each such point
    with its whole 128-thread group, the warp engine with one thread.  1,000
    points: not a multiple of the 128-row tile."""
    volts = np.array([0.0, 1500.0, 0.0])
    fs_w, axial_only = _fields(trained, volts, 'warp')
    fs_t, _ = _fields(trained, volts, 'tc')
    rng = np.random.default_rng(5)
    n = 1000
    pts = np.stack([rng.uniform(0.0, 0.9e-3, n), rng.uniform(-0.1e-3, 0.1e-3, n), rng.uniform(-9.5e-3, 9.5e-3, n)], 1)
    pts[:10, 0] = 0.985e-3  # near the tube wall: exact BEM fallback
    E_w, used_w = fs_w.kernel_field_at_points(pts)
    E_t, used_t = fs_t.kernel_field_at_points(pts)
    E_ax, _ = axial_only.kernel_field_at_points(pts)
    assert (used_t >= 0).all()  # no engine timeout
    assert (used_t == used_w).all() and used_t[:10].all()
    ok = used_w == 0
    corr = np.abs(E_w - E_ax)[ok].max()
    assert corr > 0
    assert np.abs(E_t - E_w)[ok].max() < 0.02 * corr
    assert np.abs(E_t[~ok] - E_w[~ok]).max() <= 1e-12 * np.abs(E_w[~ok]).max()


def test_tc_engine_traces_vs_bem_oracle(cuda, port, trained):
    """Tracing through the tcgen05 engine: 300 electrons (2 full groups and a
    partial one), all exit, sampled endpoints within 1 nm of the exact FP64
    BEM trace of the oracle and within 0.1 nm of the warp engine's."""
    import torch
    from traceon_b200 import geometry as G
    from oracle.oracle import EM
    volts = np.array([0.0, 1500.0, 0.0])
    fs_t, _ = _fields(trained, volts, 'tc')
    fs_w, _ = _fields(trained, volts, 'warp')
    p0, v0 = G.surrogate_beam(300, 23)
    start = torch.as_tensor(np.concatenate([p0, v0], 1), device='cuda')
    qm = torch.full((300,), EM, device='cuda', dtype=torch.float64)
    r_t = fs_t.trace_device(start, qm, G.LENS_BOUNDS, 1e-10, plane_z=G.LENS_EXIT_Z)
    r_w = fs_w.trace_device(start, qm, G.LENS_BOUNDS, 1e-10, plane_z=G.LENS_EXIT_Z)
    assert (r_t.status.cpu().numpy() == 0).all()
    d = np.abs(r_t.plane.cpu().numpy()[:, 1:3] - r_w.plane.cpu().numpy()[:, 1:3]).max()
    assert d < 1e-10
    err, _ = _endpoint_errors(port, fs_t, p0[:12], v0[:12])
    assert err.max() < 1e-9


def test_trace_session_graph_replays(cuda, trained):
    """TraceSession: pinned staging + the whole step captured as a CUDA graph.
    Two batches through one session give exactly the endpoints of the eager
    public call on the same inputs (each particle's path depends only on its
    own state), and the buffers are reused between runs."""
    from traceon_b200 import geometry as G
    fs, _ = _fields(trained, np.array([0.0, 1500.0, 0.0]))
    n = 700
    sess = fs.trace_session(n, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
    for seed in (31, 32):
        p0, v0 = G.surrogate_beam(n, seed)
        plane, final, status, counters = fs.trace_endpoints(p0, v0, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
        sp, sf, ss, sc = (a.copy() for a in sess.run(p0, v0))
        assert (ss == 0).all() and np.array_equal(ss, status)
        assert np.array_equal(sp, plane) and np.array_equal(sf, final) and np.array_equal(sc, counters)
    assert sess.h2d_bytes == n * 48 and sess.d2h_bytes == n * (112 + 4 + 24)


def test_trace_session_pipelined_batches(cuda, trained):
    """run_many: five batches of different beams with two buffer sets in
    flight give, batch by batch, exactly the endpoints of run() on the same
    inputs; an empty list returns an empty list."""
    from traceon_b200 import geometry as G
    fs, _ = _fields(trained, np.array([0.0, 1500.0, 0.0]))
    n = 500
    sess = fs.trace_session(n, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
    beams = [G.surrogate_beam(n, seed) for seed in range(50, 55)]
    want = [tuple(a.copy() for a in sess.run(p0, v0)) for p0, v0 in beams]
    got = sess.run_many(beams)
    assert len(got) == len(beams)
    for g, w in zip(got, want):
        assert (w[2] == 0).all()
        for a, b in zip(g, w):
            assert np.array_equal(a, b)
    assert sess.run_many([]) == []
    # and once more, reusing both buffer sets
    again = sess.run_many(beams[:3])
    for g, w in zip(again, want[:3]):
        assert np.array_equal(g[0], w[0])


def test_surrogate_tracer_edge_cases(cuda, trained):
    """Empty batch; particles that start outside the (inclusive) bounds end at
    once with no step; an attempt cap of 1 ends every particle with
    TRACE_MAX_ATTEMPTS after exactly one attempt (the reference would loop
    until the particle leaves the bounds).  Both engines."""
    import torch
    from traceon_b200 import geometry as G
    from oracle.oracle import EM
    for engine in ('tc', 'warp'):
        fs, _ = _fields(trained, np.array([0.0, 1500.0, 0.0]), engine)
        empty = torch.empty((0, 6), dtype=torch.float64, device='cuda')
        r = fs.trace_device(empty, torch.empty(0, dtype=torch.float64, device='cuda'), G.LENS_BOUNDS, 1e-10,
                            plane_z=G.LENS_EXIT_Z)
        assert r.status.numel() == 0
        p0, v0 = G.surrogate_beam(130, 41)
        p0[:5, 2] = -10.5e-3  # below z_min = -10 mm
        plane, final, status, counters = fs.trace_endpoints(p0, v0, G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10)
        assert (status == cuda.TRACE_EXITED).all()
        assert (counters[:5, :2] == 0).all() and np.isnan(plane[:5, 1:]).all()
        assert np.array_equal(final[:5, 1:4], p0[:5])
        assert (counters[5:, 0] > 10).all()
        plane, final, status, counters = fs.trace_endpoints(p0[5:], v0[5:], G.LENS_BOUNDS, G.LENS_EXIT_Z, atol=1e-10,
                                                            max_attempts=1)
        assert (status == cuda.TRACE_MAX_ATTEMPTS).all()
        assert (counters[:, 1] == 1).all()
