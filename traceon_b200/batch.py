"""The batching workload's device pipeline: many geometries of uneven N
filled, factored and solved in ONE persistent launch (tb_batch_solve), then
all their particles traced through the direct BEM field in one more
(tb_trace_rk45_geometries), the two captured as one CUDA graph.

The reference fills and solves one excitation at a time
(traceon/solver.py:160-232, 402-431) and traces one field at a time
(traceon/tracing.py:115-245); BatchSolve's fields equal solve_direct's for
each excitation (charges within 1e-10), and BatchPipeline's endpoints equal
Tracer.trace_endpoints through each field.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
from scipy.constants import e, m_e

from . import backend as B
from .solver import ElectrostaticSolverRadial

TB_OK, TB_SINGULAR = 0, 5


class BatchSolve:
    """The electrostatic charges of many excitations (geometries of uneven N)
    from one persistent launch that fills every matrix, factors it without
    pivoting in 64 x 64 tiles, solves it and packs the charges into the
    tracer's source rings.  Geometries the launch marks singular are solved
    again with the pivoted FP64 LU.  blocks_per_sm: CTAs per SM (0 = as many
    as fit; the autotuner may pick fewer)."""

    def __init__(self, excitations, blocks_per_sm: int = 0):
        torch = B._torch()
        self.solvers = [ElectrostaticSolverRadial(x) for x in excitations]
        if not self.solvers:
            raise ValueError('no excitations')
        n = len(self.solvers)
        self.blocks_per_sm = int(blocks_per_sm)
        items = (B.TbBatchItem * n)()
        self._keep = []
        self.charges = []
        for g, s_ in enumerate(self.solvers):
            v, t, val, _, _ = s_.device()
            F = s_.get_right_hand_side_device()
            q = torch.empty(len(s_.vertices), dtype=torch.float64, device=v.device)
            self._keep += [v, t, val, F]
            self.charges.append(q)
            items[g] = B.TbBatchItem(v.data_ptr(), t.data_ptr(), val.data_ptr(), F.data_ptr(), q.data_ptr(),
                                     len(s_.vertices), 0, 0, 0, 0, 0, 0)
        sizes = (B.i64 * 3)()
        n_tasks = B.backend_lib.tb_batch_solve_plan(items, n, None, sizes)
        if n_tasks <= 0:
            raise B.BackendError('tb_batch_solve_plan: bad geometry sizes')
        tasks = np.empty(4 * n_tasks, dtype=np.int32)
        if B.backend_lib.tb_batch_solve_plan(items, n, tasks.ctypes.data_as(C.c_void_p), sizes) != n_tasks:
            raise B.BackendError('tb_batch_solve_plan: inconsistent task count')
        dev = self._keep[0].device
        self.n_tasks = int(n_tasks)
        self.plan = [(int(it.T), int(it.a_off), int(it.inv_off), int(it.v_off), int(it.flag_off), int(it.ring_off))
                     for it in items]
        self.tasks_host = tasks.reshape(-1, 4)
        self.items_dev = torch.frombuffer(bytearray(bytes(items)), dtype=torch.uint8).to(dev)
        self.tasks_dev = torch.from_numpy(tasks).to(dev)
        self.work = torch.empty(int(sizes[0]), dtype=torch.float64, device=dev)
        self.flags = torch.empty(int(sizes[1]), dtype=torch.int32, device=dev)
        self.rings = int(sizes[2])
        self.sources = torch.empty((3, self.rings), dtype=torch.float64, device=dev)
        self.status = torch.empty(n, dtype=torch.int32, device=dev)
        self.ring_offsets = torch.as_tensor([p[5] for p in self.plan] + [self.rings], dtype=torch.int64, device=dev)

    def __len__(self):
        return len(self.solvers)

    def launch(self):
        """Enqueues the fill + factor + solve + pack launch on the current
        stream (capturable into a CUDA graph)."""
        B._call('tb_batch_solve', self.items_dev.data_ptr(), len(self), self.tasks_dev.data_ptr(), self.n_tasks,
                self.work.data_ptr(), self.flags.data_ptr(), self.flags.numel(), self.sources.data_ptr(),
                self.rings, self.status.data_ptr(), self.blocks_per_sm, B._stream())

    def check(self):
        """After a launch: solves the geometries marked singular again with the
        pivoted FP64 LU (and repacks their sources); raises TB_TIMEOUT if the
        launch gave up on a bounded wait.  Returns the statuses."""
        st = self.status.cpu().numpy()
        if (st == -1).any():
            raise B.BackendError(f'tb_batch_solve: a bounded wait ran out (status {B.TB_TIMEOUT})')
        for g in np.nonzero(st == TB_SINGULAR)[0]:
            s_ = self.solvers[g]
            f = s_.solve_matrix(method='lu')[0]
            q = B.to_dev(f.electrostatic_point_charges.charges, B._torch().float64)
            self.charges[g].copy_(q)
            _, _, _, jac, pos = s_.device()
            o = self.plan[g][5]
            N = len(s_.vertices)
            src = B._torch().empty((3, 16 * N), dtype=B._torch().float64, device=q.device)
            B._call('tb_pack_sources', q.data_ptr(), jac.data_ptr(), pos.data_ptr(), src.data_ptr(), N, B._stream())
            self.sources[:, o:o + 16 * N].copy_(src)
        return st

    def solve(self):
        """Launch, check, and return the charges (host arrays)."""
        self.launch()
        self.check()
        return [q.cpu().numpy() for q in self.charges]

    def fields(self):
        """FieldRadialBEM of every geometry from the last launch's charges."""
        from .field import EffectivePointCharges
        out = []
        for s_, q in zip(self.solvers, self.charges):
            jac, pos = s_.jacobians_and_positions()
            out.append(s_.charges_to_field(EffectivePointCharges(q.cpu().numpy(), jac, pos)))
        return out


class BatchPipeline:
    """fill -> factor -> solve -> pack (tb_batch_solve) -> trace
    (tb_trace_rk45_geometries) for many geometries, enqueued together and,
    with capture(), recorded as one CUDA graph that replay() re-runs.
    positions[g], velocities[g]: (n_g, 3) start states of geometry g's
    particles; bounds[g]: its (3, 2) box.  Particles' end states (t, x, y, z,
    vx, vy, vz), statuses and (accepted, attempted) step counts are in
    `final`, `status`, `counters` after a run, in the concatenated order."""

    def __init__(self, excitations, positions, velocities, bounds, atol=1e-8, max_attempts=20000, mass=m_e,
                 charge=-e, team_warps=0, blocks_per_sm=0):
        torch = B._torch()
        self.batch = BatchSolve(excitations, blocks_per_sm=blocks_per_sm)
        G = len(self.batch)
        if len(positions) != G or len(velocities) != G or len(bounds) != G:
            raise ValueError('one entry of positions, velocities and bounds per excitation')
        self.counts = [len(np.atleast_2d(p)) for p in positions]
        pos = np.concatenate([np.atleast_2d(np.asarray(p, dtype=np.float64)) for p in positions])
        vel = np.concatenate([np.atleast_2d(np.asarray(v, dtype=np.float64)) for v in velocities])
        self.n = n = len(pos)
        dev = self.batch.work.device
        self.start = B.to_dev(np.concatenate([pos, vel], axis=1), torch.float64)
        self.qm = torch.full((n,), float(charge) / float(mass), dtype=torch.float64, device=dev)
        self.geom = B.to_dev(np.repeat(np.arange(G, dtype=np.int32), self.counts), torch.int32)
        self.gbounds = B.to_dev(np.stack([np.asarray(b, dtype=np.float64).reshape(6) for b in bounds]), torch.float64)
        self.status = torch.empty(n, dtype=torch.int32, device=dev)
        self.final = torch.empty((n, 7), dtype=torch.float64, device=dev)
        self.counters = torch.empty((n, 2), dtype=torch.int64, device=dev)
        self.work = torch.empty(1, dtype=torch.int32, device=dev)
        self.field = B.TbField(self.batch.sources.data_ptr(), self.batch.rings, None, 0, None, 0, None, None, None,
                               None, 0)
        o = B.TbTraceOpts()
        b0 = self.gbounds[0].cpu().numpy()
        for i in range(6):
            o.bounds[i] = float(b0[i])
        o.atol, o.plane_z, o.record_plane = float(atol), 0.0, 0
        o.max_attempts, o.max_rows, o.team_warps = int(max_attempts), 0, int(team_warps)
        self.opts = o
        self.graph = None

    def enqueue(self):
        """The two launches on the current stream."""
        self.batch.launch()
        B._call('tb_trace_rk45_geometries', self.start.data_ptr(), None, self.qm.data_ptr(), self.geom.data_ptr(),
                self.n, C.byref(self.field), self.batch.ring_offsets.data_ptr(), len(self.batch),
                self.gbounds.data_ptr(), C.byref(self.opts), None, None, self.status.data_ptr(),
                self.final.data_ptr(), None, self.counters.data_ptr(), self.work.data_ptr(), B._stream())

    def trace_subset(self, idx, team_warps: int, max_attempts: int = 2000):
        """The trace launch on the particles idx (a device index tensor) with
        the given team size and attempt cap, into scratch outputs: the
        autotuner's sample (the cap keeps the few trapped particles from
        dominating its time)."""
        torch = B._torch()
        idx = idx.to(self.start.device)
        st, qm, geom = self.start[idx].contiguous(), self.qm[idx].contiguous(), self.geom[idx].contiguous()
        m = st.shape[0]
        status = torch.empty(m, dtype=torch.int32, device=st.device)
        final = torch.empty((m, 7), dtype=torch.float64, device=st.device)
        counters = torch.empty((m, 2), dtype=torch.int64, device=st.device)
        work = torch.empty(1, dtype=torch.int32, device=st.device)
        o = B.TbTraceOpts.from_buffer_copy(self.opts)
        o.team_warps = int(team_warps)
        o.max_attempts = min(int(o.max_attempts), int(max_attempts))
        B._call('tb_trace_rk45_geometries', st.data_ptr(), None, qm.data_ptr(), geom.data_ptr(), m,
                C.byref(self.field), self.batch.ring_offsets.data_ptr(), len(self.batch), self.gbounds.data_ptr(),
                C.byref(o), None, None, status.data_ptr(), final.data_ptr(), None, counters.data_ptr(),
                work.data_ptr(), B._stream())
        return final

    def capture(self):
        """Records enqueue() as a CUDA graph (after one eager run on the
        capture stream, which sets the kernels' attributes)."""
        torch = B._torch()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.enqueue()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode='thread_local'):
            self.enqueue()
        torch.cuda.synchronize()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.enqueue()
        else:
            self.graph.replay()

    def results(self):
        """Per geometry (final (n_g, 7), status (n_g,), counters (n_g, 2)),
        after checking the solve's statuses."""
        st = self.batch.status.cpu().numpy()
        if (st != TB_OK).any():
            raise B.BackendError(f'tb_batch_solve statuses {st.tolist()}: singular or timed-out geometries need '
                                 'BatchSolve.check() before tracing')
        cuts = np.cumsum(self.counts)[:-1]
        out = [a.cpu().numpy() for a in (self.final, self.status, self.counters)]
        return [tuple(x) for x in zip(*(np.split(a, cuts) for a in out))]
