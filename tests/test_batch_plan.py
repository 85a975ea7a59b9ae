"""The batched solve's plan (tb_batch_solve_plan, host code) and its tile
algorithm, on the CPU.  The plan must list every task after the tasks it
waits for, and the few flags each task waits on must imply (through the
waits of those tasks, transitively) every tile and block it reads.  The tile
algorithm itself (left-looking LU without pivoting, diagonal tiles inverted,
block sweeps) is restated in numpy, executed in the plan's task order, and
compared with LAPACK on lens matrices."""
import ctypes as C

import numpy as np
import pytest

from traceon_b200 import backend as B

FILL, FACT, FWD, BWD = range(4)
BT = 64


def plan(sizes):
    n = len(sizes)
    items = (B.TbBatchItem * n)()
    for g, N in enumerate(sizes):
        items[g].N = N
    sz = (B.i64 * 3)()
    nt = B.backend_lib.tb_batch_solve_plan(items, n, None, sz)
    tasks = np.empty(4 * max(nt, 1), dtype=np.int32)
    assert B.backend_lib.tb_batch_solve_plan(items, n, tasks.ctypes.data_as(C.c_void_p), sz) == nt
    return items, tasks.reshape(-1, 4)[:nt], [int(x) for x in sz]


def waits(task, T):
    """The flags the kernel waits on for `task`, as the tasks that set them."""
    ty, g, i, j = (int(x) for x in task)
    if ty == FILL:
        return []
    if ty == FACT:
        s = min(i, j)
        w = [(FILL, g, i, j)]
        if s > 0:
            w += [(FACT, g, i, s - 1), (FACT, g, s - 1, j)]
        if i != j:
            w.append((FACT, g, s, s))
        return w
    if ty == FWD:
        return [(FACT, g, i, i)] + [(FWD, g, k, 0) for k in range(i)]
    return [(FWD, g, T - 1, 0)] + [(BWD, g, k, 0) for k in range(i + 1, T)]


def test_plan_sizes_and_offsets():
    sizes = [130, 64, 1, 500, 65]
    items, tasks, (work, flags, rings) = plan(sizes)
    Ts = [(N + BT - 1) // BT for N in sizes]
    assert [it.T for it in items] == Ts
    assert len(tasks) == sum(2 * T * T + 2 * T for T in Ts)
    assert rings == 16 * sum(sizes)
    # workspace regions: disjoint, in order, 16-byte aligned (even offsets)
    end = 0
    for it in items:
        Np = it.T * BT
        assert it.a_off == end and it.inv_off == it.a_off + Np * Np and it.v_off == it.inv_off + it.T * BT * BT
        end = it.v_off + Np
        assert it.a_off % 2 == 0 and it.inv_off % 2 == 0 and it.v_off % 2 == 0
    assert work == end
    assert items[0].flag_off == 32 and flags == 32 + sum(T * T + 2 * T + 1 for T in Ts)
    assert [it.ring_off for it in items] == list(np.cumsum([0] + [16 * N for N in sizes[:-1]]))
    assert B.backend_lib.tb_batch_solve_plan(items, 0, None, (B.i64 * 3)()) == -1
    bad = (B.TbBatchItem * 1)()
    bad[0].N = 0
    assert B.backend_lib.tb_batch_solve_plan(bad, 1, None, (B.i64 * 3)()) == -1


def test_plan_order_and_sufficient_waits():
    sizes = [300, 64, 1, 700, 129]
    items, tasks, _ = plan(sizes)
    Ts = [it.T for it in items]
    index = {tuple(int(x) for x in t): k for k, t in enumerate(tasks)}
    assert len(index) == len(tasks)
    # every task waits only on tasks listed before it
    for k, t in enumerate(tasks):
        for d in waits(t, Ts[t[1]]):
            assert index[d] < k, (tuple(t), d)
    # the waits imply every input: transitive closure over the wait edges
    closure = {}
    for k, t in enumerate(tasks):
        key = tuple(int(x) for x in t)
        c = set()
        for d in waits(t, Ts[t[1]]):
            c.add(d)
            c |= closure[d]
        closure[key] = c
    for t in tasks:
        ty, g, i, j = (int(x) for x in t)
        T = Ts[g]
        c = closure[(ty, g, i, j)]
        if ty == FACT:
            s = min(i, j)
            need = {(FACT, g, i, k) for k in range(s)} | {(FACT, g, k, j) for k in range(s)}
            if i != j:
                need.add((FACT, g, s, s))
        elif ty == FWD:
            need = {(FACT, g, i, k) for k in range(i + 1)} | {(FWD, g, k, 0) for k in range(i)}
        elif ty == BWD:
            need = {(FACT, g, i, k) for k in range(i, T)} | {(FWD, g, k, 0) for k in range(T)} | \
                   {(BWD, g, k, 0) for k in range(i + 1, T)}
        else:
            need = set()
        assert need <= c, (ty, g, i, j, sorted(need - c)[:4])


def run_plan_numpy(A_list, F_list, tasks):
    """The kernel's tile algorithm in numpy, executed in task order."""
    out = []
    st = []
    for A, F in zip(A_list, F_list):
        N = len(A)
        T = (N + BT - 1) // BT
        Np = T * BT
        P = np.eye(Np)
        st.append({'A': P, 'A0': A, 'F': np.concatenate([F, np.zeros(Np - N)]), 'N': N, 'T': T, 'inv': {},
                   'v': np.zeros(Np)})
    for ty, g, i, j in tasks:
        S = st[g]
        P, T = S['A'], S['T']
        blk = lambda a, b: (slice(a * BT, a * BT + BT), slice(b * BT, b * BT + BT))  # noqa: E731
        if ty == FILL:
            N = S['N']
            sub = np.zeros((BT, BT))
            r0, c0 = i * BT, j * BT
            for a in range(BT):
                for b in range(BT):
                    r, c = r0 + a, c0 + b
                    sub[a, b] = S['A0'][r, c] if (r < N and c < N) else float(r == c)
            P[blk(i, j)] = sub
        elif ty == FACT:
            s = min(i, j)
            C_ = P[blk(i, j)].copy()
            for k in range(s):
                C_ -= P[blk(i, k)] @ P[blk(k, j)]
            if i == j:
                LU = C_.copy()
                for p in range(BT):
                    LU[p + 1:, p] /= LU[p, p]
                    LU[p + 1:, p + 1:] -= np.outer(LU[p + 1:, p], LU[p, p + 1:])
                L = np.tril(LU, -1) + np.eye(BT)
                U = np.triu(LU)
                S['inv'][i] = (np.linalg.inv(L), np.linalg.inv(U))
            elif i > j:
                P[blk(i, j)] = C_ @ S['inv'][s][1]
            else:
                P[blk(i, j)] = S['inv'][s][0] @ C_
        elif ty == FWD:
            r = S['F'][i * BT:(i + 1) * BT].copy()
            for k in range(i):
                r -= P[blk(i, k)] @ S['v'][k * BT:(k + 1) * BT]
            S['v'][i * BT:(i + 1) * BT] = S['inv'][i][0] @ r
        else:
            r = S['v'][i * BT:(i + 1) * BT].copy()
            for k in range(i + 1, T):
                r -= P[blk(i, k)] @ S['v'][k * BT:(k + 1) * BT]
            S['v'][i * BT:(i + 1) * BT] = S['inv'][i][1] @ r
    for S in st:
        out.append(S['v'][:S['N']])
    return out


def test_tile_algorithm_matches_lapack(port):
    """Two small lens matrices (the oracle's fill) solved by the tile
    algorithm in the plan's order: charges within 1e-12 of LAPACK's."""
    from traceon_b200 import geometry as G
    A_list, F_list = [], []
    for seed, n in ((3, (150, 150)), (8, (70, 70))):
        m = G.mirror_lens(seed, n_range=n)
        geo = m.geometry
        vals = geo.voltages_to_values(m.voltages)
        A_list.append(port.matrix(geo.vertices, np.ones(len(geo), np.uint8), vals, threads=4))
        F_list.append(vals)
    _, tasks, _ = plan([len(a) for a in A_list])
    for x, A, F in zip(run_plan_numpy(A_list, F_list, tasks), A_list, F_list):
        x0 = np.linalg.solve(A, F)
        assert np.max(np.abs(x - x0)) / np.max(np.abs(x0)) < 1e-12


def test_hermite_position_at_is_exact_for_cubics():
    """The equal-time endpoint comparison of the batching workload: cubic
    Hermite interpolation of stored states reproduces any cubic-in-time
    trajectory, between states and past the last one."""
    from oracle.oracle import hermite_position_at
    t = np.array([0.0, 0.3, 0.7, 1.2])
    a = np.array([[1.0, -2.0, 0.5], [0.2, 0.1, -0.3], [3.0, 0.0, 1.0], [-1.0, 0.5, 0.25]])  # x(t) = sum a_k t^k

    def x(tt):
        return sum(a[k] * tt**k for k in range(4))

    def v(tt):
        return sum(k * a[k] * tt**(k - 1) for k in range(1, 4))

    states = np.array([np.concatenate([x(tt), v(tt)]) for tt in t])
    for tt in (0.0, 0.1, 0.5, 1.0, 1.2, 1.35):
        assert np.allclose(hermite_position_at(t, states, tt), x(tt), rtol=0, atol=1e-12)
