"""The multi-GPU host logic on CPU (gpurify_b200/multigpu.py): the window
partition and the column blocks, and, with two gloo ranks (world size 2 on
127.0.0.1), one window's conductor columns spread over the ranks and
all-gathered, and a batch of windows spread over the ranks and gathered.
The column / window solver on CPU is the oracle's dense LU (test
infrastructure standing in for each rank's GPU solve); the gathered results
must equal the single-process results exactly."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gpurify_b200 import multigpu


def test_partition_windows_covers_once_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.lognormal(10, 1.2, size=37)
    for world in (1, 2, 3, 8):
        parts = multigpu.partition_windows(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # largest-first greedy: no rank exceeds the lightest by more than one window
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert parts == multigpu.partition_windows(list(costs), world)  # deterministic
    assert multigpu.partition_windows([], 4) == [[], [], [], []]


def test_column_blocks_cover_once():
    for n in (0, 1, 5, 64, 511):
        for world in (1, 2, 3, 8):
            blocks = multigpu.column_blocks(n, world)
            assert len(blocks) == world
            assert sum(c for _, c in blocks) == n
            b = 0
            for b0, c in blocks:
                assert b0 == b and c >= 0
                b += c
            assert max(c for _, c in blocks) - min(c for _, c in blocks) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _small_problem(k):
    """Conductor plates over a ground plate (k + 2 conductors)."""
    import oracle

    vs, cs = [], []
    for i in range(k + 1):
        v, c = oracle.plate(1.5e-6 * i, 0.0, 0.4e-6 + 0.1e-6 * (i % 2), 1.0e-6, 1.0e-6, 5, 5, i)
        vs.append(v)
        cs.append(c)
    g, cg = oracle.plate(1.5e-6 * k / 2, 0.0, 0.0, 2.0e-6 * (k + 2), 3.0e-6, 8, 4, k + 1)
    return np.vstack(vs + [g]), np.concatenate(cs + [cg]), k + 2


def _skip_ground_reference(D):
    R = D.shape[0] - 1
    C = D.copy()
    C[:R, R] = D[R, :R]
    C[R, R] = np.nan
    return C


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import oracle

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        verts, cond, nc = _small_problem(4)
        D = oracle.cap_dense(verts, cond, nc)
        calls = []

        def column_solver(b, c):
            calls.append((b, c))
            return oracle.cap_dense(verts, cond, nc)[:, b : b + c]

        C = multigpu.solve_window_sharded(nc, dist, skip_ground_rhs=True, column_solver=column_solver)
        Cfull = multigpu.solve_window_sharded(nc, dist, skip_ground_rhs=False, column_solver=column_solver)
        # panels in several media: the matrix is not symmetric, the skipped column stays NaN
        eps = np.where(cond % 2 == 0, 3.9, 2.5)
        Deps = oracle.cap_dense_eps(verts, cond, nc, eps)
        Ceps = multigpu.solve_window_sharded(nc, dist, skip_ground_rhs=True, symmetric=False,
                                             column_solver=lambda b, c: Deps[:, b : b + c])
        probs = [_small_problem(k) for k in (1, 3, 2, 5, 1)]
        costs = [len(v) * (n - 1) for v, _, n in probs]

        def window_solver(idx):
            return [oracle.cap_dense(*probs[i]) for i in idx]

        W = multigpu.solve_windows_partitioned(costs, dist, window_solver)
        dist.barrier()
        q.put((rank, calls, C, Cfull, D, W, [oracle.cap_dense(*p) for p in probs], Ceps, Deps))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_columns_and_windows():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, calls, C, Cfull, D, W, Wref, Ceps, Deps in res:
        R = D.shape[0] - 1
        np.testing.assert_array_equal(Ceps[:, :R], Deps[:, :R])
        assert np.all(np.isnan(Ceps[:, R]))
        # rank r solved only its own block: nets split 3 + 2, all conductors 3 + 3
        assert calls == ([(0, 3), (0, 3)] if rank == 0 else [(3, 2), (3, 3)])
        np.testing.assert_array_equal(C[:, :R], D[:, :R])
        np.testing.assert_array_equal(np.isnan(C), np.isnan(_skip_ground_reference(D)))
        np.testing.assert_array_equal(C[:R, R], D[R, :R])
        np.testing.assert_array_equal(Cfull, D)
        assert len(W) == len(Wref)
        for a, b in zip(W, Wref):
            np.testing.assert_array_equal(a, b)
