"""The bench's multi-rank path on CPU: two gloo ranks (world size 2, on
127.0.0.1), each with its own seeded window (weak scaling, no data-path
collective), and the max-over-ranks timing reduction rank 0 reports."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import bench
    from gpurify_b200 import _lib

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lay = bench.workload(rank, 6, 8.0)
        p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                 mesh_max_edge_m=0.5e-6, max_panels=-1)
        t = bench.max_over_ranks(10.0 + rank, dist, device="cpu")
        dist.barrier()
        q.put((rank, len(p["verts"]), float(p["verts"].sum()), t))
    finally:
        dist.destroy_process_group()


def test_two_ranks_weak_scaling_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, n0, s0, t0), (r1, n1, s1, t1) = res
    assert (r0, r1) == (0, 1)
    assert (n0, s0) != (n1, s1)  # each rank panelises its own seeded window
    assert t0 == t1 == 11.0     # the slowest rank's time on every rank
