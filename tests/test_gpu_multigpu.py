"""GPU side of the multi-GPU path: a window's conductor columns solved in
blocks (gpx_solve_opts.col_begin / col_count) equal the same columns of one
full solve, and the sharded solve of gpurify_b200/multigpu.py run through a
one-rank process group returns the full solve's matrix.  (Every GPU call of
this pool gets one GPU; the two-rank partition and gather logic is covered
on CPU by tests/test_multigpu_cpu.py.)"""
import socket

import numpy as np
import pytest

from gpurify_b200 import _lib, layouts, multigpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def window():
    lay = layouts.routing_window(7, 8.0, seed=5)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=0.4e-6, max_panels=-1)
    return p["verts"], p["cond"], len(p["nets"]) + 1


KW = dict(order=4, max_level=-1, far_quad=1, precond=1, dense_below=-1, tol=1e-10)


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED])
def test_column_blocks_match_full_solve(ctx, window, precision):
    verts, cond, nc = window
    R = nc - 1
    C, _ = ctx.cap_solve(verts, cond, nc, skip_ground_rhs=1, precision=precision, **KW)
    d = np.abs(np.diag(C[:R, :R]))
    for b, c in multigpu.column_blocks(R, 3):
        Cb, rep = ctx.cap_solve(verts, cond, nc, skip_ground_rhs=1, col_begin=b, col_count=c, precision=precision,
                                **KW)
        assert rep["n_rhs"] == c
        blk = Cb[:, b : b + c]
        assert np.isfinite(blk).all()
        assert (np.abs(blk[:R] - C[:R, b : b + c]) / d[b : b + c]).max() < 1e-9
        others = np.delete(Cb, np.arange(b, b + c), axis=1)
        assert np.isnan(others).all()


def test_column_subset_rejects_out_of_range(ctx, window):
    verts, cond, nc = window
    with pytest.raises(_lib.GpxError, match="column subset"):
        ctx.cap_solve(verts, cond, nc, col_begin=nc - 1, col_count=2, **KW)


def test_sharded_solve_through_a_process_group(ctx, window):
    import torch.distributed as dist

    verts, cond, nc = window
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        C = multigpu.solve_window_sharded(nc, dist, skip_ground_rhs=True, ctx=ctx, verts=verts, cond=cond,
                                          precision=_lib.PREC_FP64, **KW)
    finally:
        dist.destroy_process_group()
    ref, _ = ctx.cap_solve(verts, cond, nc, skip_ground_rhs=1, precision=_lib.PREC_FP64, **KW)
    np.testing.assert_array_equal(np.isnan(C), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.abs(C[ok] - ref[ok]).max() / np.abs(ref[ok]).max() < 1e-12
