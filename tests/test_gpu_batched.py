"""Batched windows (gpx_cap_solve_batched) and graph-captured operator applies.

* A batch of uneven windows (conductor counts log-uniform in 2..48, sides
  5..60 um) solved through the work queue on several streams gives, window by
  window, exactly the Maxwell matrix of a separate gpx_cap_solve call (same
  code path, fixed-order reductions: bit-identical), in FP64 and mixed.
* Operator applies replayed from captured CUDA graphs, and the Arnoldi steps
  run as a device-side graph loop, give results identical to direct launches
  and the same iteration count.
* A failing window names itself and fails the call."""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def windows(n=8, edge=0.5e-6):
    out = []
    for w in layouts.window_batch(n, seed=3):
        p = _lib.bridge_panelize(w.store.arrays(), w.deck.layer_table(), 1.0, w.net_of_poly, mesh_max_edge_m=edge,
                                 max_panels=-1)
        out.append((p["verts"], p["cond"], len(p["nets"]) + 1))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_equals_separate_solves(ctx, precision):
    probs = windows()
    kw = dict(order=5, max_level=-1, precision=precision, skip_ground_rhs=1, far_quad=1, precond=1)
    res = ctx.cap_solve_batched(probs, batch_streams=4, **kw)
    assert len(res) == len(probs)
    for (v, c, nc), (C, rep) in zip(probs, res):
        C1, rep1 = ctx.cap_solve(v, c, nc, **kw)
        assert rep["converged"] == 1 and rep["n_panels"] == len(v)
        assert np.array_equal(C, C1, equal_nan=True)
        assert rep["iterations"] == rep1["iterations"]


def test_graph_replay_matches_direct_launches(ctx):
    v, c, nc = windows(3)[1]
    for precision in (0, 1):
        kw = dict(order=5, max_level=-1, precision=precision, skip_ground_rhs=1, far_quad=1)
        Cg, rg = ctx.cap_solve(v, c, nc, **kw)
        Cd, rd = ctx.cap_solve(v, c, nc, no_graphs=1, **kw)
        assert np.array_equal(Cg, Cd, equal_nan=True)
        assert rg["iterations"] == rd["iterations"]
        # per Arnoldi step the device loop runs its loop-control kernel where
        # the host-driven loop runs its active-column count; each launch of
        # the loop graph adds one loop-entry kernel (one per restart cycle)
        extra = rg["kernel_launches"] - rd["kernel_launches"]
        assert 0 <= extra <= 4 * max(1, rg["outer_iterations"]), (rg["kernel_launches"], rd["kernel_launches"])


def test_batched_error_names_window(ctx):
    probs = windows(3)
    v, c, nc = probs[2]
    bad = c.copy()
    bad[0] = nc  # conductor index out of range
    probs[2] = (v, bad, nc)
    with pytest.raises(_lib.GpxError) as e:
        ctx.cap_solve_batched(probs, batch_streams=3)
    assert e.value.status == 1 and "window 2" in e.value.message
