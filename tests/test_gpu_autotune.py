"""Autotuner (gpx_autotune): the chosen far-field configuration meets the
error target against the all-pairs solve, the choice is cached by problem
signature, and an unreachable target fails closed."""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def window():
    lay = layouts.routing_window(12, 15.0, seed=11)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=0.3e-6, max_panels=-1)
    return p["verts"], p["cond"], len(p["nets"]) + 1


@pytest.mark.parametrize("precision", [0, 1])
def test_tuned_configuration_meets_target(ctx, tmp_path, precision):
    v, c, nc = window()
    base = dict(precision=precision, skip_ground_rhs=1, precond=1)
    cache = str(tmp_path / "tune.txt")
    tuned, rep = ctx.autotune(v, c, nc, target=1e-4, cache_path=cache, **base)
    assert rep["from_cache"] == 0 and rep["candidates"] >= 9
    assert rep["est_rel_err"] <= 0.5e-4 and rep["apply_ms"] > 0
    assert tuned["order"] in (4, 5, 6) and tuned["dense_below"] == -1
    C, r = ctx.cap_solve(v, c, nc, **tuned)
    Cd, _ = ctx.cap_solve(v, c, nc, dense_below=2**31 - 1, skip_ground_rhs=1, tol=1e-10, precond=1)
    R = nc - 1
    d = np.abs(np.diag(Cd[:R, :R]))
    assert (np.abs(C[:R, :R] - Cd[:R, :R]) / d[:, None]).max() < 1e-4
    again, rep2 = ctx.autotune(v, c, nc, target=1e-4, cache_path=cache, **base)
    assert rep2["from_cache"] == 1 and rep2["candidates"] == 0
    assert {k: again[k] for k in ("order", "max_level", "far_quad", "mixed_near")} == \
        {k: tuned[k] for k in ("order", "max_level", "far_quad", "mixed_near")}


def test_unreachable_target_fails_closed(ctx):
    v, c, nc = window()
    with pytest.raises(_lib.GpxError) as e:
        ctx.autotune(v, c, nc, target=1e-12)
    assert e.value.status == 15 and "target error" in e.value.message
