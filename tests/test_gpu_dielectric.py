"""Stacks of several dielectric constants on the GPU, through the C ABI
(gpx_extract_quasistatic and gpx_cap_solve_groups).

The bridge gives every panel a conductor role in its own layer's k
(bridge.rs:409-430 -> cap/dielectric.rs:76-150): the vacuum potential system,
each panel's charge counted k times.  The reference takes that path below 500
panels only (all pairs, LU); this solver at any size.

* All pairs (410 panels, three k, nets crossing layers): per-net C against
  the oracle's restatement (dense LU), 1e-8.
* FMM (821 panels, one k per net): the Maxwell matrix is the vacuum one with
  each row scaled by its net's k (the substrate's by the lowest layer's), to
  rounding: the k never enters the operator, so both solves produce the same
  charges.
* FMM (1,155 panels, nets crossing layers): C is linear in the layer k,
  C(a) + C(b) = C(a + b) to rounding, for the same reason.
* gpx_cap_solve_groups gives the per-net values of gpx_extract_quasistatic on
  the same groups; the matrix of several k is not symmetric, so a skipped
  substrate column comes back NaN instead of filled by symmetry.
* gpx_cap_solve_eps refuses a permittivity that is not finite and positive,
  naming the panel, before any set-up.
"""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts, pex
from tests.helpers import rect_groups, with_layer_k

pytestmark = pytest.mark.gpu

KS = {"met1": 3.9, "met2": 3.0, "met3": 2.5}


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def test_all_pairs_stack_matches_oracle(ctx, orc):
    lay = with_layer_k(layouts.routing_window(4, 6.0, seed=11), KS)
    p = orc.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0)
    assert len(np.unique(p["eps"])) == 3 and len(p["verts"]) < 500
    ref = orc.cap_dense_eps(p["verts"], p["cond"], len(p["nets"]) + 1, p["eps"])
    rep = {}
    out = pex.extract_quasistatic(lay.store, lay.deck, lay.net_of_poly, ctx=ctx, report=rep)
    assert rep["dense"] == 1 and rep["converged"] == 1
    for i, net in enumerate(p["nets"].tolist()):
        want = ref[i, i] * 1e18
        assert abs(out[net].cap_af - want) <= 1e-8 * want, (net, out[net].cap_af, want)


def test_fmm_rows_scale_with_each_nets_k(ctx):
    lay = with_layer_k(layouts.bus_crossing(), {"met2": 3.0, "met3": 2.5})
    groups, rects, scale = rect_groups(lay.store, lay.deck, lay.net_of_poly)
    nets, af, Ck, rep = ctx.cap_solve_groups(groups, rects, scale)
    assert rep["dense"] == 0 and rep["converged"] == 1
    vac = [(g[0], g[1], g[2], 1.0, g[4], g[5]) for g in groups]
    _, _, C1, rep1 = ctx.cap_solve_groups(vac, rects, scale)
    assert rep1["dense"] == 0
    k_of = {g[0]: g[3] for g in groups}
    lowest = min(groups, key=lambda g: g[1])[3]
    row_k = np.array([k_of[n] for n in nets.tolist()] + [lowest])
    assert np.all(np.isfinite(Ck))
    assert np.abs(Ck - row_k[:, None] * C1).max() <= 1e-12 * np.abs(np.diag(C1)).max()
    assert np.allclose(af, np.diag(Ck)[:-1] * 1e18, rtol=1e-15, atol=0)


def test_fmm_stack_is_linear_in_layer_k(ctx):
    def solve(ks):
        lay = with_layer_k(layouts.routing_window(8, 10.0, seed=3), ks)
        groups, rects, scale = rect_groups(lay.store, lay.deck, lay.net_of_poly)
        _, _, C, rep = ctx.cap_solve_groups(groups, rects, scale)
        assert rep["dense"] == 0 and rep["converged"] == 1
        return C

    a = {"met1": 3.9, "met2": 3.0, "met3": 2.5}
    b = {"met1": 1.0, "met2": 2.0, "met3": 0.5}
    ab = {k: a[k] + b[k] for k in a}
    Ca, Cb, Cab = solve(a), solve(b), solve(ab)
    assert np.abs(Ca + Cb - Cab).max() <= 1e-12 * np.abs(np.diag(Cab)).max()


def test_groups_entry_matches_extract_and_leaves_skipped_column_nan(ctx):
    lay = with_layer_k(layouts.routing_window(4, 6.0, seed=11), KS)
    groups, rects, scale = rect_groups(lay.store, lay.deck, lay.net_of_poly)
    nets, af, C, rep = ctx.cap_solve_groups(groups, rects, scale, skip_ground_rhs=1)
    out = pex.extract_quasistatic(lay.store, lay.deck, lay.net_of_poly, ctx=ctx, skip_ground_rhs=1)
    for net, v in zip(nets.tolist(), af.tolist()):
        assert abs(out[net].cap_af - v) <= 1e-10 * v
    n = len(nets)
    assert np.all(np.isfinite(C[:, :n]))
    assert np.all(np.isnan(C[:, n]))


def test_invalid_permittivity_is_refused_before_any_work(ctx, orc):
    a, ca = orc.plate(0, 0, 0, 0.2, 0.2, 4, 4, 0)
    b, cb = orc.plate(0, 0, 0.02, 0.2, 0.2, 4, 4, 1)
    v, c = np.vstack([a, b]), np.concatenate([ca, cb])
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        eps = np.full(len(v), 2.0)
        eps[3] = bad
        with pytest.raises(_lib.GpxError) as e:
            ctx.cap_solve(v, c, 2, eps=eps)
        assert e.value.status == 1 and "panel 3" in e.value.message
