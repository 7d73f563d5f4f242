"""Stacks of several dielectric constants, CPU side.

The bridge solves a stack of several k with every panel a conductor panel in
its own surrounding k (bridge.rs:409-430 -> cap/dielectric.rs:76-150 with
conductor roles): the potential system is the vacuum one, and each panel's
charge counts k times, C[i][j] = sum_{k on i} eps_k sigma_k a_k.  The
substrate plate takes the k of the lowest group (bridge.rs:362-365).

* The oracle's restatement reduces to k times the vacuum solve when every k
  is equal, scales each row by its conductor's k when the k is uniform per
  conductor, and is linear in the k.
* The product's panelisation carries the per-panel k bit-exact with the
  oracle's on stacks of several k, the substrate's being the lowest layer's.
"""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts
from tests.helpers import with_layer_k

KS = {"met1": 3.9, "met2": 3.0, "met3": 2.5}


def plates(orc):
    a, ca = orc.plate(0, 0, 0, 0.2, 0.2, 6, 6, 0)
    b, cb = orc.plate(0, 0, 0.02, 0.2, 0.2, 6, 6, 1)
    return np.vstack([a, b]), np.concatenate([ca, cb])


def test_oracle_stack_reduces_to_the_vacuum_solve(orc):
    v, c = plates(orc)
    C0 = orc.cap_dense(v, c, 2)
    C = orc.cap_dense_eps(v, c, 2, np.full(len(v), 3.9))
    assert np.abs(C - 3.9 * C0).max() <= 1e-13 * np.abs(C0).max()
    # one k per conductor: row i scales by conductor i's k
    eps = np.where(c == 0, 3.9, 2.0)
    C = orc.cap_dense_eps(v, c, 2, eps)
    assert np.abs(C - np.array([[3.9], [2.0]]) * C0).max() <= 1e-13 * np.abs(C0).max()


def test_oracle_stack_is_linear_in_k(orc):
    lay = with_layer_k(layouts.routing_window(3, 5.0, seed=5), KS)
    p = orc.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0)
    nc = len(p["nets"]) + 1
    rng = np.random.default_rng(1)
    a, b = rng.uniform(1.0, 4.0, len(p["verts"])), rng.uniform(1.0, 4.0, len(p["verts"]))
    Ca = orc.cap_dense_eps(p["verts"], p["cond"], nc, a)
    Cb = orc.cap_dense_eps(p["verts"], p["cond"], nc, b)
    Cab = orc.cap_dense_eps(p["verts"], p["cond"], nc, a + b)
    assert np.abs(Ca + Cb - Cab).max() <= 1e-13 * np.abs(Cab).max()


@pytest.mark.parametrize("make", [lambda: layouts.routing_window(4, 6.0, seed=11), layouts.bus_crossing])
def test_product_panelisation_carries_per_panel_k(orc, make):
    lay = with_layer_k(make(), KS)
    a, lt = lay.store.arrays(), lay.deck.layer_table()
    ref = orc.bridge_panelize(a, lt, lay.net_of_poly, 1.0, 0.0, -1)
    got = _lib.bridge_panelize(a, lt, 1.0, lay.net_of_poly, max_panels=-1)
    for key in ("verts", "cond", "eps", "nets"):
        assert np.array_equal(got[key], ref[key]), key
    assert len(np.unique(got["eps"])) > 1
    # the substrate plate takes the k of the lowest group's layer
    ground = got["cond"] == len(got["nets"])
    lowest = min((lay.deck.pex[lid].height_nm, lay.deck.pex[lid].dielectric_k)
                 for lid in set(a["poly_layer"].tolist()) if lay.deck.pex[lid].thickness_nm > 0)[1]
    assert np.all(got["eps"][ground] == lowest)
