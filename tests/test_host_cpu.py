"""CPU tests of the product library's host side: the C ABI loads and exports
every symbol include/gpx_pex.h declares; the bridge panelisation is bit-exact
with the oracle; the octree plan covers every panel pair exactly once; bridge
errors carry the reference's messages (bridge.rs:35-56, rects.rs:10-31)."""
import re

import numpy as np
import pytest

from gpurify_b200 import _lib, layouts
from gpurify_b200.geometry import GeometryStore
from tests.helpers import bridge_test_deck

HEADER = "include/gpx_pex.h"


def test_header_symbols_exported():
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    text = open(os.path.join(root, HEADER)).read()
    declared = set(re.findall(r"^(?:gpx_status|void|void\*|const char\*)\s+(gpx_\w+)\(", text, re.M))
    assert declared == set(_lib.EXPORTS)
    L = _lib.load()
    for name in declared:
        assert hasattr(L, name), name


def test_no_device_is_reported_not_faked():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.GpxError) as e:
        _lib.Context(0)
    assert e.value.status == 3


LAYOUTS = [layouts.two_wires, lambda: layouts.routing_window(12, 15.0, seed=5), layouts.bus_crossing]


@pytest.mark.parametrize("make", LAYOUTS)
@pytest.mark.parametrize("edge", [0.0, 0.3e-6])
def test_panelize_bit_exact_vs_oracle(orc, make, edge):
    lay = make()
    a, lt = lay.store.arrays(), lay.deck.layer_table()
    ref = orc.bridge_panelize(a, lt, lay.net_of_poly, 1.0, edge, -1)
    got = _lib.bridge_panelize(a, lt, 1.0, lay.net_of_poly, mesh_max_edge_m=edge, max_panels=-1)
    assert got["verts"].shape == ref["verts"].shape
    assert np.array_equal(got["verts"], ref["verts"])  # bit-exact coordinates
    assert np.array_equal(got["cond"], ref["cond"])
    assert np.array_equal(got["eps"], ref["eps"])
    assert np.array_equal(got["nets"], ref["nets"])


def test_two_wire_reference_mesh_counts():
    lay = layouts.two_wires()
    got = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)
    assert len(got["verts"]) == 513
    assert np.bincount(got["cond"]).tolist() == [94, 94, 325]


def test_same_net_overlaps_are_unioned(orc):
    deck = bridge_test_deck()
    st = GeometryStore()
    m1 = deck.layer_id("met1")
    st.add_rect(m1, 0, 0, 1000, 500)
    st.add_rect(m1, 500, 0, 1000, 500)
    got = _lib.bridge_panelize(st.arrays(), deck.layer_table(), 1.0, [3, 3])
    ref = orc.bridge_panelize(st.arrays(), deck.layer_table(), [3, 3], 1.0)
    assert np.array_equal(got["verts"], ref["verts"])
    # the union is one 1500 x 500 block: no sidewall at x = 500 or 1000 inside it
    xs = got["verts"][got["cond"] == 0].reshape(-1, 4, 3)[:, :, 0]
    side_x = [v[0] for v in xs if np.all(v == v[0])]
    assert all(abs(x - 500e-9) > 1e-15 for x in side_x)


def test_non_manhattan_fails_closed():
    deck = bridge_test_deck()
    st = GeometryStore()
    st.add_polygon(deck.layer_id("met1"), [(0, 0), (1000, 0), (800, 500), (0, 500)])
    with pytest.raises(_lib.GpxError) as e:
        _lib.bridge_panelize(st.arrays(), deck.layer_table(), 1.0, [1])
    assert e.value.status == 12 and e.value.polygon == 0
    assert "non-rectilinear" in e.value.message


def test_invalid_dbu_and_process_values():
    deck = bridge_test_deck()
    st = GeometryStore()
    st.add_rect(deck.layer_id("met1"), 0, 0, 1000, 500)
    for dbu in (0.0, -1.0, float("nan")):
        with pytest.raises(_lib.GpxError) as e:
            _lib.bridge_panelize(st.arrays(), deck.layer_table(), dbu, [1])
        assert e.value.status == 10
    lt = deck.layer_table()
    for d in lt:
        d["dielectric_k"] = float("inf")
    with pytest.raises(_lib.GpxError) as e:
        _lib.bridge_panelize(st.arrays(), lt, 1.0, [1])
    assert e.value.status == 11


def test_panel_capacity_limit():
    lay = layouts.routing_window(64)
    with pytest.raises(_lib.GpxError) as e:
        _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=0.25e-6)
    assert e.value.status == 14 and "limit is 20000" in e.value.message


def test_via_only_net_makes_no_panels():
    deck = bridge_test_deck()
    st = GeometryStore()
    v1 = deck.layer_id("via1")
    st.add_rect(v1, 0, 0, 100, 100)
    st.add_rect(v1, 200, 0, 100, 100)
    got = _lib.bridge_panelize(st.arrays(), deck.layer_table(), 1.0, [9, 9])
    assert len(got["verts"]) == 0


@pytest.mark.parametrize("depth", [1, 2, 3, 4, 5])
def test_plan_covers_every_pair_once(depth):
    lay = layouts.bus_crossing()
    got = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)
    st = _lib.plan_check(got["verts"], 4, depth)  # raises on any broken invariant
    n = len(got["verts"])
    assert st["near_pairs"] + st["far_panel_pairs"] == n * n
    if depth == 1:
        assert st["m2l_box_pairs"] == 0
