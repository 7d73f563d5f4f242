"""CPU tests of the product library's host side: the C ABI loads and exports
every symbol include/gpx_pex.h declares, and the Python binding's structs have
the header's layout; the bridge panelisation is bit-exact
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


ABI_STRUCTS = {
    "gpx_solve_opts": _lib.SolveOpts, "gpx_solve_report": _lib.SolveReport, "gpx_tune_report": _lib.TuneReport,
    "gpx_panel_problem": _lib.PanelProblem, "gpx_volume_group": _lib.VolumeGroup,
    "gpx_geometry_store": _lib.GeometryStoreC, "gpx_layer_params": _lib.LayerParamsC, "gpx_deck": _lib.DeckC,
    "gpx_net_parasitics": _lib.NetParasiticsC,
}


def test_ctypes_structs_match_header_layout(tmp_path):
    """Every struct the Python binding passes across the ABI has the size and
    field offsets the C compiler gives the header's declaration."""
    import ctypes
    import os
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "gpx_pex.h"', "int main(void) {"]
    for cname, py in ABI_STRUCTS.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c99", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                  text=True).stdout.splitlines())
    for cname, py in ABI_STRUCTS.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


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


def test_plan_rebuilt_after_another_problem_is_identical():
    """The plan builder keeps its per-thread scratch between calls: a plan
    built after a larger and a smaller problem equals the first build, and
    still covers every panel pair exactly once."""
    def panels(nets, side, seed):
        lay = layouts.routing_window(nets, side, seed=seed)
        return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                    mesh_max_edge_m=0.4e-6, max_panels=-1)["verts"]

    a, big, small = panels(8, 10.0, 3), panels(24, 20.0, 4), panels(3, 5.0, 5)
    first = _lib.plan_check(a, 5, 4)
    _lib.plan_check(big, 5, 5)
    _lib.plan_check(small, 4, 3)
    assert _lib.plan_check(a, 5, 4) == first


def test_sensitivity_velocity_fields():
    """Width stretches one wire across its axis (long sides +-1/2), spacing
    translates the same-layer wires past it, thickness moves top faces by +1
    and bottom faces not at all, height lifts the layer, k moves nothing."""
    from gpurify_b200 import sensitivity

    lay = layouts.bus_crossing(bits=3, wires=1, length_nm=6000, cross_pitch_nm=2000)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly, max_panels=-1)
    z0, z1 = sensitivity.layer_span(lay.deck, "met2")
    params = [("width", 1), ("spacing", 0), ("thickness", z0, z1), ("height", z0, z1), ("k",)]
    V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params).reshape(len(params), -1, 4, 3)
    pts = p["verts"].reshape(-1, 4, 3)
    c = p["cond"]
    w = V[0][c == 1]
    assert np.allclose(np.unique(np.round(w[..., 1], 12)).min(), -0.5) and np.allclose(w[..., 1].max(), 0.5)
    assert np.all(V[0][c != 1] == 0) and np.all(V[0][..., [0, 2]] == 0)
    assert np.all(V[1][c == 0] == 0) and np.all(V[1][(c == 1) | (c == 2)][..., 1] == 1.0)
    assert np.all(V[1][c >= 3] == 0)  # the crossing met3 wire and the substrate stay
    th = V[2][c <= 2][..., 2]
    zz = pts[c <= 2][..., 2]
    assert np.allclose(th[np.isclose(zz, z1)], 1.0) and np.allclose(th[np.isclose(zz, z0)], 0.0)
    assert np.all(V[3][c <= 2][..., 2] == 1.0) and np.all(V[3][c > 2] == 0)
    assert np.all(V[4] == 0)
    with pytest.raises(ValueError):
        sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], [("length", 0)])


def test_plan_matches_pinned_checksums():
    """The plan builder reproduces, bit for bit, every plan array of the
    pinned problems (tests/golden/plan_checksums.json, made by
    tests/golden/make_plan_checksums.py), so the device kernels index the same
    plan however the host builds it."""
    import json
    import os

    from tests.golden.make_plan_checksums import cases

    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "plan_checksums.json")))["cases"]
    seen = set()
    for name, verts, order, depth in cases():
        st = _lib.plan_check(verts, order, depth)
        st["n_panels"] = len(verts)
        assert st == gold[name], name
        seen.add(name)
    assert seen == set(gold)


def test_concurrent_host_calls_match_serial():
    """Panelisation keeps its buffers per calling thread and the plan builder
    spreads its panel loops over helper threads: calls from several threads
    at once (ctypes releases the GIL) give exactly the serial results."""
    from concurrent.futures import ThreadPoolExecutor

    # 18k to 40k panels: the plan builder's panel loops run on 2 to 4 helper threads
    lays = [layouts.routing_window(24, 25.0, seed=s) for s in (4, 5)] + [layouts.routing_window(40, 32.0, seed=6),
                                                                      layouts.bus_crossing(), layouts.two_wires()]

    def one(lay):
        p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                 mesh_max_edge_m=0.3e-6, max_panels=-1)
        return p["verts"], p["cond"], _lib.plan_check(p["verts"], 5, 4)["checksum"]

    serial = [one(lay) for lay in lays]
    with ThreadPoolExecutor(4) as ex:
        for _ in range(3):
            for (v, c, h), (v0, c0, h0) in zip(ex.map(one, lays), serial):
                assert np.array_equal(v, v0) and np.array_equal(c, c0) and h == h0
