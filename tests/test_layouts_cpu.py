"""The seeded synthetic layouts that the benchmark workloads are built from.

A routing window must never let two different nets touch on one metal layer:
the bridge groups polygons by (net, layer) and does not detect shorts, so an
overlap would silently merge two conductors.  The batch generator must follow
its stated distributions (conductor counts in 2..48, sides 5..60 um), and the
generators must be reproducible from their seed.  The 6-layer large block
keeps 0.15 um between nets, reaches its stated density and panel count, and
its layer parameters (height, thickness) move exactly that layer's metal."""
import math

import numpy as np
import pytest

from gpurify_b200 import layouts


def rects(lay):
    a = lay.store.arrays()
    out = []
    for i in range(len(a["poly_layer"])):
        s, n = int(a["poly_vert_start"][i]), int(a["poly_vert_len"][i])
        xs, ys = a["verts_x"][s:s + n], a["verts_y"][s:s + n]
        out.append((int(a["poly_layer"][i]), int(xs.min()), int(ys.min()), int(xs.max()), int(ys.max())))
    return out


def metal_layers(lay):
    return {lid for name, lid in lay.deck.layers.items() if name.startswith("met")}


@pytest.mark.parametrize("nets,side,seed", [(64, 40.0, 2024), (24, 12.0, 5), (48, 30.0, 11)])
def test_routing_window_nets_never_touch_on_a_layer(nets, side, seed):
    lay = layouts.routing_window(nets, side, seed=seed)
    r = rects(lay)
    metals = metal_layers(lay)
    assert len(r) == len(lay.net_of_poly)
    by_layer = {}
    for (layer, x0, y0, x1, y1), net in zip(r, lay.net_of_poly):
        if layer in metals:
            by_layer.setdefault(layer, []).append((x0, y0, x1, y1, net))
    for layer, items in by_layer.items():
        arr = np.array(items, dtype=np.int64)
        for i in range(len(arr)):
            x0, y0, x1, y1, net = arr[i]
            other = arr[i + 1:]
            hit = ((other[:, 0] < x1) & (other[:, 2] > x0) & (other[:, 1] < y1) & (other[:, 3] > y0) &
                   (other[:, 4] != net))
            assert not hit.any(), f"nets {net} and {other[hit][0, 4]} overlap on layer {layer}"
    # every polygon stays inside the window and every placed net has a metal segment
    side_nm = int(round(side * 1000 / 50)) * 50
    for layer, x0, y0, x1, y1 in r:
        if layer in metals:
            assert 0 <= x0 < x1 <= side_nm and 0 <= y0 < y1 <= side_nm
    placed = set(lay.net_of_poly)
    with_metal = {net for (layer, *_), net in zip(r, lay.net_of_poly) if layer in metals}
    assert placed == with_metal
    assert len(placed) >= 0.9 * nets


def test_routing_window_is_reproducible():
    a = layouts.routing_window(16, 10.0, seed=3)
    b = layouts.routing_window(16, 10.0, seed=3)
    c = layouts.routing_window(16, 10.0, seed=4)
    assert rects(a) == rects(b) and a.net_of_poly == b.net_of_poly
    assert rects(a) != rects(c)


def test_window_batch_follows_its_distributions():
    batch = layouts.window_batch(40, seed=7)
    assert len(batch) == 40
    counts = []
    for lay in batch:
        counts.append(len(set(lay.net_of_poly)))
        a = lay.store.arrays()
        span = max(int(a["verts_x"].max()), int(a["verts_y"].max())) / 1000.0
        assert span <= 60.0 + 1e-9
    assert min(counts) >= 1 and max(counts) <= 48
    # log-uniform in [2, 48]: the median sits near the geometric mean (~9.8)
    assert 4 <= float(np.median(counts)) <= 20
    assert len({lay.name for lay in batch}) == len(batch)


def test_bus_crossing_geometry():
    lay = layouts.bus_crossing()
    r = rects(lay)
    m2, m3 = lay.deck.layers["met2"], lay.deck.layers["met3"]
    bus = [x for x in r if x[0] == m2]
    cross = [x for x in r if x[0] == m3]
    assert len(bus) == 8 and len(cross) == 4
    assert all(x1 - x0 == 30000 and y1 - y0 == 200 for _, x0, y0, x1, y1 in bus)
    assert sorted(y0 for _, _, y0, _, _ in bus) == [400 * b for b in range(8)]
    assert all(x1 - x0 == 400 for _, x0, _, x1, _ in cross)
    xs = sorted(x0 for _, x0, _, _, _ in cross)
    assert all(b - a == 5000 for a, b in zip(xs, xs[1:]))
    assert lay.net_of_poly == list(range(12))


def test_two_wires_geometry():
    lay = layouts.two_wires()
    r = rects(lay)
    assert r == [(lay.deck.layers["met1"], 0, 0, 20000, 140), (lay.deck.layers["met1"], 0, 280, 20000, 420)]
    assert math.isclose(lay.deck.pex[lay.deck.layers["met1"]].thickness_nm, 360.0)


def min_gap_between_nets(lay, layer_ids):
    """Smallest Chebyshev gap (nm) between metal of different nets on one layer."""
    r = rects(lay)
    worst = None
    for lid in layer_ids:
        arr = np.array([(x0, y0, x1, y1, net) for (l, x0, y0, x1, y1), net in zip(r, lay.net_of_poly) if l == lid],
                       dtype=np.int64)
        for i in range(len(arr)):
            o = arr[i + 1:]
            o = o[o[:, 4] != arr[i, 4]]
            if len(o) == 0:
                continue
            gap = np.maximum(np.maximum(o[:, 0] - arr[i, 2], arr[i, 0] - o[:, 2]),
                             np.maximum(o[:, 1] - arr[i, 3], arr[i, 1] - o[:, 3])).min()
            worst = gap if worst is None else min(worst, gap)
    return worst


def layer_density(lay, lid, side_nm, cell=50):
    m = np.zeros((side_nm // cell, side_nm // cell), bool)
    for l, x0, y0, x1, y1 in rects(lay):
        if l == lid:
            m[x0 // cell:x1 // cell, y0 // cell:y1 // cell] = True
    return m.mean()


def test_large_block_clearance_density_and_size():
    from gpurify_b200 import _lib

    lay = layouts.large_block()
    metals = [lid for _, lid, _, _ in layouts.BLOCK_LAYERS]
    assert len(set(lay.net_of_poly)) == 512
    assert min_gap_between_nets(lay, metals) >= 150
    dens = [layer_density(lay, lid, 200000) for lid in metals]
    assert all(0.2 <= d <= 0.5 for d in dens), dens
    # thickness 0.36 to 1.2 um, layers stacked with dielectric between them
    t = [lay.deck.pex[lid].thickness_nm for lid in metals]
    h = [lay.deck.pex[lid].height_nm for lid in metals]
    assert min(t) == 360.0 and max(t) == 1200.0
    assert all(h[i] + t[i] < h[i + 1] for i in range(5))
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=0.8e-6, max_panels=-1)
    assert 1.2e6 <= len(p["verts"]) <= 2.0e6
    assert len(p["nets"]) == 512


def test_layer_parameters_move_only_their_layer():
    """Height and thickness fields of a multi-layer block: each layer's
    parameter moves the panels of that layer's metal only, never the plate."""
    from gpurify_b200 import _lib, sensitivity

    lay = layouts.large_block(n_nets=48, side_um=30.0, seed=9)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=0.8e-6, max_panels=-1)
    names = [name for name, *_ in layouts.BLOCK_LAYERS]
    spans = [sensitivity.layer_span(lay.deck, n) for n in names]
    V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], [("height", a, b) for a, b in spans] +
                                    [("thickness", a, b) for a, b in spans])
    n = len(p["verts"])
    z = p["verts"].reshape(n, 4, 3)[:, :, 2]
    plate = p["cond"] == len(p["nets"])
    covered = np.zeros(n, int)
    for q, (z0, z1) in enumerate(spans):
        Vh = V[q].reshape(n, 4, 3)
        moved = np.abs(Vh).max(axis=(1, 2)) > 0
        assert moved.any()
        assert np.all((z[moved] >= z0 - 1e-12) & (z[moved] <= z1 + 1e-12))
        assert np.all(Vh[moved][:, :, 2] == 1.0) and np.all(Vh[:, :, :2] == 0.0)
        Vt = V[6 + q].reshape(n, 4, 3)[:, :, 2]
        np.testing.assert_allclose(Vt[moved], (z[moved] - z0) / (z1 - z0))
        covered += moved
    assert covered.max() == 1
    assert not np.any(covered[plate])
    assert np.all(covered[~plate] == 1)


def test_config_parity_fixture_meshes_are_the_product_meshes():
    """The product library's host panelisation reproduces, bit for bit, the
    meshes the oracle fixtures of tests/golden/config_parity.json were made
    on (the config-2-style window, the 64-net benchmark window, the bus)."""
    import json
    import os

    from gpurify_b200 import _lib
    from tests.golden import make_config_golden as mk

    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_parity.json")))

    def panelize(lay, edge):
        return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                    mesh_max_edge_m=edge, max_panels=-1)

    assert mk.verts_sha256(mk.window16_panels(panelize)["verts"]) == gold["window16"]["verts_sha256"]
    assert mk.verts_sha256(mk.window64_panels(panelize)["verts"]) == gold["window64"]["verts_sha256"]
    assert mk.verts_sha256(mk.bus_panels(panelize)[1]["verts"]) == gold["bus"]["verts_sha256"]
