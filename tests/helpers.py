"""Shared fixtures-free helpers for the tests (geometry builders that mirror
the reference's test geometries)."""
import numpy as np

from gpurify_b200.geometry import Deck, GeometryStore, PexLayerParams


def bridge_test_deck(method="field_solver"):
    """crates/pex/tests/bridge.rs:8-43: met1 (sheet 0.1, t 200 nm, h 500 nm,
    k 3.9) and via1 (fixed 5 ohm)."""
    return Deck.from_dict({
        "layers": {"met1": {"layer": 68, "datatype": 20}, "via1": {"layer": 67, "datatype": 44}},
        "pex_method": method,
        "pex": {
            "met1": {"sheet_res_ohm_sq": 0.1, "area_cap_af_um2": 25.0, "fringe_cap_af_um": 40.0,
                     "coupling_cap_af_um": 100.0, "coupling_ref_spacing_nm": 200.0, "thickness_nm": 200.0,
                     "height_nm": 500.0, "dielectric_k": 3.9},
            "via1": {"sheet_res_ohm_sq": 0.0, "area_cap_af_um2": 0.0, "fringe_cap_af_um": 0.0,
                     "coupling_cap_af_um": 0.0, "coupling_ref_spacing_nm": 1.0, "via_res_ohm": 5.0,
                     "thickness_nm": 200.0, "height_nm": 300.0, "dielectric_k": 3.9},
        },
    })


def rel_max(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def with_layer_k(lay, ks):
    """The layout with its deck's dielectric constants set per metal layer
    name (a stack of several k)."""
    for name, k in ks.items():
        lay.deck.pex[lay.deck.layers[name]].dielectric_k = k
    return lay


def rect_groups(store, deck, net_of_poly):
    """bridge.rs:94-142 for layouts of rectangles: one (net, layer) group per
    volume-conductor layer of a net (bridge.rs:171-178), z from the layer's
    height and thickness, in BTreeMap<(net, layer)> order.  Returns (groups,
    rects, xy_scale_m) for gpx_cap_solve_groups."""
    a = store.arrays()
    grouped = {}
    for i, layer in enumerate(a["poly_layer"].tolist()):
        p = deck.pex.get(layer)
        if p is None:
            continue
        volume = (p.sheet_res_ohm_sq != 0.0 or p.area_cap_af_um2 != 0.0 or p.fringe_cap_af_um != 0.0
                  or p.coupling_cap_af_um != 0.0 or p.interlayer_cap_af_um2 != 0.0
                  or (p.thickness_nm > 0.0 and p.via_res_ohm == 0.0))
        if not volume:
            continue
        s, n = int(a["poly_vert_start"][i]), int(a["poly_vert_len"][i])
        xs, ys = a["verts_x"][s:s + n], a["verts_y"][s:s + n]
        assert n == 4, "rectangles only"
        key = (int(net_of_poly[i]), layer)
        g = grouped.setdefault(key, {"z": (p.height_nm * 1e-9, (p.height_nm + p.thickness_nm) * 1e-9),
                                     "k": p.dielectric_k, "rects": []})
        g["rects"].append((int(xs.min()), int(ys.min()), int(xs.max()), int(ys.max())))
    groups, rects = [], []
    for (net, _), g in sorted(grouped.items()):
        groups.append((net, g["z"][0], g["z"][1], g["k"], len(rects), len(g["rects"])))
        rects.extend(g["rects"])
    return groups, np.array(rects, dtype=np.int32).reshape(-1, 4), deck.dbu_nm * 1e-9
