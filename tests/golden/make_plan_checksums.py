"""Pins the host plan builder: for a set of panel problems and (order, depth)
pairs, the plan statistics and the 64-bit checksum of every plan array
(gpx_plan_check) as the builder produced them when this file was written.
A faster builder must reproduce each checksum bit for bit, so the device
kernels see the same plan.  The cases from ``one_panel_o5_d4`` on were added
with the threaded builder, after its plan arrays had been compared equal to
those of the serial builder on the same inputs.

    python tests/golden/make_plan_checksums.py   # rewrites plan_checksums.json
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def random_panels(n, seed):
    """Seeded panels with mixed sizes in a flat slab: quadrilaterals and
    triangles (fourth vertex repeating the third), some sharing centroids."""
    rng = np.random.default_rng(seed)
    c = rng.uniform([0, 0, 0], [40e-6, 30e-6, 3e-6], (n, 3))
    c[n // 10 : n // 10 + 20] = c[0]  # coincident centroids
    s = rng.uniform(0.05e-6, 1.5e-6, (n, 2))
    v = np.zeros((n, 4, 3))
    v[:, 0] = c + np.c_[-s[:, 0], -s[:, 1], np.zeros(n)] / 2
    v[:, 1] = c + np.c_[s[:, 0], -s[:, 1], np.zeros(n)] / 2
    v[:, 2] = c + np.c_[s[:, 0], s[:, 1], np.zeros(n)] / 2
    v[:, 3] = c + np.c_[-s[:, 0], s[:, 1], np.zeros(n)] / 2
    tri = rng.random(n) < 0.3
    v[tri, 3] = v[tri, 2]
    return v.reshape(n, 12)


def cases():
    from gpurify_b200 import _lib, layouts

    def bridge(lay, edge=0.0):
        return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                    mesh_max_edge_m=edge, max_panels=-1)["verts"]

    bench = bridge(layouts.routing_window(64, 40.0, seed=2024), 0.25e-6)
    mid = bridge(layouts.routing_window(16, 20.0, seed=7), 0.3e-6)
    yield "bench_window_o5_d5", bench, 5, 5
    yield "bench_window_o4_d4", bench, 4, 4
    yield "window16_o6_d3", mid, 6, 3
    yield "window16_o5_d6", mid, 5, 6
    yield "window16_o3_d2", mid, 3, 2
    yield "window16_o4_d1", mid, 4, 1
    yield "two_wires_o4_d4", bridge(layouts.two_wires()), 4, 4
    yield "bus_crossing_o6_d4", bridge(layouts.bus_crossing()), 6, 4
    yield "random_o5_d7", random_panels(20000, 11), 5, 7
    yield "random_o2_d3", random_panels(3000, 12), 2, 3
    # sizes around the plan builder's 8192-panel chunks, one panel, depth 12,
    # and panels that all share one centroid (a zero-size bounding box)
    yield "one_panel_o5_d4", random_panels(1, 21), 5, 4
    yield "random8193_o6_d7", random_panels(8193, 25), 6, 7
    yield "random16385_o3_d12", random_panels(16385, 26), 3, 12
    yield "random40000_o5_d4", random_panels(40000, 27), 5, 4
    same = random_panels(500, 28).reshape(-1, 4, 3)
    same[:] = same[0]
    yield "one_centroid_o5_d4", same.reshape(-1, 12), 5, 4


def generate():
    from gpurify_b200 import _lib

    out = {"generator": "tests/golden/make_plan_checksums.py", "cases": {}}
    for name, verts, order, depth in cases():
        st = _lib.plan_check(verts, order, depth)
        st["n_panels"] = int(len(verts))
        out["cases"][name] = st
    return out


if __name__ == "__main__":
    data = generate()
    with open(os.path.join(HERE, "plan_checksums.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print(json.dumps(data, indent=1)[:2000])
