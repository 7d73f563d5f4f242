"""Generates tests/golden/config_parity.json: the CPU oracle's results on the
benchmark configurations' own geometries, for the GPU parity tests in
tests/test_gpu_config_parity.py.

The reference publishes no field-solver numbers; the oracle (oracle/orc.cpp,
a restatement of the reference's CPU field solver pinned by
tests/test_oracle_pins.py) stands in for it.  Fixtures:

* ``window16``: a config-2-style routing window (16 nets, 15 x 15 um, the
  3-layer stack, seed 11) at a 0.4 um panel edge, 6,079 panels.  Oracle dense
  LU Maxwell matrix (cap/solver.rs:100-134, the FP64 dense-direct reference)
  and the oracle FMM in the reference's mode (order 4, depth 4, centroid
  sources, Jacobi, cap/fmm_solver.rs:147-172) at GMRES tol 1e-10, every
  conductor.
* ``window64``: the benchmark's 64-net 40 x 40 um window (seed 2024, 0.25 um
  edge, 69,253 panels), oracle FMM in the reference's mode at depth 5 (order
  4, centroid sources, Jacobi, tol 1e-10), columns of 4 nets spread over the
  window.
* ``bus``: the config-4 bus (8-bit met2 bus crossed by 4 met3 wires, 0.14 um
  edge, 42,588 panels): central differences (relative step 1e-3) of the
  oracle FMM (order 5, depth 5, centroid sources, tol 1e-10) along the width
  of bus bit 3 and the spacing after bit 3, on conductor columns 3 and 4.

Run:  python tests/golden/make_config_golden.py   (several minutes on 8 cores)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "config_parity.json")

WINDOW16 = dict(nets=16, side_um=15.0, seed=11, edge_m=0.4e-6)
WINDOW64 = dict(nets=64, side_um=40.0, seed=2024, edge_m=0.25e-6, columns=[0, 21, 42, 63], order=4, depth=5)
BUS = dict(edge_m=0.14e-6, order=5, depth=5, params=[("width", 3), ("spacing", 3)], columns=[3, 4], rel_step=1e-3)


def verts_sha256(verts: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(verts, dtype="<f8").tobytes()).hexdigest()


def window16_panels(panelize):
    from gpurify_b200 import layouts

    lay = layouts.routing_window(WINDOW16["nets"], WINDOW16["side_um"], seed=WINDOW16["seed"])
    return panelize(lay, WINDOW16["edge_m"])


def window64_panels(panelize):
    from gpurify_b200 import layouts

    lay = layouts.routing_window(WINDOW64["nets"], WINDOW64["side_um"], seed=WINDOW64["seed"])
    return panelize(lay, WINDOW64["edge_m"])


def bus_panels(panelize):
    from gpurify_b200 import layouts

    lay = layouts.bus_crossing()
    return lay, panelize(lay, BUS["edge_m"])


def oracle_panelize(lay, edge):
    import oracle

    return oracle.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0,
                                  mesh_max_edge_m=edge, max_panels=-1)


def bus_step(lay, kind):
    """The parameter's value (metres) the relative step is taken of: the bus
    wire width (0.2 um) for width, the bus gap (0.2 um) for spacing."""
    return 0.2e-6


def generate() -> dict:
    import oracle
    from gpurify_b200 import sensitivity

    oracle.build()
    out = {"generator": "tests/golden/make_config_golden.py", "units": "farads (Maxwell), metres (geometry)"}

    t0 = time.time()
    p = window16_panels(oracle_panelize)
    nc = len(p["nets"]) + 1
    Cd = oracle.cap_dense(p["verts"], p["cond"], nc)
    Cf, rep = oracle.cap_fmm(p["verts"], p["cond"], nc, order=4, max_level=4, tol=1e-10)
    out["window16"] = dict(WINDOW16, n_panels=int(len(p["verts"])), verts_sha256=verts_sha256(p["verts"]),
                           nets=p["nets"].tolist(), maxwell_dense=Cd.tolist(), maxwell_fmm_ref=Cf.tolist(),
                           fmm_ref={"order": 4, "max_level": 4, "tol": 1e-10,
                                    "max_iterations": int(rep["max_iterations"])})
    print(f"window16: {len(p['verts'])} panels, {time.time() - t0:.1f} s", flush=True)

    t0 = time.time()
    p = window64_panels(oracle_panelize)
    nc = len(p["nets"]) + 1
    sv = oracle.FmmSolver(p["verts"], p["cond"], nc, order=WINDOW64["order"], max_level=WINDOW64["depth"])
    cols = []
    for j in WINDOW64["columns"]:
        col, r = sv.solve_column(j, tol=1e-10)
        assert r["converged"]
        cols.append(col.tolist())
    sv.close()
    out["window64"] = dict(WINDOW64, n_panels=int(len(p["verts"])), verts_sha256=verts_sha256(p["verts"]),
                           maxwell_columns=cols, tol=1e-10)
    print(f"window64: {len(p['verts'])} panels, {time.time() - t0:.1f} s", flush=True)

    t0 = time.time()
    lay, p = bus_panels(oracle_panelize)
    nc = len(p["nets"]) + 1
    params = [(k, b) for k, b in BUS["params"]]
    V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
    fd = []
    for q, (kind, bit) in enumerate(params):
        h = BUS["rel_step"] * bus_step(lay, kind)
        cols = {}
        for sgn in (1, -1):
            v = p["verts"] + sgn * h * V[q]
            sv = oracle.FmmSolver(v, p["cond"], nc, order=BUS["order"], max_level=BUS["depth"])
            for j in BUS["columns"]:
                col, r = sv.solve_column(j, tol=1e-10)
                assert r["converged"]
                cols[(sgn, j)] = col
            sv.close()
        fd.append({"param": [kind, bit], "step_m": h,
                   "dC_columns": [((cols[(1, j)] - cols[(-1, j)]) / (2 * h)).tolist() for j in BUS["columns"]]})
    out["bus"] = dict(edge_m=BUS["edge_m"], order=BUS["order"], depth=BUS["depth"], columns=BUS["columns"],
                      rel_step=BUS["rel_step"], n_panels=int(len(p["verts"])), verts_sha256=verts_sha256(p["verts"]),
                      fd=fd, tol=1e-10)
    print(f"bus: {len(p['verts'])} panels, {time.time() - t0:.1f} s", flush=True)
    return out


def main():
    doc = generate()
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
