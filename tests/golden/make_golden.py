"""Generates the golden fixtures of the field-solver path (tests/golden/*.json).

The reference publishes no field-solver numbers, so the goldens are outputs
of the CPU oracle (oracle/orc.cpp, a restatement of the reference's CPU field
solver that tests/test_oracle_pins.py pins against the reference's own
known-answer tests).  They freeze the oracle's results on:

* the two-wire met1 layout on the reference mesh (513 panels incl. the
  325-panel ground plate), which the reference bridge sends to
  fmm_solver::solve(order 4, depth 4, tol 1e-8) (bridge.rs:403);
* a three-net layout on the bridge tests' deck (tests/bridge.rs:8-43 deck
  values: met1 200 nm thick, 500 nm high, k 3.9), below 500 panels, so the
  reference takes its dense LU path (cap/solver.rs:100-134);
* the isolated sphere (cap_validation.rs:9-30, 320 panels) and the
  parallel plates (cap_validation.rs:32-60);
* a few Wilton integrals (integrals/panel.rs:147-208);
* the precorrected operator apply y = P sigma on the two-wire mesh
  (cap/fmm_solver.rs:109-129) for one seeded sigma.

Run:  python tests/golden/make_golden.py   (writes tests/golden/field_solver.json)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "field_solver.json")


def verts_sha256(verts: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(verts, dtype="<f8").tobytes()).hexdigest()


def bridge_deck_layout():
    """Three met1 nets on the bridge tests' deck: two parallel wires and a
    short stub, DBU 1 nm (own geometry; the deck values are the reference
    test's)."""
    from gpurify_b200.geometry import GeometryStore
    from tests.helpers import bridge_test_deck

    deck = bridge_test_deck()
    m1 = deck.layer_id("met1")
    st = GeometryStore()
    st.add_rect(m1, 0, 0, 4000, 300)
    st.add_rect(m1, 0, 600, 4000, 300)
    st.add_rect(m1, 1000, 1400, 1500, 500)
    return st, deck, [10, 20, 30]


def generate() -> dict:
    import oracle
    from gpurify_b200 import layouts

    oracle.build()
    out = {"generator": "tests/golden/make_golden.py", "units": "farads (Maxwell), metres (geometry)"}

    # config 1 on the reference mesh
    lay = layouts.two_wires()
    p = oracle.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0)
    ncond = len(p["nets"]) + 1
    C, rep = oracle.cap_fmm(p["verts"], p["cond"], ncond, order=4, max_level=4, tol=1e-8)
    k = float(p["eps"][0])
    out["two_wires_reference_mesh"] = {
        "n_panels": int(len(p["verts"])),
        "panels_per_conductor": np.bincount(p["cond"]).tolist(),
        "verts_sha256": verts_sha256(p["verts"]),
        "nets": p["nets"].tolist(),
        "dielectric_k": k,
        "solver": {"order": 4, "max_level": 4, "tol": 1e-8},
        "maxwell": C.tolist(),
        "cap_af": [float(C[i, i] * k * 1e18) for i in range(ncond - 1)],
        "gmres_iterations_max": int(rep["max_iterations"]),
    }

    # operator apply on the same mesh
    rng = np.random.default_rng(7)
    sigma = rng.standard_normal(len(p["verts"]))
    y, nnz = oracle.fmm_cap_apply(p["verts"], sigma, 4, 4)
    out["two_wires_operator_apply"] = {"order": 4, "max_level": 4, "nnz_near": int(nnz), "sigma": sigma.tolist(),
                                       "y": y.tolist()}

    # bridge deck, dense path
    st, deck, nets = bridge_deck_layout()
    p = oracle.bridge_panelize(st.arrays(), deck.layer_table(), nets, 1.0)
    ncond = len(p["nets"]) + 1
    assert len(p["verts"]) < 500, len(p["verts"])
    C = oracle.cap_dense(p["verts"], p["cond"], ncond)
    k = float(p["eps"][0])
    out["bridge_deck_three_nets"] = {
        "n_panels": int(len(p["verts"])),
        "verts_sha256": verts_sha256(p["verts"]),
        "nets": p["nets"].tolist(),
        "dielectric_k": k,
        "maxwell": C.tolist(),
        "cap_af": [float(C[i, i] * k * 1e18) for i in range(ncond - 1)],
    }

    # sphere and plates
    v, c = oracle.icosphere([0, 0, 0], 1.0, 2, 0)
    out["sphere_320"] = {"center": [0, 0, 0], "radius": 1.0, "subdivisions": 2,
                         "maxwell": oracle.cap_dense(v, c, 1).tolist()}
    a, ca = oracle.plate(0, 0, 0, 0.2, 0.2, 10, 10, 0)
    b, cb = oracle.plate(0, 0, 0.02, 0.2, 0.2, 10, 10, 1)
    out["plates_10x10"] = {"side": 0.2, "gap": 0.02, "n": 10,
                           "maxwell": oracle.cap_dense(np.vstack([a, b]), np.concatenate([ca, cb]), 2).tolist()}

    # Wilton integrals: self, near off-plane, edge-aligned, far
    cases = []
    quad = [[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.5, 0.5, 0.0], [-0.5, 0.5, 0.0]]
    tri = [[0, 0, 0], [1, 0, 0], [0.2, 0.9, 0], [0.2, 0.9, 0]]
    for verts, pt in ((quad, [0, 0, 0]), (quad, [0.1, 0.2, 0.3]), (quad, [0.5, 0.0, 0.0]), (quad, [2.0, -1.0, 0.5]),
                      (quad, [0, 0, 50.0]), (tri, [0.3, 0.2, 0.0]), (tri, [0.4, 0.3, -0.2])):
        cases.append({"verts": verts, "point": pt, "value": oracle.potential_integral(verts, pt)})
    out["wilton"] = cases
    return out


def main():
    doc = generate()
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
