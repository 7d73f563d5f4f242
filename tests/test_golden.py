"""Golden fixtures of the field-solver path (tests/golden/field_solver.json,
made by tests/golden/make_golden.py from the CPU oracle).

CPU: the oracle still reproduces every fixture, and the product library's
host panelisation reproduces the fixture meshes bit for bit.
GPU: the CUDA path through the C ABI reproduces the fixtures at the parity
bars (Wilton 1e-12, operator apply 1e-11, dense-path Maxwell 1e-9, FMM-path
Maxwell 1e-6 = the reference's GMRES tolerance regime)."""
import hashlib
import json
import os

import numpy as np
import pytest

from gpurify_b200 import _lib, layouts
from tests.golden.make_golden import bridge_deck_layout

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "field_solver.json")))


def sha(verts):
    return hashlib.sha256(np.ascontiguousarray(verts, dtype="<f8").tobytes()).hexdigest()


def max_rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def two_wire_panels():
    lay = layouts.two_wires()
    return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)


# ---------------- CPU ----------------

def test_product_panelisation_matches_golden_meshes():
    g = GOLDEN["two_wires_reference_mesh"]
    p = two_wire_panels()
    assert len(p["verts"]) == g["n_panels"]
    assert np.bincount(p["cond"]).tolist() == g["panels_per_conductor"]
    assert sha(p["verts"]) == g["verts_sha256"]
    assert p["nets"].tolist() == g["nets"]
    st, deck, nets = bridge_deck_layout()
    p = _lib.bridge_panelize(st.arrays(), deck.layer_table(), 1.0, nets)
    assert sha(p["verts"]) == GOLDEN["bridge_deck_three_nets"]["verts_sha256"]


def test_oracle_reproduces_golden(orc):
    lay = layouts.two_wires()
    p = orc.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0)
    C, _ = orc.cap_fmm(p["verts"], p["cond"], 3, order=4, max_level=4, tol=1e-8)
    assert max_rel(C, GOLDEN["two_wires_reference_mesh"]["maxwell"]) < 1e-12
    g = GOLDEN["two_wires_operator_apply"]
    y, nnz = orc.fmm_cap_apply(p["verts"], np.array(g["sigma"]), 4, 4)
    assert nnz == g["nnz_near"]
    assert max_rel(y, g["y"]) < 1e-13
    st, deck, nets = bridge_deck_layout()
    p = orc.bridge_panelize(st.arrays(), deck.layer_table(), nets, 1.0)
    C = orc.cap_dense(p["verts"], p["cond"], 4)
    assert max_rel(C, GOLDEN["bridge_deck_three_nets"]["maxwell"]) < 1e-12
    for case in GOLDEN["wilton"]:
        v = orc.potential_integral(case["verts"], case["point"])
        assert abs(v - case["value"]) <= 1e-14 * abs(case["value"])


# ---------------- GPU ----------------

@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
def test_gpu_two_wire_maxwell_matches_golden(ctx):
    g = GOLDEN["two_wires_reference_mesh"]
    p = two_wire_panels()
    C, rep = ctx.cap_solve(p["verts"], p["cond"], 3, order=4, max_level=4, tol=1e-8)
    assert rep["dense"] == 0 and rep["converged"] == 1
    ref = np.array(g["maxwell"])
    assert (np.abs(C - ref) / np.abs(ref)).max() < 1e-6


@pytest.mark.gpu
def test_gpu_operator_apply_matches_golden(ctx):
    g = GOLDEN["two_wires_operator_apply"]
    p = two_wire_panels()
    y, rep = ctx.operator_apply(p["verts"], np.array(g["sigma"]), order=4, max_level=4, dense_below=-1)
    assert rep["nnz_near"] == g["nnz_near"]
    assert np.linalg.norm(y[:, 0] - g["y"]) / np.linalg.norm(g["y"]) < 1e-11


@pytest.mark.gpu
def test_gpu_per_net_capacitance_matches_golden(ctx):
    from gpurify_b200 import pex

    g = GOLDEN["bridge_deck_three_nets"]
    st, deck, nets = bridge_deck_layout()
    out = pex.run_pex_by_net_checked(st, deck, nets, ctx=ctx)
    assert sorted(out) == g["nets"]
    for net, af in zip(g["nets"], g["cap_af"]):
        assert abs(out[net].cap_af - af) <= 1e-9 * af


@pytest.mark.gpu
def test_gpu_sphere_plates_wilton_match_golden(ctx, orc):
    v, c = orc.icosphere([0, 0, 0], 1.0, 2, 0)
    C, _ = ctx.cap_solve(v, c, 1)
    assert max_rel(C, GOLDEN["sphere_320"]["maxwell"]) < 1e-9
    a, ca = orc.plate(0, 0, 0, 0.2, 0.2, 10, 10, 0)
    b, cb = orc.plate(0, 0, 0.02, 0.2, 0.2, 10, 10, 1)
    C, _ = ctx.cap_solve(np.vstack([a, b]), np.concatenate([ca, cb]), 2)
    assert max_rel(C, GOLDEN["plates_10x10"]["maxwell"]) < 1e-9
    coef = 1.0 / (4.0 * np.pi * 8.854187812800e-12)
    for case in GOLDEN["wilton"]:
        vq = np.array(case["verts"], dtype=np.float64).reshape(1, 12)
        got = ctx.potential_matrix(vq, np.array([case["point"]]))[0, 0]
        assert abs(got - coef * case["value"]) <= 1e-12 * abs(coef * case["value"])
