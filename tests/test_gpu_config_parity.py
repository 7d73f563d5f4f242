"""GPU parity against the CPU oracle on the benchmark configurations' own
geometries (fixtures in tests/golden/config_parity.json, made by
tests/golden/make_config_golden.py).

* A config-2-style routing window (16 nets, 6,079 panels):
  - the FP64 GPU path in the reference's mode (order 4, depth 4, centroid
    sources, diagonal Jacobi, cap/fmm_solver.rs:147-172) against the
    oracle's FMM solve: every coupled entry within 1e-6 of itself;
  - the FP64 and the mixed GPU paths against the oracle's dense LU
    (cap/solver.rs:100-134, the FP64 dense-direct reference).  With the
    benchmark's options (order 5, 2x2 Gauss far-field sources, leaf
    block-Jacobi; mixed: TF32 tensor cores inside FP64 refinement): every
    entry within 1e-4 of its row's diagonal, and the entries of at least a
    tenth of their diagonal within 1e-3 of themselves.  With order 6 at
    depth 3: every entry within 2e-5 of its diagonal and every entry of at
    least 3 % of its diagonal within 1e-4 of itself.  The entry-wise error
    is the far field's discretisation error (the same in FP64 and mixed);
    smaller couplings carry the same absolute error, a larger share of them.
* The benchmark's 64-net window at full size (69,253 panels), reference mode
  at depth 5, against the oracle's FMM on 4 conductor columns spread over the
  window: 1e-6.
* The config-4 bus at full size (42,588 panels): the FP64 FMM adjoint
  dC/d(width), dC/d(spacing) against the oracle's central differences
  (relative step 1e-3), columns 3 and 4.

"Coupled" entries are those with |C_ij| >= 1e-3 |C_ii|; below that an
entry's own relative error measures the solver tolerance, not the operator.
"""
import json
import os

import numpy as np
import pytest

from gpurify_b200 import _lib, layouts, sensitivity
from tests.golden import make_config_golden as mk

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_parity.json")))


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def product_panelize(lay, edge):
    return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                mesh_max_edge_m=edge, max_panels=-1)


def errors(C, ref, coupling=1e-3):
    """(max |dC_ij| / |ref_ii|, max |dC_ij| / |ref_ij| over the entries with
    |ref_ij| >= coupling |ref_ii|)."""
    C, ref = np.asarray(C), np.asarray(ref)
    d = np.abs(np.diag(ref))[:, None]
    err = np.abs(C - ref)
    coupled = np.abs(ref) >= coupling * d
    return float((err / d).max()), float((err / np.abs(ref))[coupled].max())


REF_MODE = dict(order=4, max_level=4, far_quad=0, precond=0, m2l_mode=0, precision=_lib.PREC_FP64,
                dense_below=-1)
HEADLINE = dict(order=5, max_level=-1, far_quad=1, m2l_mode=0, mixed_m2l=2, dense_below=-1, tol=1e-8)


def test_window16_reference_mode_matches_oracle_fmm(ctx):
    g = GOLD["window16"]
    p = mk.window16_panels(product_panelize)
    assert mk.verts_sha256(p["verts"]) == g["verts_sha256"]
    nc = len(p["nets"]) + 1
    C, rep = ctx.cap_solve(p["verts"], p["cond"], nc, tol=1e-10, **REF_MODE)
    assert rep["converged"] and not rep["dense"]
    diag, coupled = errors(C, g["maxwell_fmm_ref"])
    assert diag < 1e-7, diag
    assert coupled < 1e-6, coupled


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("accuracy", ["bench", "order6"])
def test_window16_matches_oracle_dense(ctx, prec, accuracy):
    g = GOLD["window16"]
    p = mk.window16_panels(product_panelize)
    nc = len(p["nets"]) + 1
    kw = dict(HEADLINE, precision=_lib.PREC_MIXED if prec == "mixed" else _lib.PREC_FP64,
              precond=1 if prec == "mixed" else 2)
    if accuracy == "order6":
        kw.update(order=6, max_level=3, mixed_m2l=3)
    C, rep = ctx.cap_solve(p["verts"], p["cond"], nc, **kw)
    assert rep["converged"] and not rep["dense"]
    R = nc - 1
    ref = np.asarray(g["maxwell_dense"])[:R, :R]
    if accuracy == "bench":
        diag, strong = errors(C[:R, :R], ref, coupling=0.1)
        assert diag < 1e-4, diag
        assert strong < 1e-3, strong
    else:
        diag, coupled = errors(C[:R, :R], ref, coupling=0.03)
        assert diag < 2e-5, diag
        assert coupled < 1e-4, coupled


def test_window64_reference_mode_matches_oracle_columns(ctx):
    g = GOLD["window64"]
    p = mk.window64_panels(product_panelize)
    assert mk.verts_sha256(p["verts"]) == g["verts_sha256"]
    nc = len(p["nets"]) + 1
    C, rep = ctx.cap_solve(p["verts"], p["cond"], nc, tol=1e-10, skip_ground_rhs=1,
                           **dict(REF_MODE, max_level=g["depth"]))
    assert rep["converged"]
    R = nc - 1
    for j, col in zip(g["columns"], g["maxwell_columns"]):
        ref = np.asarray(col)[:R]
        got = C[:R, j]
        d = abs(ref[j])
        coupled = np.abs(ref) >= 1e-3 * d
        assert np.abs(got - ref).max() / d < 1e-7, j
        assert (np.abs(got - ref) / np.abs(ref))[coupled].max() < 1e-6, j


def test_bus_adjoint_matches_oracle_central_differences(ctx):
    g = GOLD["bus"]
    lay, p = mk.bus_panels(product_panelize)
    assert mk.verts_sha256(p["verts"]) == g["verts_sha256"]
    nc = len(p["nets"]) + 1
    params = [tuple(f["param"]) for f in g["fd"]]
    V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
    C, dC, rep = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, order=g["order"], max_level=g["depth"],
                                     far_quad=0, precond=2, tol=1e-10, dense_below=-1, skip_ground_rhs=1,
                                     precision=_lib.PREC_FP64)
    R = nc - 1
    for q, f in enumerate(g["fd"]):
        for j, col in zip(g["columns"], f["dC_columns"]):
            ref = np.asarray(col)[:R]
            got = dC[q, :R, j]
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 2e-3, (f["param"], j, err)
