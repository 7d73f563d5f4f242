"""Adjoint sensitivities dC/dp (gpx_cap_sensitivity) on the GPU.

Checks, on a three-bit met2 bus crossed by a met3 wire (the bus geometry of
the sensitivity workload, scaled down), for the width, spacing, thickness and
height parameters:
* the all-pairs (dense) adjoint against central finite differences of the
  GPU all-pairs solve on the displaced vertices (step 1e-3 relative);
* the same against central finite differences of the CPU oracle's dense LU
  solve (the FP64 dense-path reference gradient);
* the FMM-path adjoint against the all-pairs adjoint (FMM truncation only);
* the mixed-precision adjoint against the FP64 one;
* the per-net API: dC/dk = C / k and the capacitance equals the per-net
  extraction's."""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts, pex, sensitivity

pytestmark = pytest.mark.gpu

DENSE = dict(dense_below=2**31 - 1, skip_ground_rhs=0)


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def bus(edge):
    lay = layouts.bus_crossing(bits=3, wires=1, length_nm=6000, cross_pitch_nm=2000)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=edge, max_panels=-1)
    z0, z1 = sensitivity.layer_span(lay.deck, "met2")
    params = [("width", 1), ("spacing", 0), ("thickness", z0, z1), ("height", z0, z1)]
    steps = [0.2e-6, 0.2e-6, 0.85e-6, 1.4e-6]  # parameter values; FD step = 1e-3 x value
    V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
    return lay, p, params, steps, V


def fd(solve, verts, V, h):
    Cp = solve(verts + h * V)
    Cm = solve(verts - h * V)
    return (Cp - Cm) / (2 * h)


def test_dense_adjoint_matches_central_differences(ctx):
    lay, p, params, steps, V = bus(0.15e-6)
    nc = len(p["nets"]) + 1
    C, dC, rep = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, **DENSE)
    assert rep["dense"] == 1 and rep["converged"] == 1
    C0, _ = ctx.cap_solve(p["verts"], p["cond"], nc, **DENSE)
    assert np.abs(C - C0).max() <= 1e-12 * np.abs(C0).max()
    for q in range(len(params)):
        ref = fd(lambda v: ctx.cap_solve(v, p["cond"], nc, **DENSE)[0], p["verts"], V[q], 1e-3 * steps[q])
        err = np.abs(dC[q] - ref).max() / np.abs(ref).max()
        assert err < 1e-5, (params[q], err)


def test_dense_adjoint_matches_oracle_differences(ctx, orc):
    lay, p, params, steps, V = bus(0.0)
    nc = len(p["nets"]) + 1
    _, dC, _ = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, **DENSE)
    for q in (0, 1):
        ref = fd(lambda v: orc.cap_dense(v, p["cond"], nc), p["verts"], V[q], 1e-3 * steps[q])
        err = np.abs(dC[q] - ref).max() / np.abs(ref).max()
        assert err < 1e-5, (params[q], err)


@pytest.mark.parametrize("order", [4, 5])
def test_fmm_adjoint_tracks_dense_adjoint(ctx, order):
    lay, p, params, steps, V = bus(0.1e-6)
    nc = len(p["nets"]) + 1
    _, dD, _ = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, **DENSE)
    C, dF, rep = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, order=order, max_level=4, dense_below=-1,
                                     far_quad=1, precond=1, tol=1e-10)
    assert rep["dense"] == 0 and rep["m2l_pairs"] > 0
    bar = 5e-3 if order == 4 else 5e-4  # Chebyshev truncation of the far field and of its derivative
    for q in range(len(params)):
        err = np.abs(dF[q] - dD[q]).max() / np.abs(dD[q]).max()
        assert err < bar, (params[q], err)


def test_mixed_adjoint_matches_fp64(ctx):
    lay, p, params, steps, V = bus(0.1e-6)
    nc = len(p["nets"]) + 1
    kw = dict(order=5, max_level=4, dense_below=-1, precond=1, skip_ground_rhs=1)
    C64, d64, _ = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, precision=0, **kw)
    C32, d32, rep = ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, precision=1, **kw)
    assert rep["outer_iterations"] >= 2
    R = nc - 1
    assert np.isnan(d64[0, R, R]) and np.isnan(d64[0, 0, R])
    for q in range(len(params)):
        err = np.abs(d32[q, :R, :R] - d64[q, :R, :R]).max() / np.abs(d64[q, :R, :R]).max()
        assert err < 1e-6, (params[q], err)


def test_per_net_sensitivity_api(ctx):
    lay = layouts.bus_crossing(bits=3, wires=1, length_nm=6000, cross_pitch_nm=2000)
    z0, z1 = sensitivity.layer_span(lay.deck, "met2")
    params = [("width", 1), ("height", z0, z1), ("k",)]
    res = pex.run_pex_sensitivity_checked(lay.store, lay.deck, lay.net_of_poly, params, ctx=ctx, skip_ground_rhs=0)
    k = 3.9
    assert np.allclose(res.grad[("k",)] * k, res.maxwell_af, rtol=1e-14, atol=0)
    per_net = pex.run_pex_by_net_checked(lay.store, lay.deck, lay.net_of_poly, ctx=ctx)
    for i, net in enumerate(res.nets):
        assert abs(res.maxwell_af[i, i] - per_net[net].cap_af) <= 1e-9 * per_net[net].cap_af
    # widening a wire raises its own capacitance; moving the layer up lowers
    # the bus wires' coupling to the substrate
    assert res.grad[("width", 1)][1, 1] > 0
    assert res.grad[("height", z0, z1)][0, -1] > 0  # C_ij < 0 off-diagonal: weaker coupling -> less negative


def test_row_subset_and_chunked_columns(ctx, orc):
    """145 conductors (144 plates and no substrate split): forward columns and
    transposed rows both run in chunks of 128.  dC/dp for a few listed rows
    (gpx_cap_sensitivity_rows) equals those rows of the full computation and
    the central differences of the all-pairs solve; unlisted rows are NaN."""
    verts, cond = [], []
    for i in range(12):
        for j in range(12):
            v, c = orc.plate(i * 0.3, j * 0.3, 0.05 * ((i + j) % 3), 0.2, 0.2, 2, 2, 12 * i + j)
            verts.append(v)
            cond.append(c)
    verts, cond = np.vstack(verts), np.concatenate(cond)
    nc = 144
    # parameter: plate 17 lifted along z
    V = np.zeros((1,) + verts.shape)
    lift = cond == 17
    V[0, lift, 2::3] = 1.0
    kw = dict(dense_below=2**31 - 1, skip_ground_rhs=0)
    C, dC, rep = ctx.cap_sensitivity(verts, cond, nc, V, **kw)
    assert rep["n_rhs"] == 144 and rep["converged"] == 1
    rows = [5, 17, 130]
    Cs, dCs, _ = ctx.cap_sensitivity(verts, cond, nc, V, grad_rows=rows, **kw)
    assert np.array_equal(C, Cs)
    scale = np.abs(dC[0, rows]).max()
    assert np.abs(dCs[0, rows] - dC[0, rows]).max() <= 1e-10 * scale
    others = np.setdiff1d(np.arange(nc), rows)
    assert np.isnan(dCs[0, others]).all()
    h = 1e-3 * 0.05
    ref = fd(lambda v: ctx.cap_solve(v, cond, nc, **kw)[0], verts, V[0], h)
    err = np.abs(dCs[0, rows] - ref[rows]).max() / np.abs(ref[rows]).max()
    assert err < 1e-5, err
    with pytest.raises(_lib.GpxError, match="gradient row"):
        ctx.cap_sensitivity(verts, cond, nc, V, grad_rows=[5, 5], **kw)
