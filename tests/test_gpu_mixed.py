"""Mixed-precision path: near-field apply on the tcgen05 TF32 tensor cores (or
FP32 CUDA cores, mixed_near=1) and FP32 far field with the tcgen05 TF32 M2L,
inside an FP64 iterative-refinement loop.

Bars: the FP32/TF32 operator apply is within 1e-3 (norm-wise, per column) of the FP64
operator (TF32 keeps 10 mantissa bits, rounded to nearest), also with the
M2L in the shared rank-64 basis (mixed_m2l 3, orders 5 and 6);
the refined Maxwell matrix is within 1e-6 of the plain FP64 solve, because
the refinement residual is the FP64 operator's."""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts
from tests.helpers import rel_max

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def window(nets=12, side=15.0, edge=0.3e-6):
    lay = layouts.routing_window(nets, side, seed=11)
    return _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                mesh_max_edge_m=edge, max_panels=-1)


@pytest.mark.parametrize("mixed_near", [0, 1, 2, 3])
@pytest.mark.parametrize("nrhs", [3, 64, 100])
def test_mixed_operator_close_to_fp64(ctx, nrhs, mixed_near):
    p = window()
    rng = np.random.default_rng(5)
    sig = rng.standard_normal((len(p["verts"]), nrhs))
    kw = dict(order=4, max_level=5, dense_below=-1, m2l_mode=1)
    y64, rep = ctx.operator_apply(p["verts"], sig, precision=0, **kw)
    y32, _ = ctx.operator_apply(p["verts"], sig, precision=1, mixed_near=mixed_near, **kw)
    assert rep["m2l_pairs"] > 0
    for j in range(nrhs):
        e = np.linalg.norm(y32[:, j] - y64[:, j]) / np.linalg.norm(y64[:, j])
        assert e < 1e-3, (j, e)


@pytest.mark.parametrize("order,m2l_mode,mixed_m2l,far_quad", [(4, 0, 0, 0), (4, 0, 0, 1), (4, 0, 1, 1), (5, 0, 0, 0),
                                                               (5, 0, 0, 1), (5, 1, 0, 0), (6, 0, 0, 1),
                                                               (5, 0, 3, 0), (5, 0, 3, 1), (5, 1, 3, 1),
                                                               (6, 0, 3, 1)])
def test_mixed_operator_close_to_fp64_high_order(ctx, order, m2l_mode, mixed_m2l, far_quad):
    """FP32 far field with the M2L on the tensor cores (orders 4-5, centroid
    sources) or in the factored low-rank form on the CUDA cores, against the
    FP64 operator with the same M2L operators.  The shared rank-64 basis
    (mixed_m2l 3) adds its compression error (about 1e-3 of the apply at
    orders 5 and 6) to the TF32 one."""
    p = window()
    rng = np.random.default_rng(5)
    sig = rng.standard_normal((len(p["verts"]), 64))
    kw = dict(order=order, max_level=5, dense_below=-1, far_quad=far_quad, m2l_mode=m2l_mode)
    y64, rep = ctx.operator_apply(p["verts"], sig, precision=0, **kw)
    y32, _ = ctx.operator_apply(p["verts"], sig, precision=1, mixed_m2l=mixed_m2l, **kw)
    assert rep["m2l_pairs"] > 0
    e = np.linalg.norm(y32 - y64, axis=0) / np.linalg.norm(y64, axis=0)
    assert e.max() < (2e-3 if mixed_m2l == 3 else 1e-3), e.max()


@pytest.mark.parametrize("order,far_quad,mixed_m2l,mixed_near", [(4, 1, 1, 2), (5, 0, 1, 2), (5, 1, 1, 2),
                                                                  (4, 1, 0, 0), (5, 0, 0, 0), (5, 1, 3, 0)])
def test_tensor_core_p2m_l2p_match_cuda_cores(ctx, order, far_quad, mixed_m2l, mixed_near):
    """The tensor-core P2M and L2P (weights, charges and local expansions split
    into TF32 hi and lo parts: products good to about 2^-21) against the FP32
    CUDA-core P2M and L2P (about 2^-24).  With a linear, FP32-accurate rest of
    the operator (factored FP32 M2L, near blocks split hi/lo) the two agree to
    5e-5, and the tensor-core operator stays within twice the CUDA-core one's
    distance from FP64 (with Gauss-point sources the large alternating source
    weights amplify both rounding levels alike).  A single-pass TF32 M2L
    rounds its inputs, so there both stay within the FP32 operator's bar
    against FP64 (centroid sources; with Gauss sources that M2L alone loses
    1e-2 on this window)."""
    p = window()
    rng = np.random.default_rng(6)
    sig = rng.standard_normal((len(p["verts"]), 64))
    kw = dict(order=order, max_level=5, dense_below=-1, far_quad=far_quad, precision=1, mixed_m2l=mixed_m2l,
              mixed_near=mixed_near)
    y0, _ = ctx.operator_apply(p["verts"], sig, **kw)
    y1, _ = ctx.operator_apply(p["verts"], sig, mixed_far_tc=1, **kw)
    y2, _ = ctx.operator_apply(p["verts"], sig, mixed_far_tc=2, **kw)  # P2M only
    y64, _ = ctx.operator_apply(p["verts"], sig, **dict(kw, precision=0, mixed_m2l=0, mixed_near=0))
    n64 = np.linalg.norm(y64, axis=0)
    d01 = np.linalg.norm(y1 - y0, axis=0) / np.linalg.norm(y0, axis=0)
    e0 = np.linalg.norm(y0 - y64, axis=0) / n64
    e1 = np.linalg.norm(y1 - y64, axis=0) / n64
    e2 = np.linalg.norm(y2 - y64, axis=0) / n64
    if mixed_m2l == 1:
        assert d01.max() < 5e-5, d01.max()
        assert e2.max() <= 2.0 * e0.max() + 1e-7, (e2.max(), e0.max())
        assert e1.max() <= 2.0 * e0.max() + 1e-7, (e1.max(), e0.max())
        assert e1.max() < 1e-4, e1.max()
    else:
        assert e1.max() < (2e-3 if mixed_m2l == 3 else 1e-3), e1.max()
        assert e2.max() < (2e-3 if mixed_m2l == 3 else 1e-3), e2.max()


def test_mixed_exact_m2l_needs_centroid_sources(ctx):
    p = window()
    with pytest.raises(_lib.GpxError) as ei:
        ctx.operator_apply(p["verts"], np.ones((len(p["verts"]), 4)), precision=1, order=4, max_level=5,
                           dense_below=-1, m2l_mode=1, far_quad=1)
    assert ei.value.status == 1 and "far_quad 0" in ei.value.message


@pytest.mark.parametrize("order,far_quad,mixed_near,mixed_m2l", [(4, 0, 0, 0), (4, 1, 0, 0), (4, 1, 1, 0),
                                                                 (5, 1, 0, 0), (5, 1, 0, 3), (6, 1, 0, 3),
                                                                 (5, 1, 2, 3)])
def test_mixed_solve_matches_fp64(ctx, order, far_quad, mixed_near, mixed_m2l):
    p = window()
    nc = len(p["nets"]) + 1
    kw = dict(order=order, max_level=5, dense_below=-1, far_quad=far_quad, skip_ground_rhs=1)
    C64, r64 = ctx.cap_solve(p["verts"], p["cond"], nc, precision=0, **kw)
    C32, r32 = ctx.cap_solve(p["verts"], p["cond"], nc, precision=1, mixed_near=mixed_near, mixed_m2l=mixed_m2l,
                             **kw)
    assert r32["converged"] == 1 and r32["outer_iterations"] >= 1
    assert r32["max_rel_residual"] <= 1e-8
    R = nc - 1
    d = np.abs(np.diag(C64[:R, :R]))
    err = np.abs(C32[:R, :R] - C64[:R, :R]) / d[:, None]
    assert err.max() < 1e-6, err.max()


def test_near_x_split_on_chip_matches_split_in_memory(ctx):
    """The TF32 near apply with X split before the apply (mixed_near 0) and
    with X gathered as FP32 and split on chip (mixed_near 3) compute the same
    products: the applies agree to FP32 rounding of X and accumulation order."""
    p = window()
    rng = np.random.default_rng(9)
    sig = rng.standard_normal((len(p["verts"]), 100))
    kw = dict(order=5, max_level=5, dense_below=-1, far_quad=1, precision=1, mixed_m2l=1)
    y0, _ = ctx.operator_apply(p["verts"], sig, mixed_near=0, **kw)
    y3, _ = ctx.operator_apply(p["verts"], sig, mixed_near=3, **kw)
    d = np.linalg.norm(y0 - y3, axis=0) / np.linalg.norm(y3, axis=0)
    assert d.max() < 1e-6, d.max()


def test_fp32_inner_basis_matches_fp64_basis(ctx):
    """The inner GMRES basis stored in FP32 (inner_basis32, for solves whose
    basis would not fit otherwise) against the default FP64 basis, with the
    TF32 near apply (inner tolerance floor 1e-3): both refinements meet the
    FP64 tolerance and give the same Maxwell matrix to well inside it."""
    p = window()
    nc = len(p["nets"]) + 1
    kw = dict(order=5, max_level=5, dense_below=-1, far_quad=1, skip_ground_rhs=1, precision=1, precond=1,
              mixed_near=0)
    C64, r64 = ctx.cap_solve(p["verts"], p["cond"], nc, **kw)
    C32, r32 = ctx.cap_solve(p["verts"], p["cond"], nc, inner_basis32=1, **kw)
    assert r32["converged"] == 1 and r64["converged"] == 1
    assert r32["max_rel_residual"] <= 1e-8
    R = nc - 1
    d = np.abs(np.diag(C64[:R, :R]))
    assert (np.abs(C32[:R, :R] - C64[:R, :R]) / d[:, None]).max() < 1e-7
    assert r32["iterations"] <= 1.25 * r64["iterations"] + 4, (r32["iterations"], r64["iterations"])


def test_mixed_two_wire_small_rhs(ctx):
    lay = layouts.two_wires()
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)
    C64, _ = ctx.cap_solve(p["verts"], p["cond"], 3, order=4, max_level=4)
    C32, rep = ctx.cap_solve(p["verts"], p["cond"], 3, order=4, max_level=4, precision=1)
    assert rep["converged"] == 1
    assert rel_max(C32, C64) < 1e-6


def test_refinement_stall_guard_recovers(ctx):
    """A small window whose substrate-plate panels are twice its depth-5 leaf
    size: the TF32 M2L forced with Gauss-point sources is far from the FP64
    operator there, the refinement stalls, and the stall guard continues with
    the factored FP32 M2L; the result matches the FP64 solve."""
    w = layouts.window_batch(93, seed=7)[92]
    p = _lib.bridge_panelize(w.store.arrays(), w.deck.layer_table(), 1.0, w.net_of_poly, mesh_max_edge_m=0.25e-6,
                             max_panels=-1)
    nc = len(p["nets"]) + 1
    kw = dict(order=5, max_level=5, dense_below=-1, far_quad=1, skip_ground_rhs=1, precond=1)
    C64, _ = ctx.cap_solve(p["verts"], p["cond"], nc, precision=0, **kw)
    C32, rep = ctx.cap_solve(p["verts"], p["cond"], nc, precision=1, mixed_m2l=2, **kw)
    assert rep["converged"] == 1
    R = nc - 1
    d = np.abs(np.diag(C64[:R, :R]))
    assert (np.abs(C32[:R, :R] - C64[:R, :R]) / d[:, None]).max() < 1e-6


def test_auto_depth_keeps_leaves_larger_than_panels(ctx):
    w = layouts.window_batch(93, seed=7)[92]
    p = _lib.bridge_panelize(w.store.arrays(), w.deck.layer_table(), 1.0, w.net_of_poly, mesh_max_edge_m=0.25e-6,
                             max_panels=-1)
    _, rep = ctx.cap_solve(p["verts"], p["cond"], len(p["nets"]) + 1, order=5, max_level=-1, dense_below=-1,
                           skip_ground_rhs=1, precision=1, mixed_m2l=2)
    assert rep["converged"] == 1 and rep["max_level"] <= 4
