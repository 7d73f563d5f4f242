"""Pins the CPU oracle against the reference's own known-answer tests for the
field-solver path (the reference ships no field-solver golden numbers):
crates/pex/tests/analytic.rs:14-71, cap_validation.rs:9-90, fmm.rs:37-60,
fmm_cap.rs:7-27 and the in-module tests fmm/chebyshev.rs:108-155,
fmm/tree.rs:228-274 (through the oracle's point FMM)."""
import math

import numpy as np
import pytest

FOUR_PI_EPS0 = 4.0 * math.pi * 8.854187812800e-12
SQUARE = [[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.5, 0.5, 0.0], [-0.5, 0.5, 0.0]]


def lcg_points(n, seed):
    """tests/fmm.rs:17-24 point generator (64-bit LCG, top 31 bits)."""
    s = seed
    out = []
    mask = (1 << 64) - 1
    for _ in range(3 * n):
        s = (s * 6364136223846793005 + 1442695040888963407) & mask
        out.append((s >> 33) / float(1 << 31) - 1.0)
    return np.array(out).reshape(n, 3)


def dense_matvec(pts, q):
    d = pts[:, None, :] - pts[None, :, :]
    r = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    return (q[None, :] / r).sum(1)


def rel_err(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_wilton_unit_square_self_integral(orc):
    got = orc.potential_integral(SQUARE, [0, 0, 0])
    exact = 4.0 * math.asinh(1.0)
    assert abs(got - exact) <= 1e-12 * exact


def test_wilton_far_field_is_monopole(orc):
    got = orc.potential_integral(SQUARE, [0, 0, 50.0])
    assert abs(got - 1 / 50.0) <= 1e-3 / 50.0


def test_wilton_offplane_matches_quadrature(orc):
    verts = [[0, 0, 0], [1, 0, 0], [1, 0.7, 0], [0, 0.7, 0]]
    p = np.array([0.3, 0.2, 0.4])
    got = orc.potential_integral(verts, p)
    nx, ny = 400, 280
    dx, dy = 1.0 / nx, 0.7 / ny
    X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dy, indexing="ij")
    q = (dx * dy / np.sqrt((X - p[0]) ** 2 + (Y - p[1]) ** 2 + p[2] ** 2)).sum()
    assert abs(got - q) <= 5e-4 * q


def test_triangle_padding_is_exact(orc):
    tri = [[0, 0, 0], [1, 0, 0], [0.2, 0.9, 0]]
    c, a, n = orc.panel_props(orc.quad(tri))
    assert a == pytest.approx(0.45, rel=1e-15)
    assert np.allclose(c, [(0 + 1 + 0.2) / 3, 0.3, 0.0], rtol=0, atol=1e-15)


def test_isolated_sphere_self_capacitance(orc):
    v, c = orc.icosphere([0, 0, 0], 1.0, 2, 0)
    assert len(v) == 320
    C = orc.cap_dense(v, c, 1)
    assert abs(C[0, 0] - FOUR_PI_EPS0) / FOUR_PI_EPS0 < 0.03


def test_sphere_converges_with_refinement(orc):
    errs = []
    for sub in (1, 2):
        v, c = orc.icosphere([0, 0, 0], 1.0, sub, 0)
        errs.append(abs(orc.cap_dense(v, c, 1)[0, 0] - FOUR_PI_EPS0) / FOUR_PI_EPS0)
    assert errs[1] < errs[0]


def test_parallel_plate_capacitor(orc):
    a, ca = orc.plate(0, 0, 0, 0.2, 0.2, 10, 10, 0)
    b, cb = orc.plate(0, 0, 0.02, 0.2, 0.2, 10, 10, 1)
    C = orc.cap_dense(np.vstack([a, b]), np.concatenate([ca, cb]), 2)
    ideal = 8.854187812800e-12 * 0.04 / 0.02
    ratio = abs(C[0, 1]) / ideal
    assert 0.95 < ratio < 1.35
    assert abs(C[0, 1] - C[1, 0]) / abs(C[0, 1]) < 1e-6
    assert C[0, 1] < 0 and C[0, 0] > 0


def test_direct_and_iterative_agree(orc):
    v, c = orc.icosphere([0, 0, 0], 1.0, 1, 0)
    cd = orc.cap_dense(v, c, 1)[0, 0]
    ci = orc.cap_dense_gmres(v, c, 1)[0, 0]
    assert abs(cd - ci) / abs(cd) < 1e-6


def test_fmm_capacitance_matches_dense_and_analytic(orc):
    v, c = orc.icosphere([0, 0, 0], 1.0, 2, 0)
    cd = orc.cap_dense(v, c, 1)[0, 0]
    cf, rep = orc.cap_fmm(v, c, 1, order=4, max_level=3, tol=1e-8)
    assert rep["all_converged"] == 1
    assert abs(cf[0, 0] - cd) / cd < 5e-3
    assert abs(cf[0, 0] - FOUR_PI_EPS0) / FOUR_PI_EPS0 < 0.03


def test_fmm_matvec_matches_dense(orc):
    pts = lcg_points(900, 12345)
    q = np.array([(i % 13) - 6.0 for i in range(900)])
    e = rel_err(orc.fmm_point_matvec(pts, q, 5, 3), dense_matvec(pts, q))
    assert e < 1e-3


def test_fmm_converges_with_chebyshev_order(orc):
    pts = lcg_points(800, 999)
    q = np.array([(i * 7 % 11) - 5.0 for i in range(800)])
    ex = dense_matvec(pts, q)
    e3 = rel_err(orc.fmm_point_matvec(pts, q, 3, 3), ex)
    e5 = rel_err(orc.fmm_point_matvec(pts, q, 5, 3), ex)
    assert e5 < e3 and e5 < 1e-4


def test_dot_matches_scalar(orc):
    """simd.rs:214-227: the 16-lane dot agrees with the scalar loop to 1e-13."""
    rng = np.random.default_rng(3)
    for n in (0, 1, 5, 16, 17, 100, 1003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        s = float(sum(x * y for x, y in zip(a, b)))
        assert abs(orc.dot(a, b) - s) <= 1e-13 * max(1.0, abs(s))


def test_m2l_compression_rank_and_error(orc):
    """bbfmm.rs:147-150: compression eps tracks the order; the truncated
    operator stays close to the exact Chebyshev kernel matrix."""
    K, rank = orc.m2l_table(4)
    built = rank >= 0
    assert built.sum() == 316
    assert (rank[built] > 0).all() and (rank[built] <= 64).all()
    roots = np.cos((2 * np.arange(4) + 1) * np.pi / 8)
    ref = np.array([[a, b, c] for a in roots for b in roots for c in roots])
    slot = ((2 + 3) * 7 + 0 + 3) * 7 + 0 + 3
    G = 1.0 / np.linalg.norm(ref[:, None, :] - ref[None, :, :] - np.array([4.0, 0, 0]), axis=-1)
    assert np.abs(K[slot] - G).max() / np.abs(G).max() < 1e-3
