"""CPU oracle for the field-solver capacitance path — TEST INFRASTRUCTURE ONLY.

ctypes view of ``oracle/liboracle.so`` (built from ``oracle/orc.cpp`` by
``oracle/Makefile``), a plain C++ restatement of the reference's CPU field
solver.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` may import this module, and only as the checker: the product
library (``gpurify_b200``) never imports or links it.

Parity pinning: the reference ships no field-solver golden numbers; the oracle
is pinned by re-running the reference's own known-answer tests against it
(crates/pex/tests/analytic.rs, cap_validation.rs, fmm.rs, fmm_cap.rs,
bridge.rs) in ``tests/test_oracle_pins.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

EPS0 = 8.854187812800e-12
AF_PER_F = 1.0e18


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O2 -fopenmp -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(
        os.path.getmtime(os.path.join(_HERE, f)) for f in ("orc.cpp", "orc.h")
    ):
        env = dict(os.environ)
        env.pop("CXX", None)
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"], check=True, env=env)
    return _LIB_PATH


class LayerParams(C.Structure):
    _fields_ = [
        ("layer", C.c_uint16),
        ("sheet_res_ohm_sq", C.c_double),
        ("area_cap_af_um2", C.c_double),
        ("fringe_cap_af_um", C.c_double),
        ("coupling_cap_af_um", C.c_double),
        ("interlayer_cap_af_um2", C.c_double),
        ("via_res_ohm", C.c_double),
        ("thickness_nm", C.c_double),
        ("height_nm", C.c_double),
        ("dielectric_k", C.c_double),
    ]


class FmmOpts(C.Structure):
    _fields_ = [
        ("order", C.c_int32),
        ("max_level", C.c_int32),
        ("restart", C.c_int32),
        ("max_restarts", C.c_int32),
        ("tol", C.c_double),
        ("threads", C.c_int32),
        ("rhs_limit", C.c_int32),
        ("rhs_stride", C.c_int32),
    ]


class FmmReport(C.Structure):
    _fields_ = [
        ("total_iterations", C.c_int64),
        ("max_iterations", C.c_int64),
        ("max_residual", C.c_double),
        ("all_converged", C.c_int32),
        ("nnz_near", C.c_int64),
        ("n_boxes", C.c_int64),
        ("t_setup_s", C.c_double),
        ("t_solve_s", C.c_double),
    ]


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        L = _lib
        L.orc_potential_integral.restype = C.c_double
        L.orc_dot.restype = C.c_double
        for name in ("orc_plate", "orc_icosphere", "orc_decompose_rectilinear", "orc_bridge_panelize"):
            getattr(L, name).restype = C.c_int64
        L.orc_plate.argtypes = [C.c_double] * 5 + [C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_icosphere.argtypes = [C.c_double] * 4 + [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_bridge_panelize.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                          C.c_int64, C.c_double, C.c_double, C.c_int64, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_char_p, C.c_int64]
        L.orc_cap_dense.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        L.orc_cap_dense_gmres.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        L.orc_cap_dense_eps.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_cap_fmm.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(FmmOpts), C.c_void_p,
                                  C.POINTER(FmmReport)]
        L.orc_fmm_new.restype = C.c_void_p
        L.orc_fmm_new.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                  C.POINTER(C.c_double)]
        L.orc_fmm_solve_column.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_void_p,
                                           C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.orc_fmm_free.argtypes = [C.c_void_p]
        L.orc_fmm_free.restype = None
        L.orc_dense_P.argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
        L.orc_fmm_point_matvec.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_void_p]
        L.orc_fmm_cap_apply.argtypes = [C.c_int64, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_int64)]
        L.orc_m2l_table.argtypes = [C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_dot.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    return _lib


# ---------------------------------------------------------------- geometry
def potential_integral(verts, p) -> float:
    """Wilton integral of 1/|p - r'| over one panel (integrals/panel.rs:147-208).

    ``verts`` is (3|4, 3); a triangle is padded by repeating its last vertex."""
    v = quad(verts)
    p = np.ascontiguousarray(p, dtype=np.float64)
    return lib().orc_potential_integral(_p(v), _p(p))


def quad(verts) -> np.ndarray:
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
    if v.shape[0] == 3:
        v = np.vstack([v, v[2:3]])
    return np.ascontiguousarray(v.reshape(12))


def panel_props(verts12):
    c = np.zeros(3)
    a = C.c_double()
    n = np.zeros(3)
    v = np.ascontiguousarray(verts12, dtype=np.float64)
    lib().orc_panel_props(_p(v), _p(c), C.byref(a), _p(n))
    return c, a.value, n


def plate(cx, cy, z0, lx, ly, nx, ny, conductor):
    """cap/mesh.rs:12-43 -> (verts (n,12), cond (n,))."""
    cap = nx * ny
    v = np.zeros((cap, 12))
    c = np.zeros(cap, dtype=np.int32)
    n = lib().orc_plate(cx, cy, z0, lx, ly, nx, ny, conductor, v.ctypes.data, c.ctypes.data, cap)
    return v[:n], c[:n]


def icosphere(center, r, subdivisions, conductor):
    """cap/mesh.rs:48-114 -> (verts (n,12), cond (n,))."""
    cap = 20 * 4 ** subdivisions
    v = np.zeros((cap, 12))
    c = np.zeros(cap, dtype=np.int32)
    n = lib().orc_icosphere(center[0], center[1], center[2], r, subdivisions, conductor, v.ctypes.data,
                            c.ctypes.data, cap)
    return v[:n], c[:n]


def decompose_rectilinear(xs, ys):
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    cap = max(4 * len(xs), 16)
    out = np.zeros((cap, 4), dtype=np.int32)
    n = lib().orc_decompose_rectilinear(_p(xs, C.c_int32), _p(ys, C.c_int32), len(xs), _p(out, C.c_int32), cap)
    if n < 0:
        raise ValueError(f"decompose error {n}")
    return out[:n]


class OracleBridgeError(Exception):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def bridge_panelize(store, layers, net_of_poly, dbu_nm, mesh_max_edge_m=0.0, max_panels=0, cap=None):
    """bridge.rs panelisation.  ``store`` has verts_x, verts_y, poly_vert_start,
    poly_vert_len, poly_layer arrays; ``layers`` is a list of dicts of PEX layer
    params.  Returns dict(verts, cond, eps, nets, via_r)."""
    vx = np.ascontiguousarray(store["verts_x"], dtype=np.int32)
    vy = np.ascontiguousarray(store["verts_y"], dtype=np.int32)
    ps = np.ascontiguousarray(store["poly_vert_start"], dtype=np.uint32)
    pl = np.ascontiguousarray(store["poly_vert_len"], dtype=np.uint32)
    ly = np.ascontiguousarray(store["poly_layer"], dtype=np.uint16)
    nop = np.ascontiguousarray(net_of_poly, dtype=np.uint32)
    arr = (LayerParams * max(1, len(layers)))()
    for i, d in enumerate(layers):
        for k, _ in LayerParams._fields_:
            setattr(arr[i], k, d.get(k, 0))
    if cap is None:
        cap = 4_000_000
    verts = np.zeros((cap, 12))
    cond = np.zeros(cap, dtype=np.int32)
    eps = np.zeros(cap)
    nets = np.zeros(len(nop) + 1, dtype=np.uint32)
    via_r = np.zeros(len(nop) + 1)
    nn = C.c_int64()
    err = C.create_string_buffer(512)
    n = lib().orc_bridge_panelize(vx.ctypes.data, vy.ctypes.data, ps.ctypes.data, pl.ctypes.data, ly.ctypes.data,
                                  len(ps), nop.ctypes.data, len(nop), C.cast(arr, C.c_void_p), len(layers), dbu_nm,
                                  mesh_max_edge_m, max_panels, verts.ctypes.data, cond.ctypes.data,
                                  eps.ctypes.data, cap, nets.ctypes.data, C.byref(nn), via_r.ctypes.data, err, 512)
    if n < 0:
        raise OracleBridgeError(int(n), err.value.decode())
    return dict(verts=verts[:n].copy(), cond=cond[:n].copy(), eps=eps[:n].copy(),
                nets=nets[: nn.value].copy(), via_r=via_r[: nn.value].copy())


# ---------------------------------------------------------------- solvers
def _prep(verts, cond):
    v = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 12))
    c = np.ascontiguousarray(np.asarray(cond, dtype=np.int32))
    return v, c


def cap_dense(verts, cond, ncond) -> np.ndarray:
    """cap::solve(Method::Direct): dense Wilton P + LU (cap/solver.rs:100-134)."""
    v, c = _prep(verts, cond)
    C_ = np.zeros((ncond, ncond))
    rc = lib().orc_cap_dense(len(v), v.ctypes.data, c.ctypes.data, ncond, C_.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_cap_dense rc={rc}")
    return C_


def cap_dense_eps(verts, cond, ncond, eps) -> np.ndarray:
    """The bridge's solve for a stack of several k (bridge.rs:409-430 ->
    cap/dielectric.rs:76-150, conductor roles only): dense Wilton P + LU, each
    panel's charge weighted by its surrounding permittivity ``eps`` (per panel,
    caller order).  Already k-scaled: no further multiplication by k."""
    v, c = _prep(verts, cond)
    e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
    if e.shape != (len(v),):
        raise ValueError("eps needs one value per panel")
    C_ = np.zeros((ncond, ncond))
    rc = lib().orc_cap_dense_eps(len(v), v.ctypes.data, c.ctypes.data, ncond, e.ctypes.data, C_.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_cap_dense_eps rc={rc}")
    return C_


def cap_dense_gmres(verts, cond, ncond) -> np.ndarray:
    v, c = _prep(verts, cond)
    C_ = np.zeros((ncond, ncond))
    rc = lib().orc_cap_dense_gmres(len(v), v.ctypes.data, c.ctypes.data, ncond, C_.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_cap_dense_gmres rc={rc}")
    return C_


def cap_fmm(verts, cond, ncond, order=4, max_level=4, tol=1e-8, restart=200, max_restarts=50, threads=0,
            rhs_limit=0, rhs_stride=1):
    """cap::fmm_solver::solve (cap/fmm_solver.rs:147-172). Returns (C, report dict).
    ``rhs_limit`` > 0 solves only that many conductors (bounded CPU samples):
    conductors 0, rhs_stride, 2 rhs_stride, ...; the other columns stay zero."""
    v, c = _prep(verts, cond)
    C_ = np.zeros((ncond, ncond))
    o = FmmOpts(order, max_level, restart, max_restarts, tol, threads, rhs_limit, rhs_stride)
    r = FmmReport()
    rc = lib().orc_cap_fmm(len(v), v.ctypes.data, c.ctypes.data, ncond, C.byref(o), C_.ctypes.data, C.byref(r))
    if rc != 0:
        raise RuntimeError(f"orc_cap_fmm rc={rc}")
    rep = {k: getattr(r, k) for k, _ in FmmReport._fields_}
    return C_, rep


class FmmSolver:
    """cap::fmm_solver::solve in steps (cap/fmm_solver.rs:147-172): the
    operator and Jacobi preconditioner are built once (``t_setup_s``), then
    ``solve_column(j)`` runs one conductor's GMRES and returns column j of the
    Maxwell matrix with its iteration count."""

    def __init__(self, verts, cond, ncond, order=4, max_level=4, threads=0):
        v, c = _prep(verts, cond)
        self._keep = (v, c)
        self.ncond = ncond
        t = C.c_double()
        self.h = lib().orc_fmm_new(len(v), v.ctypes.data, c.ctypes.data, ncond, order, max_level, threads,
                                   C.byref(t))
        if not self.h:
            raise RuntimeError("orc_fmm_new failed")
        self.t_setup_s = t.value

    def solve_column(self, j, tol=1e-8, restart=200, max_restarts=50):
        col = np.zeros(self.ncond)
        its, res = C.c_int64(), C.c_double()
        rc = lib().orc_fmm_solve_column(self.h, j, tol, restart, max_restarts, col.ctypes.data, C.byref(its),
                                        C.byref(res))
        if rc < 0:
            raise RuntimeError(f"orc_fmm_solve_column rc={rc}")
        return col, {"iterations": its.value, "residual": res.value, "converged": rc == 0}

    def close(self):
        if self.h:
            lib().orc_fmm_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dense_P(verts) -> np.ndarray:
    v = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 12))
    P = np.zeros((len(v), len(v)))
    lib().orc_dense_P(len(v), v.ctypes.data, P.ctypes.data)
    return P


def fmm_point_matvec(pts, q, order, max_level, with_p2p=True) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    y = np.zeros(len(q))
    lib().orc_fmm_point_matvec(len(q), pts.ctypes.data, q.ctypes.data, order, max_level, int(with_p2p),
                               y.ctypes.data)
    return y


def fmm_cap_apply(verts, sigma, order=4, max_level=4):
    """FmmCapOperator::apply (cap/fmm_solver.rs:109-129) -> (y, nnz)."""
    v = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 12))
    s = np.ascontiguousarray(sigma, dtype=np.float64)
    y = np.zeros(len(v))
    nnz = C.c_int64()
    lib().orc_fmm_cap_apply(len(v), v.ctypes.data, order, max_level, s.ctypes.data, y.ctypes.data, C.byref(nnz))
    return y, nnz.value


def m2l_table(order):
    n3 = order ** 3
    K = np.zeros((343, n3, n3))
    rank = np.zeros(343, dtype=np.int32)
    lib().orc_m2l_table(order, K.ctypes.data, rank.ctypes.data)
    return K, rank


def dot(a, b) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib().orc_dot(a.ctypes.data, b.ctypes.data, len(a))
