"""ctypes binding of the in-tree CUDA library ``libgpx_pex.so`` (C ABI in
``include/gpx_pex.h``).  The product path always goes through this library:
if it cannot be loaded, every call raises — there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpx_pex.so")

GPX_OK = 0
STATUS = {
    0: "GPX_OK", 1: "GPX_ERR_INVALID_ARG", 2: "GPX_ERR_CUDA", 3: "GPX_ERR_NO_DEVICE",
    10: "GPX_ERR_INVALID_DBU", 11: "GPX_ERR_INVALID_PROCESS", 12: "GPX_ERR_UNSUPPORTED_GEOMETRY",
    13: "GPX_ERR_GRID_CAPACITY", 14: "GPX_ERR_PANEL_CAPACITY", 15: "GPX_ERR_CAPACITANCE",
    16: "GPX_ERR_NON_FINITE", 20: "GPX_ERR_OUTPUT_CAPACITY", 21: "GPX_ERR_OUT_OF_MEMORY",
    22: "GPX_ERR_INTERNAL",
}
PREC_FP64, PREC_MIXED = 0, 1
M2L_COMPRESSED, M2L_EXACT = 0, 1

# Every symbol include/gpx_pex.h declares.
EXPORTS = (
    "gpx_ctx_create", "gpx_ctx_destroy", "gpx_last_error", "gpx_version", "gpx_cap_solve",
    "gpx_cap_solve_batched", "gpx_operator_apply", "gpx_potential_matrix", "gpx_cap_solve_groups",
    "gpx_extract_quasistatic", "gpx_bridge_panelize", "gpx_plan_check", "gpx_ctx_stream",
    "gpx_ctx_set_profiling", "gpx_ctx_kernel_stats", "gpx_ctx_reset_stats", "gpx_cap_solve_small_static",
    "gpx_cap_sensitivity", "gpx_cap_sensitivity_rows", "gpx_autotune", "gpx_cap_solve_eps",
)
KERNEL_CLASSES = ("near_assemble", "near_apply", "p2m", "m2m", "m2l", "l2l", "l2p", "gs_dot", "gs_axpy", "vec",
                  "small", "near_apply_f64", "p2m_f64", "m2m_f64", "m2l_f64", "l2l_f64", "l2p_f64")


class GpxError(RuntimeError):
    def __init__(self, status: int, message: str, polygon: int = 0xFFFFFFFF):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message
        self.polygon = polygon


class SolveOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("order", C.c_int32), ("max_level", C.c_int32), ("m2l_mode", C.c_int32),
        ("tol", C.c_double), ("restart", C.c_int32), ("max_restarts", C.c_int32), ("dense_below", C.c_int32),
        ("precond", C.c_int32), ("skip_ground_rhs", C.c_int32), ("inner_tol_exp", C.c_int32),
        ("mesh_max_edge_m", C.c_double), ("max_panels", C.c_int64), ("far_quad", C.c_int32),
        ("mixed_near", C.c_int32), ("mixed_m2l", C.c_int32), ("no_graphs", C.c_int32), ("batch_streams", C.c_int32),
        ("col_begin", C.c_int32), ("col_count", C.c_int32), ("mixed_far_tc", C.c_int32),
        ("inner_basis32", C.c_int32), ("reserved", C.c_int32),
    ]


class SolveReport(C.Structure):
    _fields_ = [
        ("n_panels", C.c_int64), ("n_conductors", C.c_int32), ("n_rhs", C.c_int32), ("order", C.c_int32),
        ("max_level", C.c_int32), ("n_boxes", C.c_int64), ("n_leaves", C.c_int64), ("nnz_near", C.c_int64),
        ("m2l_pairs", C.c_int64), ("iterations", C.c_int32), ("outer_iterations", C.c_int32),
        ("operator_applies", C.c_int64), ("max_rel_residual", C.c_double), ("converged", C.c_int32),
        ("dense", C.c_int32), ("t_panelize_s", C.c_double), ("t_setup_s", C.c_double), ("t_solve_s", C.c_double),
        ("t_total_s", C.c_double), ("t_near_assembly_s", C.c_double), ("kernel_launches", C.c_int64),
        ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("restart_used", C.c_int32), ("reserved", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneReport(C.Structure):
    _fields_ = [("est_rel_err", C.c_double), ("apply_ms", C.c_double), ("setup_ms", C.c_double),
                ("candidates", C.c_int32), ("from_cache", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PanelProblem(C.Structure):
    _fields_ = [("n_panels", C.c_int64), ("verts", C.c_void_p), ("conductor", C.c_void_p),
                ("n_conductors", C.c_int32)]


class VolumeGroup(C.Structure):
    _fields_ = [("net", C.c_uint32), ("z0_m", C.c_double), ("z1_m", C.c_double), ("dielectric_k", C.c_double),
                ("rect_offset", C.c_int64), ("rect_count", C.c_int64)]


class GeometryStoreC(C.Structure):
    _fields_ = [("verts_x", C.c_void_p), ("verts_y", C.c_void_p), ("poly_vert_start", C.c_void_p),
                ("poly_vert_len", C.c_void_p), ("poly_layer", C.c_void_p), ("n_poly", C.c_int64)]


class LayerParamsC(C.Structure):
    _fields_ = [("layer", C.c_uint16), ("sheet_res_ohm_sq", C.c_double), ("area_cap_af_um2", C.c_double),
                ("fringe_cap_af_um", C.c_double), ("coupling_cap_af_um", C.c_double),
                ("interlayer_cap_af_um2", C.c_double), ("via_res_ohm", C.c_double), ("thickness_nm", C.c_double),
                ("height_nm", C.c_double), ("dielectric_k", C.c_double)]


class DeckC(C.Structure):
    _fields_ = [("layers", C.c_void_p), ("n_layers", C.c_int64), ("dbu_nm", C.c_double)]


class NetParasiticsC(C.Structure):
    _fields_ = [("net", C.c_uint32), ("r_ohm", C.c_double), ("cap_af", C.c_double)]


_lib = None
_lock = threading.Lock()


def load(build_if_missing: bool = True):
    """Load the library (building it in place when missing or stale).  Raises
    if it cannot be built or loaded — the product path has no fallback."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        from . import build as _build

        if build_if_missing and not _build.up_to_date():
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"gpx-pex CUDA library missing: {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32
        L.gpx_ctx_create.argtypes = [C.POINTER(vp), C.c_int]
        L.gpx_ctx_destroy.argtypes = [vp]
        L.gpx_ctx_destroy.restype = None
        L.gpx_last_error.argtypes = [vp]
        L.gpx_last_error.restype = C.c_char_p
        L.gpx_version.restype = C.c_char_p
        L.gpx_cap_solve.argtypes = [vp, C.POINTER(PanelProblem), C.POINTER(SolveOpts), vp, C.POINTER(SolveReport)]
        L.gpx_cap_solve_eps.argtypes = [vp, C.POINTER(PanelProblem), vp, C.POINTER(SolveOpts), vp,
                                        C.POINTER(SolveReport)]
        L.gpx_cap_solve_batched.argtypes = [vp, vp, i32, C.POINTER(SolveOpts), vp, vp]
        L.gpx_operator_apply.argtypes = [vp, C.POINTER(PanelProblem), C.POINTER(SolveOpts), i32, vp, vp,
                                         C.POINTER(SolveReport)]
        L.gpx_potential_matrix.argtypes = [vp, i64, vp, i64, vp, vp]
        L.gpx_cap_solve_groups.argtypes = [vp, vp, i64, vp, C.c_double, C.POINTER(SolveOpts), vp, vp, i64,
                                           C.POINTER(i64), vp, C.POINTER(SolveReport)]
        L.gpx_extract_quasistatic.argtypes = [vp, C.POINTER(GeometryStoreC), C.POINTER(DeckC), vp, i64,
                                              C.POINTER(SolveOpts), vp, i64, C.POINTER(i64), C.POINTER(C.c_uint32),
                                              C.POINTER(SolveReport)]
        L.gpx_bridge_panelize.argtypes = [vp, C.POINTER(GeometryStoreC), C.POINTER(DeckC), vp, i64,
                                          C.POINTER(SolveOpts), vp, vp, vp, i64, C.POINTER(i64), vp, i64,
                                          C.POINTER(i64), C.POINTER(C.c_uint32)]
        L.gpx_plan_check.argtypes = [i64, vp, i32, i32, vp]
        L.gpx_ctx_stream.argtypes = [vp]
        L.gpx_ctx_stream.restype = vp
        L.gpx_ctx_set_profiling.argtypes = [vp, i32]
        L.gpx_ctx_kernel_stats.argtypes = [vp, i32, C.POINTER(i64), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(i64)]
        L.gpx_ctx_reset_stats.argtypes = [vp]
        L.gpx_cap_solve_small_static.argtypes = [vp, i64, vp, vp, i32, vp]
        L.gpx_autotune.argtypes = [vp, C.POINTER(PanelProblem), C.POINTER(SolveOpts), C.c_double, C.c_char_p,
                                   C.POINTER(SolveOpts), C.POINTER(TuneReport)]
        L.gpx_cap_sensitivity.argtypes = [vp, C.POINTER(PanelProblem), C.POINTER(SolveOpts), i32, vp, vp, vp,
                                          C.POINTER(SolveReport)]
        L.gpx_cap_sensitivity_rows.argtypes = [vp, C.POINTER(PanelProblem), C.POINTER(SolveOpts), i32, vp, i32, vp,
                                               vp, vp, C.POINTER(SolveReport)]
        for name in EXPORTS:
            if name not in ("gpx_ctx_destroy", "gpx_last_error", "gpx_version", "gpx_ctx_stream"):
                getattr(L, name).restype = C.c_int
        _lib = L
        return _lib


def opts(**kw) -> SolveOpts:
    o = SolveOpts()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Context:
    """One device context (one CUDA stream).  Use one per thread."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        st = self.L.gpx_ctx_create(C.byref(h), device)
        if st != GPX_OK:
            raise GpxError(st, self.L.gpx_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.gpx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, polygon=0xFFFFFFFF):
        if st != GPX_OK:
            raise GpxError(st, self.L.gpx_last_error(self.h).decode(), polygon)

    def stream_handle(self) -> int:
        return int(self.L.gpx_ctx_stream(self.h) or 0)

    def set_profiling(self, on: bool):
        self._check(self.L.gpx_ctx_set_profiling(self.h, int(on)))

    def reset_stats(self):
        self._check(self.L.gpx_ctx_reset_stats(self.h))

    def kernel_stats(self):
        out = {}
        total = C.c_int64()
        for k, name in enumerate(KERNEL_CLASSES):
            n, ms, by, fl = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
            self._check(self.L.gpx_ctx_kernel_stats(self.h, k, C.byref(n), C.byref(ms), C.byref(by), C.byref(fl),
                                                    C.byref(total)))
            out[name] = dict(launches=n.value, ms=ms.value, bytes=by.value, flops=fl.value)
        out["total_launches"] = total.value
        return out

    def cap_solve(self, verts, cond, ncond, eps=None, **kw):
        """gpx_cap_solve; with ``eps`` (one relative permittivity per panel)
        gpx_cap_solve_eps, each panel's charge counted eps times."""
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
        c = np.ascontiguousarray(cond, dtype=np.int32)
        pb = PanelProblem(len(v), v.ctypes.data, c.ctypes.data, ncond)
        Cm = np.zeros((ncond, ncond))
        rep = SolveReport()
        if eps is None:
            self._check(self.L.gpx_cap_solve(self.h, C.byref(pb), C.byref(opts(**kw)), Cm.ctypes.data,
                                             C.byref(rep)))
        else:
            e = np.ascontiguousarray(eps, dtype=np.float64)
            if e.shape != (len(v),):
                raise ValueError("eps needs one value per panel")
            self._check(self.L.gpx_cap_solve_eps(self.h, C.byref(pb), e.ctypes.data, C.byref(opts(**kw)),
                                                 Cm.ctypes.data, C.byref(rep)))
        return Cm, rep.as_dict()

    def cap_solve_groups(self, groups, rects, xy_scale_m, **kw):
        """gpx_cap_solve_groups (bridge.rs:307-443 `solve_capacitance`).
        ``groups``: (net, z0_m, z1_m, dielectric_k, rect_offset, rect_count)
        tuples in BTreeMap<(net, layer)> order; ``rects``: (n, 4) int32 DBU
        rectangles (x0, y0, x1, y1).  Returns (nets, cap_af, maxwell, report):
        per net (ascending id) C[i][i] in aF, and the k-scaled Maxwell matrix
        in farads (last row/column = substrate)."""
        g = (VolumeGroup * max(1, len(groups)))(*[VolumeGroup(*t) for t in groups])
        r = np.ascontiguousarray(rects, dtype=np.int32).reshape(-1, 4)
        cap = max(1, len({t[0] for t in groups}))
        nets = np.zeros(cap, dtype=np.uint32)
        af = np.zeros(cap)
        mw = np.zeros((cap + 1) * (cap + 1))
        n = C.c_int64()
        rep = SolveReport()
        self._check(self.L.gpx_cap_solve_groups(self.h, g, len(groups), r.ctypes.data, float(xy_scale_m),
                                                C.byref(opts(**kw)), nets.ctypes.data, af.ctypes.data, cap,
                                                C.byref(n), mw.ctypes.data, C.byref(rep)))
        k = n.value
        return nets[:k].copy(), af[:k].copy(), mw[: (k + 1) * (k + 1)].reshape(k + 1, k + 1), rep.as_dict()

    def autotune(self, verts, cond, ncond, target=1e-4, cache_path=None, **kw):
        """gpx_autotune: returns (options dict to pass to cap_solve, report)."""
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
        c = np.ascontiguousarray(cond, dtype=np.int32)
        pb = PanelProblem(len(v), v.ctypes.data, c.ctypes.data, ncond)
        base = opts(**kw)
        tuned = SolveOpts()
        rep = TuneReport()
        path = cache_path.encode() if cache_path else None
        self._check(self.L.gpx_autotune(self.h, C.byref(pb), C.byref(base), float(target), path, C.byref(tuned),
                                        C.byref(rep)))
        out = dict(kw)
        for k in ("order", "max_level", "far_quad", "mixed_near", "dense_below"):
            out[k] = getattr(tuned, k)
        return out, rep.as_dict()

    def cap_solve_batched(self, problems, **kw):
        """Many independent windows in one call (gpx_cap_solve_batched).
        ``problems``: sequence of (verts, cond, ncond).  Returns a list of
        (C, report) in input order."""
        keep, pbs = [], (PanelProblem * max(1, len(problems)))()
        outs = []
        for i, (verts, cond, ncond) in enumerate(problems):
            v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
            c = np.ascontiguousarray(cond, dtype=np.int32)
            keep += [v, c]
            pbs[i] = PanelProblem(len(v), v.ctypes.data, c.ctypes.data, ncond)
            outs.append(np.zeros((ncond, ncond)))
        ptrs = (C.c_void_p * max(1, len(outs)))(*[o.ctypes.data for o in outs])
        reps = (SolveReport * max(1, len(outs)))()
        self._check(self.L.gpx_cap_solve_batched(self.h, C.cast(pbs, C.c_void_p), len(outs), C.byref(opts(**kw)),
                                                 C.cast(ptrs, C.c_void_p), C.cast(reps, C.c_void_p)))
        return [(outs[i], reps[i].as_dict()) for i in range(len(outs))]

    def cap_sensitivity(self, verts, cond, ncond, velocities, grad_rows=None, **kw):
        """Maxwell matrix and its derivatives along vertex velocity fields
        (``velocities``: n_params x n_panels x 12).  Returns (C, dC, report)
        with dC n_params x ncond x ncond (farads per unit parameter).  With
        ``grad_rows`` (conductor indices) only those rows of dC are computed
        (gpx_cap_sensitivity_rows); the other rows are NaN."""
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
        c = np.ascontiguousarray(cond, dtype=np.int32)
        V = np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1, len(v), 12)
        pb = PanelProblem(len(v), v.ctypes.data, c.ctypes.data, ncond)
        Cm = np.zeros((ncond, ncond))
        dC = np.zeros((len(V), ncond, ncond))
        rep = SolveReport()
        if grad_rows is None:
            self._check(self.L.gpx_cap_sensitivity(self.h, C.byref(pb), C.byref(opts(**kw)), len(V), V.ctypes.data,
                                                   Cm.ctypes.data, dC.ctypes.data, C.byref(rep)))
        else:
            rows = np.ascontiguousarray(grad_rows, dtype=np.int32)
            self._check(self.L.gpx_cap_sensitivity_rows(self.h, C.byref(pb), C.byref(opts(**kw)), len(V),
                                                        V.ctypes.data, len(rows), rows.ctypes.data, Cm.ctypes.data,
                                                        dC.ctypes.data, C.byref(rep)))
        return Cm, dC, rep.as_dict()

    def operator_apply(self, verts, sigma, **kw):
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        if s.ndim == 1:
            s = s[:, None]
        y = np.zeros_like(s)
        pb = PanelProblem(len(v), v.ctypes.data, None, 1)
        rep = SolveReport()
        self._check(self.L.gpx_operator_apply(self.h, C.byref(pb), C.byref(opts(**kw)), s.shape[1], s.ctypes.data,
                                              y.ctypes.data, C.byref(rep)))
        return y, rep.as_dict()

    def cap_solve_small_static(self, n_panels: int, d_verts: int, d_conductor: int, n_conductors: int,
                               d_maxwell_out: int):
        """gpx_cap_solve_small_static on device pointers (integers): the
        Maxwell matrix of <= 512 panels and <= 64 conductors, computed in the
        library's fixed static device scratch without allocating."""
        self._check(self.L.gpx_cap_solve_small_static(self.h, n_panels, d_verts, d_conductor, n_conductors,
                                                      d_maxwell_out))

    def potential_matrix(self, src_verts, points):
        v = np.ascontiguousarray(src_verts, dtype=np.float64).reshape(-1, 12)
        p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(p), len(v)))
        self._check(self.L.gpx_potential_matrix(self.h, len(v), v.ctypes.data, len(p), p.ctypes.data,
                                                out.ctypes.data))
        return out


def _store_c(arrs):
    keep = [np.ascontiguousarray(arrs["verts_x"], dtype=np.int32),
            np.ascontiguousarray(arrs["verts_y"], dtype=np.int32),
            np.ascontiguousarray(arrs["poly_vert_start"], dtype=np.uint32),
            np.ascontiguousarray(arrs["poly_vert_len"], dtype=np.uint32),
            np.ascontiguousarray(arrs["poly_layer"], dtype=np.uint16)]
    st = GeometryStoreC(*(k.ctypes.data for k in keep), len(keep[2]))
    return st, keep


def _deck_c(layer_table, dbu_nm):
    arr = (LayerParamsC * max(1, len(layer_table)))()
    for i, d in enumerate(layer_table):
        for k, _ in LayerParamsC._fields_:
            setattr(arr[i], k, d.get(k, 0))
    return DeckC(C.cast(arr, C.c_void_p), len(layer_table), dbu_nm), arr


def bridge_panelize(store_arrays, layer_table, dbu_nm, net_of_poly, **kw):
    """Host-only panelisation through the C ABI (no device needed)."""
    L = load()
    st, keep = _store_c(store_arrays)
    dk, arr = _deck_c(layer_table, dbu_nm)
    nop = np.ascontiguousarray(net_of_poly, dtype=np.uint32)
    o = opts(**kw)
    n = C.c_int64()
    nn = C.c_int64()
    poly = C.c_uint32()
    s = L.gpx_bridge_panelize(None, C.byref(st), C.byref(dk), nop.ctypes.data, len(nop), C.byref(o), None, None, None,
                              0, C.byref(n), None, 0, C.byref(nn), C.byref(poly))
    if s not in (GPX_OK, 20):
        raise GpxError(s, L.gpx_last_error(None).decode(), poly.value)
    verts = np.zeros((n.value, 12))
    cond = np.zeros(n.value, dtype=np.int32)
    eps = np.zeros(n.value)
    nets = np.zeros(max(1, nn.value), dtype=np.uint32)
    s = L.gpx_bridge_panelize(None, C.byref(st), C.byref(dk), nop.ctypes.data, len(nop), C.byref(o), verts.ctypes.data,
                              cond.ctypes.data, eps.ctypes.data, n.value, C.byref(n), nets.ctypes.data, len(nets),
                              C.byref(nn), C.byref(poly))
    if s != GPX_OK:
        raise GpxError(s, L.gpx_last_error(None).decode(), poly.value)
    return dict(verts=verts, cond=cond, eps=eps, nets=nets[: nn.value])


def plan_check(verts, order, depth):
    L = load()
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
    stats = np.zeros(8, dtype=np.int64)
    s = L.gpx_plan_check(len(v), v.ctypes.data, order, depth, stats.ctypes.data)
    if s != GPX_OK:
        raise GpxError(s, L.gpx_last_error(None).decode())
    keys = ("leaves", "boxes", "near_pairs", "m2l_box_pairs", "far_panel_pairs", "max_leaf", "max_near_row",
            "checksum")
    out = dict(zip(keys, (int(x) for x in stats[:7])))
    out["checksum"] = int(stats[7].view(np.uint64))
    return out
