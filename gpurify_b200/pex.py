"""Host-side mirror of the reference's per-net PEX entry points for the
field-solver path (crates/pex/src/lib.rs:38-126), calling the CUDA library
through its C ABI.

* ``run_pex_by_net_checked`` (lib.rs:66-76) and
  ``run_pex_by_net_with_accuracy_checked`` (lib.rs:103-126): fail closed; any
  bridge or solver failure becomes ``PexError`` carrying one
  ``ExtractionDiagnostic(layer="<quasistatic-bridge>", polygon, model="quasistatic",
  message)`` exactly as lib.rs:111-123 builds it.
* ``run_pex_by_net`` / ``run_pex_by_net_with_accuracy`` (lib.rs:53-63, :84-100):
  the reference falls back to its analytical extractor here; the analytical
  models are not part of this library, so these raise the same ``PexError``
  after logging once (bridge.rs:654-661 wording) instead of fabricating values.

What the GPU path returns per net: ``cap_af`` = C[i][i] in aF (k-scaled) and
``r_ohm`` = the deck's fixed via/contact resistances.  The sheet-resistance
FastHenry solve (bridge.rs:144, :180-299) stays with the caller and is added
to ``r_ohm`` by the caller, as the reference does.
"""
from __future__ import annotations

import enum
import sys
import threading
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .geometry import Deck, GeometryStore


class Accuracy(enum.Enum):
    ANALYTICAL = "analytical"
    QUASISTATIC = "quasistatic"


@dataclass
class NetParasitics:
    r_ohm: float = 0.0
    cap_af: float = 0.0


@dataclass
class ExtractionDiagnostic:
    layer: str
    polygon: int
    model: str
    message: str


class PexError(Exception):
    """``PexError::UnsupportedGeometry(Vec<Parasitic::ExtractionDiagnostic>)``."""

    def __init__(self, diagnostics: List[ExtractionDiagnostic], status: int = 0):
        super().__init__("; ".join(d.message for d in diagnostics))
        self.diagnostics = diagnostics
        self.status = status


_ctx_lock = threading.Lock()
_ctx: Dict[int, _lib.Context] = {}


def default_context(device: int = 0) -> _lib.Context:
    """Lazily created per-process device context (backend/src/gpu.rs:270-278)."""
    with _ctx_lock:
        if device not in _ctx:
            _ctx[device] = _lib.Context(device)
        return _ctx[device]


def extract_quasistatic(store: GeometryStore, deck: Deck, net_of_poly: Sequence[int], ctx: Optional[_lib.Context] = None,
                        report: Optional[dict] = None, **opts) -> Dict[int, NetParasitics]:
    """bridge.rs:73-147 through ``gpx_extract_quasistatic``.  Raises
    ``_lib.GpxError`` on failure (with ``.polygon`` for geometry errors)."""
    import ctypes as C

    ctx = ctx or default_context()
    arrs = store.arrays()
    st, keep = _lib._store_c(arrs)
    dk, arr = _lib._deck_c(deck.layer_table(), deck.dbu_nm)
    nop = np.ascontiguousarray(net_of_poly, dtype=np.uint32)
    cap = max(1, len(nop) + 1)
    out = (_lib.NetParasiticsC * cap)()
    n = C.c_int64()
    poly = C.c_uint32()
    rep = _lib.SolveReport()
    o = _lib.opts(**opts) if opts else None
    s = ctx.L.gpx_extract_quasistatic(ctx.h, C.byref(st), C.byref(dk), nop.ctypes.data, len(nop),
                                      C.byref(o) if o is not None else None, C.cast(out, C.c_void_p), cap,
                                      C.byref(n), C.byref(poly), C.byref(rep))
    ctx._check(s, poly.value)
    if report is not None:
        report.update(rep.as_dict())
    return {int(out[i].net): NetParasitics(out[i].r_ohm, out[i].cap_af) for i in range(n.value)}


def _diagnostic(err: _lib.GpxError) -> PexError:
    polygon = err.polygon if err.status == 12 else 0xFFFFFFFF
    return PexError([ExtractionDiagnostic("<quasistatic-bridge>", polygon, "quasistatic", err.message)], err.status)


def run_pex_by_net_with_accuracy_checked(store, deck, net_of_poly, accuracy=Accuracy.QUASISTATIC, **kw):
    """lib.rs:103-126 (fail-closed)."""
    if accuracy is Accuracy.ANALYTICAL:
        raise NotImplementedError("analytical extraction is not part of the GPU field-solver library")
    try:
        return extract_quasistatic(store, deck, net_of_poly, **kw)
    except _lib.GpxError as e:
        raise _diagnostic(e) from None


def run_pex_by_net_checked(store, deck, net_of_poly, **kw):
    """lib.rs:66-76: accuracy from ``deck.pex_method``."""
    acc = Accuracy.QUASISTATIC if deck.pex_method == "field_solver" else Accuracy.ANALYTICAL
    return run_pex_by_net_with_accuracy_checked(store, deck, net_of_poly, acc, **kw)


_warned = False


def run_pex_by_net_with_accuracy(store, deck, net_of_poly, accuracy=Accuracy.QUASISTATIC, **kw):
    """lib.rs:84-100.  Logs the failure once; no analytical values are made up."""
    global _warned
    try:
        return run_pex_by_net_with_accuracy_checked(store, deck, net_of_poly, accuracy, **kw)
    except PexError as e:
        if not _warned:
            _warned = True
            print(f"pex: quasi-static extraction failed ({e}); no analytical fallback in this library",
                  file=sys.stderr)
        raise


def run_pex_by_net(store, deck, net_of_poly, **kw):
    acc = Accuracy.QUASISTATIC if deck.pex_method == "field_solver" else Accuracy.ANALYTICAL
    return run_pex_by_net_with_accuracy(store, deck, net_of_poly, acc, **kw)


@dataclass
class CapSensitivity:
    """Maxwell matrix and its parameter derivatives of one layout.

    ``nets``: net ids in conductor order (the substrate plate is the last
    conductor).  ``maxwell_af``: k-scaled Maxwell matrix in aF.  ``grad``:
    per parameter, dC/dp in aF per um for geometric parameters and aF per unit
    of k for ``("k",)``."""
    nets: List[int]
    maxwell_af: np.ndarray
    grad: Dict[tuple, np.ndarray]
    report: dict = field(default_factory=dict)


def run_pex_sensitivity_checked(store: GeometryStore, deck: Deck, net_of_poly: Sequence[int], params,
                                ctx: Optional[_lib.Context] = None, **opts) -> CapSensitivity:
    """Capacitance sensitivities beside the checked field-solver result
    (fail-closed like ``run_pex_by_net_checked``): the layout is panelised as
    the bridge does, the Maxwell matrix and dC/dp for every parameter of
    ``params`` (see ``sensitivity.velocity_fields``) come from one forward and
    one transposed solve on the GPU."""
    from . import sensitivity

    ctx = ctx or default_context()
    panel_kw = {k: opts.pop(k) for k in ("mesh_max_edge_m", "max_panels") if k in opts}
    try:
        p = _lib.bridge_panelize(store.arrays(), deck.layer_table(), deck.dbu_nm, net_of_poly, **panel_kw)
        if len(p["verts"]) == 0:
            raise _lib.GpxError(15, "no panels in geometry")
        eps = p["eps"]
        if np.any(np.abs(eps - eps[0]) > 1e-12 * abs(eps[0])):
            raise _lib.GpxError(15, "sensitivities need one dielectric constant for the whole stack "
                                    "(a stack of several k is solved by run_pex_by_net_checked, not differentiated)")
        k = float(eps[0])
        ncond = len(p["nets"]) + 1
        V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
        C, dC, rep = ctx.cap_sensitivity(p["verts"], p["cond"], ncond, V, **opts)
    except _lib.GpxError as e:
        raise _diagnostic(e) from None
    grad = {}
    for q, prm in enumerate(params):
        grad[tuple(prm)] = C * 1e18 if prm[0] == "k" else k * dC[q] * 1e18 * 1e-6
    return CapSensitivity([int(x) for x in p["nets"]], k * C * 1e18, grad, rep)
