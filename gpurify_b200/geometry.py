"""Layout-side data model mirrored from the reference's core crate.

``GeometryStore`` follows crates/core/src/geometry/store.rs:14-134 (flat SoA
polygon store: ``verts_x``, ``verts_y``, ``poly_layer``, ``poly_vert_start``,
``poly_vert_len``; ``add_rect(layer, x, y, w, h)`` at store.rs:132-134).
``Deck`` carries the per-layer PEX parameters of crates/core/src/io/pdk.rs:520-554
(``PexLayerParams``), the ``pex_method`` selector and ``dbu_nm``
(io/pdk.rs:619-621, default 1.0 at :1402).
"""
from __future__ import annotations

from dataclasses import dataclass, field, asdict
from typing import Dict, List, Sequence, Tuple

import numpy as np


class GeometryStore:
    """Flat structure-of-arrays polygon store in database units (i32)."""

    def __init__(self) -> None:
        self._vx: List[int] = []
        self._vy: List[int] = []
        self._layer: List[int] = []
        self._start: List[int] = []
        self._len: List[int] = []

    def add_polygon(self, layer: int, pts: Sequence[Tuple[int, int]]) -> int:
        """Append a closed ring (first point not repeated); returns its PolyId."""
        self._start.append(len(self._vx))
        self._len.append(len(pts))
        for x, y in pts:
            self._vx.append(int(x))
            self._vy.append(int(y))
        self._layer.append(int(layer))
        return len(self._layer) - 1

    def add_rect(self, layer: int, x: int, y: int, w: int, h: int) -> int:
        """store.rs:132-134: the ring (x,y), (x+w,y), (x+w,y+h), (x,y+h)."""
        return self.add_polygon(layer, [(x, y), (x + w, y), (x + w, y + h), (x, y + h)])

    def poly_count(self) -> int:
        return len(self._layer)

    def arrays(self) -> Dict[str, np.ndarray]:
        return dict(
            verts_x=np.asarray(self._vx, dtype=np.int32),
            verts_y=np.asarray(self._vy, dtype=np.int32),
            poly_vert_start=np.asarray(self._start, dtype=np.uint32),
            poly_vert_len=np.asarray(self._len, dtype=np.uint32),
            poly_layer=np.asarray(self._layer, dtype=np.uint16),
        )


@dataclass
class PexLayerParams:
    """io/pdk.rs:520-544 (all floats; serde defaults are 0)."""

    sheet_res_ohm_sq: float = 0.0
    area_cap_af_um2: float = 0.0
    fringe_cap_af_um: float = 0.0
    coupling_cap_af_um: float = 0.0
    coupling_ref_spacing_nm: float = 0.0
    via_res_ohm: float = 0.0
    interlayer_cap_af_um2: float = 0.0
    thickness_nm: float = 0.0
    height_nm: float = 0.0
    dielectric_k: float = 0.0


@dataclass
class Deck:
    """The parts of the reference ``Deck`` the field-solver path reads."""

    layers: Dict[str, int] = field(default_factory=dict)  # name -> LayerId
    pex: Dict[int, PexLayerParams] = field(default_factory=dict)  # LayerId -> params
    pex_method: str = "analytical"  # "analytical" | "field_solver"
    dbu_nm: float = 1.0

    def layer_id(self, name: str) -> int:
        return self.layers[name]

    def layer_table(self) -> List[dict]:
        out = []
        for lid, p in self.pex.items():
            d = asdict(p)
            d["layer"] = lid
            out.append(d)
        return out

    @staticmethod
    def from_dict(doc: dict) -> "Deck":
        """Accepts the JSON shape of the reference deck (layers / pex / pex_method)."""
        names = list(doc.get("layers", {}).keys())
        layers = {n: i for i, n in enumerate(names)}
        pex = {}
        for name, p in doc.get("pex", {}).items():
            pex[layers[name]] = PexLayerParams(**{k: float(v) for k, v in p.items()})
        return Deck(layers=layers, pex=pex, pex_method=doc.get("pex_method", "analytical"),
                    dbu_nm=float(doc.get("dbu_nm", 1.0)))
