"""Geometric parameters of a panelised layout as vertex velocity fields, for
the adjoint sensitivities of ``gpx_cap_sensitivity``.

A parameter p moves every panel vertex x with velocity dx/dp (metres per
metre of parameter); the panel topology (the mesh) is held fixed, so the
derivative is that of the discretised Maxwell matrix.  Supported parameters
(straight Manhattan wires; the layout's bus geometry):

* ``("width", net)``     the wire of ``net`` widens symmetrically about its
  centre line: vertices stretch linearly across the wire, the two long sides
  move by -1/2 and +1/2;
* ``("spacing", net)``   the gap between ``net`` and the next wire of the same
  layer (higher coordinate across the wires) grows: every same-layer wire past
  ``net`` translates by +1;
* ``("thickness", z0, z1)`` the metal of the layer spanning [z0, z1] (the
  panels with every vertex in that span) thickens upward: vertices stretch
  linearly, the top faces move by +1;
* ``("height", z0, z1)``  the metal of that layer moves up by +1;
* ``("k",)``             the dielectric constant: no vertex moves; with a
  homogeneous dielectric dC/dk = C / k exactly (the reference scales the
  vacuum Maxwell matrix by k, bridge.rs:405-407).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

Param = Tuple


def _conductor_boxes(verts: np.ndarray, cond: np.ndarray, ncond: int) -> np.ndarray:
    """Per conductor: [xmin, ymin, zmin, xmax, ymax, zmax] of its vertices."""
    pts = verts.reshape(-1, 4, 3)
    box = np.full((ncond, 6), np.nan)
    for c in range(ncond):
        sel = pts[cond == c].reshape(-1, 3)
        if len(sel):
            box[c, :3] = sel.min(0)
            box[c, 3:] = sel.max(0)
    return box


def _width_axis(box: np.ndarray) -> int:
    """Across-wire axis of a straight wire: the shorter of its x / y extents."""
    return 0 if (box[3] - box[0]) < (box[4] - box[1]) else 1


def velocity_fields(verts: np.ndarray, cond: np.ndarray, nets: Sequence[int], params: Sequence[Param]) -> np.ndarray:
    """Vertex velocity fields (len(params) x n_panels x 12) for ``params`` on
    the panels of a bridge panelisation (conductor index = rank of the net in
    ``nets``; the last conductor is the substrate plate, which never moves)."""
    verts = np.asarray(verts, dtype=np.float64).reshape(-1, 12)
    cond = np.asarray(cond)
    nets = [int(x) for x in nets]
    ncond = len(nets) + 1
    box = _conductor_boxes(verts, cond, ncond)
    pts = verts.reshape(-1, 4, 3)
    out = np.zeros((len(params), len(verts), 4, 3))
    for q, prm in enumerate(params):
        kind = prm[0]
        if kind == "width":
            c = nets.index(int(prm[1]))
            ax = _width_axis(box[c])
            lo, hi = box[c, ax], box[c, 3 + ax]
            sel = cond == c
            out[q, sel, :, ax] = (pts[sel, :, ax] - 0.5 * (lo + hi)) / (hi - lo)
        elif kind == "spacing":
            c = nets.index(int(prm[1]))
            ax = _width_axis(box[c])
            zc = box[c, 2]
            centre = 0.5 * (box[c, ax] + box[c, 3 + ax])
            for o in range(ncond - 1):
                if o == c or abs(box[o, 2] - zc) > 1e-12:
                    continue
                if 0.5 * (box[o, ax] + box[o, 3 + ax]) > centre:
                    out[q, cond == o, :, ax] = 1.0
        elif kind in ("thickness", "height"):
            # the panels of the layer's metal: every vertex within [z0, z1]
            # (a net routed over several layers moves only its part on this
            # layer; the substrate plate never moves)
            z0, z1 = float(prm[1]), float(prm[2])
            tol = 1e-12 + 1e-9 * abs(z1 - z0)
            zv = pts[:, :, 2]
            sel = (cond != ncond - 1) & np.all((zv >= z0 - tol) & (zv <= z1 + tol), axis=1)
            if kind == "height":
                out[q, sel, :, 2] = 1.0
            else:
                out[q, sel, :, 2] = (pts[sel, :, 2] - z0) / (z1 - z0)
        elif kind == "k":
            pass
        else:
            raise ValueError(f"unknown sensitivity parameter {prm!r}")
    return out.reshape(len(params), len(verts), 12)


def layer_span(deck, layer_name: str) -> Tuple[float, float]:
    """(z0, z1) in metres of a deck layer's conductors (thickness above height)."""
    lp = deck.pex[deck.layer_id(layer_name)]
    return lp.height_nm * 1e-9, (lp.height_nm + lp.thickness_nm) * 1e-9
