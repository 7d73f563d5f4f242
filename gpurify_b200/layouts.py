"""Seeded synthetic layouts for the field-solver workloads.

No public layout corpus is used: every workload is generated here from a seed,
with the shapes, sizes and value distributions the workloads are specified
with.  Units: DBU = 1 nm unless stated.

* ``two_wires``      — two parallel met1 wires, 0.14 um wide x 0.36 um thick x
  20 um long, 0.14 um spacing, 0.4 um above the substrate, k = 3.9.
* ``routing_window`` — a Manhattan routing window: N nets, each a seeded random
  walk of 3..12 rectilinear segments on 3 metal layers (t = 0.36/0.85/0.85 um,
  h = 0.4/1.4/3.0 um, k = 3.9), widths U[0.14, 0.40] um snapped to a 0.05 um
  grid, 0.15 um square vias (fixed-resistance, not panelised) where a walk
  changes layer; different nets never overlap on a layer (a short would merge
  two conductors, which the bridge does not detect).
* ``bus_crossing``   — 8-bit met2 bus (0.2 um wide, 0.4 um pitch, 30 um long)
  crossed by 4 met3 wires (0.4 um wide, 5 um pitch).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

from .geometry import Deck, GeometryStore, PexLayerParams

SKY_LAYERS = {  # name -> (LayerId, thickness nm, height nm)
    "met1": (1, 360.0, 400.0),
    "met2": (3, 850.0, 1400.0),
    "met3": (5, 850.0, 3000.0),
}


def sky_like_deck(method: str = "field_solver", k: float = 3.9) -> Deck:
    """A sky130-like three-metal deck with explicit 3-D geometry.

    The shipped reference PDK carries no thickness/height/k, so this deck is
    written here.  Metal layers have a sheet resistance (volume conductors);
    via layers have a fixed resistance and no sheet resistance, so the bridge
    adds their R and does not panelise them (bridge.rs:171-178)."""
    d = Deck(pex_method=method, dbu_nm=1.0)
    for name, (lid, t, h) in SKY_LAYERS.items():
        d.layers[name] = lid
        d.pex[lid] = PexLayerParams(sheet_res_ohm_sq=0.125 if name == "met1" else 0.047,
                                    thickness_nm=t, height_nm=h, dielectric_k=k)
    for name, lid, h in (("via1", 2, 760.0), ("via2", 4, 2250.0)):
        d.layers[name] = lid
        d.pex[lid] = PexLayerParams(via_res_ohm=4.5, thickness_nm=0.0, height_nm=h, dielectric_k=k)
    return d


@dataclass
class Layout:
    store: GeometryStore
    deck: Deck
    net_of_poly: List[int]
    name: str


def two_wires(length_nm: int = 20000, width_nm: int = 140, spacing_nm: int = 140) -> Layout:
    deck = sky_like_deck()
    met1 = deck.layers["met1"]
    st = GeometryStore()
    st.add_rect(met1, 0, 0, length_nm, width_nm)
    st.add_rect(met1, 0, width_nm + spacing_nm, length_nm, width_nm)
    return Layout(st, deck, [0, 1], "two_wires")


def routing_window(n_nets: int = 64, side_um: float = 40.0, seed: int = 2024, seg_min: int = 3,
                   seg_max: int = 12, len_um: Tuple[float, float] = (1.0, 8.0)) -> Layout:
    """Random Manhattan routing window (see module docstring)."""
    rng = np.random.default_rng(seed)
    deck = sky_like_deck()
    metals = ["met1", "met2", "met3"]
    vias = ["via1", "via2"]
    grid = 50  # nm
    side = int(round(side_um * 1000 / grid)) * grid
    ncell = side // grid
    occ = np.full((3, ncell + 1, ncell + 1), -1, dtype=np.int32)  # owner net per 50 nm cell
    space = 150  # nm clearance to other nets on the same layer
    st = GeometryStore()
    nets: List[int] = []

    def cells(x0, y0, x1, y1, pad):
        a = max(0, (x0 - pad) // grid)
        b = min(ncell, -(-(x1 + pad) // grid))
        c = max(0, (y0 - pad) // grid)
        d = min(ncell, -(-(y1 + pad) // grid))
        return a, b, c, d

    def free(layer, net, r):
        a, b, c, d = cells(*r, space)
        blk = occ[layer, a:b, c:d]
        return not np.any((blk >= 0) & (blk != net))

    def mark(layer, net, r):
        a, b, c, d = cells(*r, 0)
        occ[layer, a:b, c:d] = net

    for net in range(n_nets):
        nseg = int(rng.integers(seg_min, seg_max + 1))
        for _attempt in range(200):
            x = int(rng.integers(1, ncell)) * grid
            y = int(rng.integers(1, ncell)) * grid
            layer = int(rng.integers(0, 3))
            horiz = bool(rng.integers(0, 2))
            placed = []
            ok = True
            for s in range(nseg):
                w = int(round(rng.uniform(0.14, 0.40) * 1000 / grid)) * grid
                w = max(w, 150)
                done = False
                for _t in range(40):
                    L = int(round(rng.uniform(*len_um) * 1000 / grid)) * grid
                    sgn = 1 if rng.integers(0, 2) else -1
                    if horiz:
                        x1 = min(max(x + sgn * L, 0), side)
                        xa, xb = min(x, x1), max(x, x1)
                        r = (xa - w // 2, y - w // 2, xb + w // 2, y + w // 2)
                        nx, ny = x1, y
                    else:
                        y1 = min(max(y + sgn * L, 0), side)
                        ya, yb = min(y, y1), max(y, y1)
                        r = (x - w // 2, ya - w // 2, x + w // 2, yb + w // 2)
                        nx, ny = x, y1
                    r = (max(r[0], 0), max(r[1], 0), min(r[2], side), min(r[3], side))
                    if r[2] - r[0] < 100 or r[3] - r[1] < 100:
                        continue
                    if free(layer, net, r):
                        placed.append((layer, r))
                        mark(layer, net, r)
                        x, y = nx, ny
                        done = True
                        break
                if not done:
                    ok = s >= seg_min
                    break
                # next segment: turn, and change layer with probability 1/2
                horiz = not horiz
                if rng.integers(0, 2):
                    nl = layer + (1 if (layer == 0 or (layer == 1 and rng.integers(0, 2))) else -1)
                    placed.append(("via", min(layer, nl), (x - 75, y - 75, x + 75, y + 75)))
                    layer = nl
            if ok and len([p for p in placed if p[0] != "via"]) >= seg_min:
                for p in placed:
                    if p[0] == "via":
                        lid = deck.layers[vias[p[1]]]
                        r = p[2]
                    else:
                        lid = deck.layers[metals[p[0]]]
                        r = p[1]
                    st.add_rect(lid, r[0], r[1], r[2] - r[0], r[3] - r[1])
                    nets.append(net)
                break
            # roll back marks of a failed attempt
            for p in placed:
                if p[0] != "via":
                    a, b, c, d = cells(*p[1], 0)
                    blk = occ[p[0], a:b, c:d]
                    blk[blk == net] = -1
    return Layout(st, deck, nets, f"routing_window_{n_nets}nets_{side_um:g}um_seed{seed}")


def bus_crossing(bits: int = 8, wires: int = 4, width_nm: int = 200, pitch_nm: int = 400, length_nm: int = 30000,
                 cross_w_nm: int = 400, cross_pitch_nm: int = 5000) -> Layout:
    deck = sky_like_deck()
    m2, m3 = deck.layers["met2"], deck.layers["met3"]
    st = GeometryStore()
    nets = []
    for b in range(bits):
        st.add_rect(m2, 0, b * pitch_nm, length_nm, width_nm)
        nets.append(b)
    span = (bits - 1) * pitch_nm + width_nm
    x0 = (length_nm - (wires - 1) * cross_pitch_nm - cross_w_nm) // 2
    for w in range(wires):
        st.add_rect(m3, x0 + w * cross_pitch_nm, -2000, cross_w_nm, span + 4000)
        nets.append(bits + w)
    return Layout(st, deck, nets, "bus_crossing")


def window_batch(n_windows: int = 256, seed: int = 7) -> List[Layout]:
    """Many independent windows: conductor counts log-uniform in [2, 48], side
    uniform in [5, 60] um, each generated like ``routing_window``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_windows):
        nets = int(round(math.exp(rng.uniform(math.log(2), math.log(48)))))
        side = float(rng.uniform(5.0, 60.0))
        out.append(routing_window(nets, side, seed=seed * 100003 + i, len_um=(0.5, min(8.0, side / 3))))
    return out
