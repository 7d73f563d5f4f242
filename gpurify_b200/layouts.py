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
* ``large_block``    — a 200 x 200 um block on 6 metal layers (t = 0.36 to
  1.2 um, k = 3.9): 512 nets, each a seeded walk of 3..12 segments like the
  routing window's, routed on tracks in each layer's preferred direction.
  The layers reach 23-30 % metal density (the specified 30-50 % needs more
  wire than 512 walks of at most 12 segments place at random).
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


BLOCK_LAYERS = (  # name, LayerId, thickness nm, height nm (0.6 um of dielectric between layers)
    ("met1", 1, 360.0, 400.0),
    ("met2", 3, 500.0, 1360.0),
    ("met3", 5, 850.0, 2460.0),
    ("met4", 7, 850.0, 3910.0),
    ("met5", 9, 1200.0, 5360.0),
    ("met6", 11, 1200.0, 7160.0),
)


def block_deck(method: str = "field_solver", k: float = 3.9) -> Deck:
    """Six metal layers (horizontal preferred direction on met1, met3, met5)
    and the five via layers between them (fixed resistance, not panelised)."""
    d = Deck(pex_method=method, dbu_nm=1.0)
    for name, lid, t, h in BLOCK_LAYERS:
        d.layers[name] = lid
        d.pex[lid] = PexLayerParams(sheet_res_ohm_sq=0.125 if lid == 1 else 0.047, thickness_nm=t, height_nm=h,
                                    dielectric_k=k)
    for i in range(len(BLOCK_LAYERS) - 1):
        lid = BLOCK_LAYERS[i][1] + 1
        top = BLOCK_LAYERS[i][3] + BLOCK_LAYERS[i][2]
        d.layers[f"via{i + 1}"] = lid
        d.pex[lid] = PexLayerParams(via_res_ohm=4.5, thickness_nm=0.0, height_nm=top, dielectric_k=k)
    return d


def large_block(n_nets: int = 512, side_um: float = 200.0, seed: int = 5150, pitch_nm: int = 550,
                seg_len_um: Tuple[float, float] = (100.0, 200.0)) -> Layout:
    """Dense multi-layer block (see module docstring).

    Layers alternate horizontal and vertical tracks at ``pitch_nm``; a wire of
    width w (U[0.14, 0.40] um on the 0.05 um grid, at least 0.15 um) is centred
    on a track, so wires of different nets on one layer keep at least
    pitch - 0.40 um = 0.15 um apart across tracks, and along a track the
    wires keep 0.15 um of clearance at their ends.  A walk turns at every
    segment end onto the layer above or below (a 0.15 um via at the turn), so
    consecutive segments alternate direction as in ``routing_window``.  A
    segment that runs into another net's wire is cut short before it, and it
    ends at the crossing track that leaves the longest run for the next
    segment; walks with fewer than 3 segments are retried.  With the defaults
    the layers reach 23-30 % metal density and the bridge makes about 1.6 M
    panels at a 0.8 um mesh edge."""
    rng = np.random.default_rng(seed)
    deck = block_deck()
    nl = len(BLOCK_LAYERS)
    grid = 50
    side = int(round(side_um * 1000 / grid)) * grid
    ntrack = side // pitch_nm
    if pitch_nm % grid:
        raise ValueError("track pitch must be a multiple of the 50 nm grid")
    tracks = [t * pitch_nm + (pitch_nm // 2) // grid * grid for t in range(ntrack)]  # uniform pitch, on grid
    space = 150
    # occupied intervals per (layer, track): sorted list of (lo, hi, net)
    occ: List[List[List[Tuple[int, int, int]]]] = [[[] for _ in range(ntrack)] for _ in range(nl)]
    horiz = [i % 2 == 0 for i in range(nl)]
    st = GeometryStore()
    nets: List[int] = []

    def room(layer, tr, a, b, net, hw):
        """Largest run [a, b'] (b' towards b) whose metal, the run widened by
        hw at both ends, keeps ``space`` from other nets' metal on the track;
        None when even the start is too close."""
        lo, hi = (a, b) if a <= b else (b, a)
        for (x0, x1, owner) in occ[layer][tr]:
            if owner == net:
                continue
            if x1 + space <= lo - hw or x0 - space >= hi + hw:
                continue
            # conflict: cut the segment before it, keeping the start
            if a <= b:
                if x0 - space - hw <= a:
                    return None
                hi = min(hi, x0 - space - hw)
            else:
                if x1 + space + hw >= a:
                    return None
                lo = max(lo, x1 + space + hw)
        return (lo, hi)

    def take(layer, tr, lo, hi, net):  # lo, hi: the metal extent along the track
        occ[layer][tr].append((lo, hi, net))

    def snap_track(c):
        return int(np.clip(np.searchsorted(tracks, c), 0, ntrack - 1))

    def reach(layer, tr, pos, L, sgn, net, hw=200):
        """Free run from ``pos`` along track ``tr`` of ``layer`` for a wire of
        half-width hw, at most L long in direction sgn: (lo, hi), or None
        when under 1 um."""
        end = int(np.clip(pos + sgn * L, tracks[0], tracks[-1]))
        r = room(layer, tr, pos, end, net, hw)
        if r is None or r[1] - r[0] < 1000:
            return None
        return r

    def neighbours(layer):
        if layer == 0:
            return [1]
        if layer == nl - 1:
            return [nl - 2]
        return [layer + 1, layer - 1] if rng.integers(0, 2) else [layer - 1, layer + 1]

    start_p = np.array([2.0] + [1.0] * (nl - 2) + [2.0])
    start_p /= start_p.sum()
    for net in range(n_nets):
        nseg = int(rng.integers(3, 13))
        for _attempt in range(50):
            # walks start on the outer layers twice as often: those are
            # reached from one neighbour only
            layer = int(rng.choice(nl, p=start_p))
            tr = int(rng.integers(0, ntrack))           # track of the first segment
            pos = tracks[int(rng.integers(0, ntrack))]  # start along it (on a crossing track)
            placed = []
            for s in range(nseg):
                w = max(150, int(round(rng.uniform(0.14, 0.40) * 1000 / grid)) * grid)
                L = int(round(rng.uniform(*seg_len_um) * 1000 / grid)) * grid
                sgn = 1 if rng.integers(0, 2) else -1
                r = reach(layer, tr, pos, L, sgn, net, w // 2)
                if r is None:
                    sgn = -sgn
                    r = reach(layer, tr, pos, L, sgn, net, w // 2)
                if r is None:
                    break
                c = tracks[tr]
                # crossing tracks inside the run, farthest first; the segment
                # ends where this segment plus the free run that the turn onto
                # a neighbour layer leaves for the next one is longest (ties:
                # the farthest)
                lo, hi = r
                ks = [k for k in range(ntrack) if lo <= tracks[k] <= hi and abs(tracks[k] - pos) >= 1000]
                if sgn > 0:  # farthest first
                    ks.reverse()
                turn, best = None, 0
                if s < nseg - 1:
                    for k in ks[:60]:
                        for nlyr in neighbours(layer):
                            for d in (1, -1):
                                q = reach(nlyr, k, c, seg_len_um[1] * 1000, d, net)
                                if q and q[1] - q[0] + abs(tracks[k] - pos) > best:
                                    turn, best = (k, nlyr), q[1] - q[0] + abs(tracks[k] - pos)
                if turn is None and not ks:
                    break
                k = turn[0] if turn else ks[0]
                lo, hi = (pos, tracks[k]) if sgn > 0 else (tracks[k], pos)
                take(layer, tr, lo - w // 2, hi + w // 2, net)
                if horiz[layer]:
                    rect = (lo - w // 2, c - w // 2, hi + w // 2, c + w // 2)
                else:
                    rect = (c - w // 2, lo - w // 2, c + w // 2, hi + w // 2)
                placed.append((layer, tr, lo - w // 2, hi + w // 2, rect))
                if turn is None:
                    break
                nlyr = turn[1]
                x, y = (tracks[k], c) if horiz[layer] else (c, tracks[k])
                placed.append(("via", min(layer, nlyr), (x - 75, y - 75, x + 75, y + 75)))
                layer, tr, pos = nlyr, k, c
            metal = [p for p in placed if p[0] != "via"]
            if len(metal) >= 3:
                while placed and placed[-1][0] == "via":
                    placed.pop()
                for p in placed:
                    if p[0] == "via":
                        lid, r = BLOCK_LAYERS[p[1]][1] + 1, p[2]
                    else:
                        lid, r = BLOCK_LAYERS[p[0]][1], p[4]
                    st.add_rect(lid, r[0], r[1], r[2] - r[0], r[3] - r[1])
                    nets.append(net)
                break
            for p in metal:  # roll back a walk that stayed too short
                occ[p[0]][p[1]].remove((p[2], p[3], net))
    return Layout(st, deck, nets, f"large_block_{n_nets}nets_{side_um:g}um_seed{seed}")
