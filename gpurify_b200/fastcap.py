"""FastCap input decks in front of the field solver.

* ``parse`` reads the quickif panel format, ``.qui`` (cap/geometry.rs:1-135):
  ``Q c`` + 12 coordinates (quadrilateral), ``T c`` + 9 (triangle), ``N c name``
  (conductor name), and title / comment lines starting with ``0``, ``*`` or
  ``%``.  Conductors are numbered by FastCap's conductor number and indexed
  0, 1, ... in the order their first panel appears; an unnamed conductor is
  called ``cond<number>``.  ``C`` include lines are rejected, as in the
  reference.  Errors read ``line <n>: <message>`` (geometry.rs:36-40).
* ``parse_list_str`` / ``parse_list_file`` read a list file, ``.lst``
  (cap/listfile.rs:1-115): ``C <file> <outerperm> <xt> <yt> <zt> [+|-]`` adds
  the conductors of one ``.qui`` file, translated, as new conductors named
  ``<file>:<index>``.  The reference sends list files to its multi-dielectric
  solver (cap/dielectric.rs:76-150), where every ``C`` panel is a conductor
  panel in its line's permittivity: one permittivity for all lines scales
  the Maxwell matrix; several are kept per panel and each panel's charge
  counts with its own (``gpx_cap_solve_eps``).  ``D`` (dielectric interface)
  lines are rejected.
* ``solve`` computes the Maxwell capacitance matrix in farads through
  ``gpx_cap_solve`` (cap::solve, cap/solver.rs:100-134): one right-hand side
  per conductor, no ground.  Below ``dense_below`` panels (default 500) the
  all-pairs operator stands in for the reference's dense LU; above it the
  Chebyshev FMM runs, where the reference would still factor the dense matrix.

A triangle is stored as a quadrilateral whose fourth vertex repeats the third,
which the panel integrals treat as a zero-length edge.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib


class FastCapError(ValueError):
    """A deck that cannot be read: the message names the line."""


@dataclass
class Geometry:
    """Panels of a FastCap deck: ``verts`` N x 12 (four corners, metres after
    scaling), ``cond`` N conductor indices, one name per conductor, and the
    relative permittivity of the surrounding medium: ``eps_r`` when it is one
    for the whole deck, else ``panel_eps`` (N values, one per panel)."""
    verts: np.ndarray
    cond: np.ndarray
    conductor_names: List[str]
    eps_r: float = 1.0
    numbers: List[int] = field(default_factory=list)  # FastCap conductor number of each index
    panel_eps: Optional[np.ndarray] = None

    def num_conductors(self) -> int:
        return len(self.conductor_names)


def _numbers(tokens: List[str], count: int, line: int) -> List[float]:
    if len(tokens) < count:
        raise FastCapError(f"line {line}: expected {count} numbers, got {len(tokens)}")
    out = []
    for t in tokens[:count]:
        try:
            out.append(float(t))
        except ValueError:
            raise FastCapError(f"line {line}: bad number '{t}'") from None
    return out


def _int_token(tokens: List[str], i: int) -> Optional[int]:
    if len(tokens) <= i:
        return None
    try:
        return int(tokens[i])
    except ValueError:
        return None


def parse(text: str, scale: float = 1.0) -> Geometry:
    """A ``.qui`` deck; ``scale`` multiplies every coordinate (geometry.rs:55-135)."""
    corners: List[List[float]] = []
    cond: List[int] = []
    index_of: Dict[int, int] = {}
    names: List[str] = []
    numbers: List[int] = []
    named: Dict[int, str] = {}

    def conductor(num: int) -> int:
        if num not in index_of:
            index_of[num] = len(names)
            numbers.append(num)
            names.append(named.get(num, f"cond{num}"))
        return index_of[num]

    for n, raw in enumerate(text.splitlines(), start=1):
        line = raw.strip()
        if not line:
            continue
        kind = line[0]
        tokens = line.split()
        if kind in "0*%":
            continue
        if kind in "QqTt":
            quad = kind in "Qq"
            num = _int_token(tokens, 1)
            if num is None:
                raise FastCapError(f"line {n}: {kind.upper()}: missing conductor number")
            xyz = _numbers(tokens[2:], 12 if quad else 9, n)
            pts = [[xyz[3 * k] * scale, xyz[3 * k + 1] * scale, xyz[3 * k + 2] * scale] for k in range(len(xyz) // 3)]
            if not quad:
                pts.append(list(pts[2]))
            corners.append([c for p in pts for c in p])
            cond.append(conductor(num))
        elif kind in "Nn":
            num = _int_token(tokens, 1)
            if num is not None and len(tokens) > 2:
                named[num] = tokens[2]
                if num in index_of:
                    names[index_of[num]] = tokens[2]
        elif kind in "Cc":
            raise FastCapError(f"line {n}: C (sub-file include) not yet supported")
        else:
            raise FastCapError(f"line {n}: unrecognized line: {line}")
    verts = np.asarray(corners, dtype=np.float64).reshape(-1, 12)
    return Geometry(verts, np.asarray(cond, dtype=np.int32), names, 1.0, numbers)


def _list_number(tokens: List[str], i: int, line: int, what: str) -> float:
    try:
        return float(tokens[i])
    except (IndexError, ValueError):
        raise FastCapError(f"line {line}: expected number for {what}") from None


def parse_list_str(text: str, base_dir: str = ".") -> Geometry:
    """A conductor list file; sub-file paths are relative to ``base_dir``
    (listfile.rs:42-101, conductor lines only)."""
    blocks: List[np.ndarray] = []
    conds: List[np.ndarray] = []
    names: List[str] = []
    block_eps: List[float] = []
    for n, raw in enumerate(text.splitlines(), start=1):
        line = raw.strip()
        if not line or line[0] in "*%":
            continue
        tokens = line.split()
        kind = tokens[0]
        if kind in ("D", "d"):
            raise FastCapError(f"line {n}: dielectric interfaces (D lines) are not solved by this library; "
                               "it takes conductor panels (C lines), each in its own medium")
        if kind not in ("C", "c"):
            raise FastCapError(f"line {n}: unrecognized list line: {line}")
        if len(tokens) < 2:
            raise FastCapError(f"line {n}: C: missing file")
        fname = tokens[1]
        outer = _list_number(tokens, 2, n, "outer permittivity")
        shift = np.array([_list_number(tokens, 3 + k, n, w) for k, w in enumerate(("xtrans", "ytrans", "ztrans"))])
        path = os.path.join(base_dir, fname)
        try:
            with open(path) as f:
                sub_text = f.read()
        except OSError as e:
            raise FastCapError(f"cannot read '{path}': {e}") from None
        try:
            sub = parse(sub_text, 1.0)
        except FastCapError as e:
            raise FastCapError(f"geometry parse error in '{fname}': {e} (line {n} of list)") from None
        first = len(names)
        names.extend(f"{fname}:{k}" for k in range(sub.num_conductors()))
        v = sub.verts.copy()
        v.reshape(-1, 4, 3)[:] += shift
        blocks.append(v)
        conds.append(sub.cond + first)
        block_eps.append(outer)
    verts = np.concatenate(blocks) if blocks else np.zeros((0, 12))
    cond = np.concatenate(conds).astype(np.int32) if conds else np.zeros(0, dtype=np.int32)
    if len(set(block_eps)) <= 1:
        return Geometry(verts, cond, names, block_eps[0] if block_eps else 1.0, list(range(len(names))))
    panel_eps = np.concatenate([np.full(len(b), e) for b, e in zip(blocks, block_eps)])
    return Geometry(verts, cond, names, 1.0, list(range(len(names))), panel_eps)


def parse_list_file(path: str) -> Geometry:
    """A list file on disk; sub-files are resolved next to it (listfile.rs:34-40)."""
    try:
        with open(path) as f:
            text = f.read()
    except OSError as e:
        raise FastCapError(f"cannot read '{path}': {e}") from None
    return parse_list_str(text, os.path.dirname(path) or ".")


def solve(geo: Geometry, ctx: Optional[_lib.Context] = None, **opts) -> Tuple[np.ndarray, dict]:
    """Maxwell capacitance matrix (farads, scaled by the media's
    permittivities) and the solve report.  ``opts`` are ``gpx_solve_opts``
    fields."""
    if len(geo.verts) == 0:
        raise FastCapError("no panels in the deck")
    if ctx is None:
        from .pex import default_context
        ctx = default_context()
    kw = dict(skip_ground_rhs=0)
    kw.update(opts)
    if geo.panel_eps is not None:
        return ctx.cap_solve(geo.verts, geo.cond, geo.num_conductors(), eps=geo.panel_eps, **kw)
    C, rep = ctx.cap_solve(geo.verts, geo.cond, geo.num_conductors(), **kw)
    return C * geo.eps_r, rep
