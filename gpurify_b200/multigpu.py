"""Several GPUs for the field-solver capacitance path, one process per GPU
(``torch.distributed``; NCCL on GPUs, gloo on CPU).

The path shards without any exchange of operator data:

* windows are independent problems: ``partition_windows`` spreads a batch
  over the ranks by estimated cost (panels x right-hand sides, largest first
  to the least-loaded rank), each rank solves its own windows through
  ``gpx_cap_solve_batched``, and ``solve_windows_partitioned`` gathers the
  Maxwell matrices;
* within one window the conductor columns are independent given the
  operator: every rank builds the same operator (near blocks, tree, M2L
  tables) on its own GPU and solves one contiguous block of columns
  (``column_blocks``; ``gpx_solve_opts.col_begin/col_count``), and
  ``gather_columns`` assembles the Maxwell matrix with one all-gather of the
  column blocks (nets x columns FP64, kilobytes to a few megabytes) per solve.

The reference solves its conductors one after another on one CPU
(crates/pex/src/quasistatic/cap/fmm_solver.rs:166-170); the column split is
that loop spread over ranks.  Every rank takes the same collective steps in
the same order, also when its own share is empty.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def partition_windows(costs: Sequence[float], world: int) -> List[List[int]]:
    """Window indices per rank: largest cost first, each to the rank with the
    smallest load so far (ties to the lower rank).  Deterministic, so every
    rank computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def column_blocks(n_cols: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous (begin, count) column blocks per rank covering [0, n_cols)
    once; the first n_cols % world ranks get one column more."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    base, extra = divmod(n_cols, world)
    out, b = [], 0
    for r in range(world):
        c = base + (1 if r < extra else 0)
        out.append((b, c))
        b += c
    return out


def _device_for(dist) -> str:
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def gather_columns(block: np.ndarray, blocks: Sequence[Tuple[int, int]], ncond: int, dist) -> np.ndarray:
    """All-gather of the ranks' Maxwell column blocks.  ``block`` is this
    rank's ncond x count slice (columns begin..begin+count of ``blocks[rank]``);
    returns the ncond x sum(count) matrix on every rank.  One collective: the
    blocks are padded to the largest count."""
    import torch

    world = dist.get_world_size()
    wmax = max(c for _, c in blocks) if blocks else 0
    dev = _device_for(dist)
    mine = torch.zeros((ncond, max(wmax, 1)), dtype=torch.float64, device=dev)
    if block.shape[1]:
        mine[:, : block.shape[1]] = torch.from_numpy(np.ascontiguousarray(block)).to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine)
    ncols = sum(c for _, c in blocks)
    out = np.empty((ncond, ncols))
    for (b, c), t in zip(blocks, parts):
        if c:
            out[:, b : b + c] = t[:, :c].cpu().numpy()
    return out


ColumnSolver = Callable[[int, int], np.ndarray]


def solve_window_sharded(ncond: int, dist, skip_ground_rhs: bool = True,
                         column_solver: Optional[ColumnSolver] = None, ctx=None, verts=None, cond=None,
                         symmetric: Optional[bool] = None, **solve_kw) -> np.ndarray:
    """Maxwell matrix of one window with its conductor columns spread over the
    ranks.  Each rank solves ``column_blocks(R, world)[rank]`` (R = nets, or
    every conductor without ``skip_ground_rhs``) with ``column_solver(begin,
    count)`` -> ncond x count, by default ``ctx.cap_solve`` with
    ``col_begin/col_count`` on this rank's GPU; the blocks are all-gathered
    and, with ``skip_ground_rhs``, the substrate column is filled by symmetry
    (C[last][last] NaN), exactly as a single-rank ``gpx_cap_solve`` fills it.
    A matrix of panels in several media (``eps`` per panel in ``solve_kw``,
    or ``symmetric=False``) is not symmetric: that column stays NaN, as
    ``gpx_cap_solve_eps`` leaves it."""
    if symmetric is None:
        symmetric = solve_kw.get("eps") is None
    world, rank = dist.get_world_size(), dist.get_rank()
    R = ncond - 1 if (skip_ground_rhs and ncond > 1) else ncond
    blocks = column_blocks(R, world)
    b, c = blocks[rank]
    if column_solver is None:
        if ctx is None:
            raise ValueError("solve_window_sharded needs a context or a column solver")

        def column_solver(b0, c0):
            C, _ = ctx.cap_solve(verts, cond, ncond, skip_ground_rhs=int(skip_ground_rhs), col_begin=b0,
                                 col_count=c0, **solve_kw)
            return C[:, b0 : b0 + c0]

    block = column_solver(b, c) if c else np.zeros((ncond, 0))
    cols = gather_columns(block, blocks, ncond, dist)
    if R == ncond:
        return cols
    C = np.empty((ncond, ncond))
    C[:, :R] = cols
    C[:R, R] = cols[R, :R] if symmetric else np.nan
    C[R, R] = np.nan
    return C


WindowSolver = Callable[[Sequence[int]], List[np.ndarray]]


def solve_windows_partitioned(costs: Sequence[float], dist, window_solver: WindowSolver) -> List[np.ndarray]:
    """Maxwell matrices of a batch of independent windows spread over the
    ranks by ``partition_windows``; ``window_solver(indices)`` solves this
    rank's windows (e.g. ``gpx_cap_solve_batched`` on its GPU) and returns
    their matrices in the same order.  The matrices are all-gathered (one
    object collective) and returned in batch order on every rank."""
    world, rank = dist.get_world_size(), dist.get_rank()
    parts = partition_windows(costs, world)
    mine = parts[rank]
    res = window_solver(mine) if mine else []
    gathered: List[Optional[list]] = [None] * world
    dist.all_gather_object(gathered, [(i, np.asarray(m)) for i, m in zip(mine, res)])
    out: List[Optional[np.ndarray]] = [None] * len(costs)
    for lst in gathered:
        for i, m in lst:
            out[i] = m
    return out
