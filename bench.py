#!/usr/bin/env python
"""Throughput benchmark of the field-solver capacitance path on B200.

Workload (one "step"): the full Maxwell-matrix extraction of one seeded
64-net Manhattan routing window, 40 x 40 um, 3 metal layers (t =
0.36/0.85/0.85 um, h = 0.4/1.4/3.0 um, k = 3.9), panelised with a 0.25 um
maximum panel edge (65,192 panels incl. the substrate plate), 64 right-hand
sides (one per net), GMRES relative tolerance 1e-8.

* ``value``   solves/s of ``gpx_cap_solve`` on the panel problem (panel
              buffers in host memory; device time of the call on the
              context stream, CUDA events); ``panel_rhs_per_s`` = N*R/time.
* ``e2e``     the same metric through the public per-net API
              (``run_pex_by_net_checked``: layout polygons -> per-net aF),
              host<->device copies inside the timed region; the mean over
              max(2, steps) calls, like ``value``'s mean over the steps.
* ``roofline``  the dominant kernel's algorithmic work per launch over its
              CUDA-event duration in the timed steps, against the measured
              peaks in MEASURED_PEAKS.json.
* ``cpu_baseline``  the CPU oracle (a restatement of the reference's CPU
              field solver) on the same panels and tree, all host threads:
              the operator set-up plus 4 conductor columns spread over the
              nets, scaled to the 64 columns of an extraction; and config 1
              (two wires, the reference's own mesh and FMM(4,4) mode) timed on
              1 and on all host threads, beside the GPU's FP64 time for it.

``--impl reference`` times the CPU restatement alone as the reference arm: the
operator set-up once, then one conductor column per step.
Multi-GPU (torchrun): every rank solves its own independent window (seed
offset by rank); no collective on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Maxwell-C solves/s & panel·RHS/s at 1e-4 rel err: mixed vs FP64, one B200"
EDGE_M = 0.25e-6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpx", choices=["gpx", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: time the plain FP64 path, then the mixed path (the headline value)")
    ap.add_argument("--order", type=int, default=5)
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--nets", type=int, default=64)
    ap.add_argument("--side", type=float, default=40.0, help="window side in um")
    ap.add_argument("--restart", type=int, default=200, help="GMRES restart length")
    ap.add_argument("--far-quad", type=int, default=1, help="0 centroid lumping (reference), 1 Gauss points")
    ap.add_argument("--precond", type=int, default=-1,
                    help="0 diagonal Jacobi (reference), 1 / 2 leaf block-Jacobi with 48- / 96-panel blocks; "
                         "-1: 2 for the FP64 path, 1 for the mixed path (fastest of each, measured)")
    ap.add_argument("--accuracy", type=int, default=1, help="1: report errors against the FP64 all-pairs solve")
    ap.add_argument("--inner-tol-exp", type=int, default=0, help="mixed: inner GMRES tolerance 10^-x (0: default)")
    ap.add_argument("--mixed-near", type=int, default=0, help="mixed near apply: 0 TF32 tensor cores, 1 FP32 CUDA cores")
    ap.add_argument("--m2l-mode", type=int, default=0, help="0 QR-compressed M2L operators (reference), 1 exact")
    ap.add_argument("--mixed-m2l", type=int, default=3,
                    help="mixed M2L: 0 auto, 1 factored on CUDA cores, 2 tensor cores also with Gauss sources, "
                         "3 shared rank-64 basis on the tensor cores (fastest, measured)")
    ap.add_argument("--mixed-far-tc", type=int, default=1,
                    help="mixed: 1 P2M and L2P on the tensor cores (hi/lo split operands), 2 P2M only, "
                         "0 FP32 CUDA cores")
    ap.add_argument("--workload", default="window64", choices=["window64", "twowires", "batch", "bus", "block"],
                    help="window64: the headline 64-net window; twowires: two met1 wires on a 0.05 um mesh; "
                         "batch: many uneven windows in one batched call; bus: met2 bus sensitivities; "
                         "block: 200 um, 6-layer, 512-net block with layer-parameter gradients (mixed)")
    ap.add_argument("--windows", type=int, default=256, help="batch workload: number of windows")
    ap.add_argument("--block-nets", type=int, default=512, help="block workload: nets")
    ap.add_argument("--block-side", type=float, default=200.0, help="block workload: side in um")
    ap.add_argument("--block-part", default="both", choices=["both", "capacitance", "gradients"],
                    help="block workload: time the capacitance solve, the solve with gradients, or both")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel directly (no CUDA graphs, no device-side Arnoldi loop); for profilers "
                         "that list kernel launches")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class DeviceMemoryWatch:
    """High-water mark of device memory in use (total - free, cudaMemGetInfo on
    device 0) sampled every 20 ms by a thread while the block runs; catches
    the library's stream-ordered allocations, which torch's counters miss."""

    def __enter__(self):
        import torch

        self.torch = torch
        self.peak_used = 0
        self.stop = threading.Event()
        self.t = threading.Thread(target=self._run, daemon=True)
        self._sample()
        self.t.start()
        return self

    def _sample(self):
        free, total = self.torch.cuda.mem_get_info(0)
        self.peak_used = max(self.peak_used, total - free)

    def _run(self):
        while not self.stop.wait(0.02):
            self._sample()

    def __exit__(self, *exc):
        self.stop.set()
        self.t.join()
        self._sample()
        return False


def load_peaks():
    """Measured peaks of this pool's B200s (driver-written MEASURED_PEAKS.json):
    HBM copy GB/s, and dense bf16 TFLOP/s as a burst and sustained under the
    power cap; else the fallback figures."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm": float(d["hbm_gbs"]), "bf16": float(d["bf16_tflops"]),
                "bf16_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "kind": "measured"}
    except Exception:
        return {"hbm": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0, "kind": "fallback"}


def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """The job's time is the slowest rank's: all-reduce MAX (no-op alone)."""
    if not dist:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(rank: int, nets: int, side: float = 40.0):
    from gpurify_b200 import layouts

    return layouts.routing_window(nets, side, seed=2024 + rank)


def entry_errors(C, ref):
    """Errors of a Maxwell matrix against a reference: every entry relative to
    itself, every entry relative to its row's diagonal, and entry-wise over the
    entries at least 1e-3 of their row's diagonal."""
    import numpy as np

    d = np.abs(np.diag(ref))[:, None]
    err = np.abs(C - ref)
    rel = err / np.maximum(np.abs(ref), 1e-300)
    coupled = np.abs(ref) >= 1e-3 * d
    return {"entrywise": float(rel.max()), "diag_normalised": float((err / d).max()),
            "entrywise_coupled": float(rel[coupled].max())}


def oracle_window(nets: int, side: float, rank: int = 0):
    """The bench window panelised by the oracle's own restatement of the
    reference bridge (bit-identical to the library's panels), so that the CPU
    legs load nothing of the product library."""
    import oracle

    lay = workload(rank, nets, side)
    p = oracle.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0,
                               mesh_max_edge_m=EDGE_M, max_panels=-1)
    return lay, p


def spread_columns(R: int, k: int, start: int = 0):
    """k conductor columns spread over the R nets (a stride coprime to R)."""
    stride = next(s for s in (R // k + 1, R // k + 3, 13, 17, 1) if s > 0 and gcd(s, R) == 1)
    return [(start + i * stride) % R for i in range(k)]


def gcd(a: int, b: int) -> int:
    while b:
        a, b = b, a % b
    return a


def cpu_columns(p, ncond, R, order, depth, threads, cols):
    """The oracle (the reference's CPU field solver restated,
    cap/fmm_solver.rs:147-172) on the window: operator and Jacobi
    preconditioner built once, then one timed GMRES solve per sampled
    conductor column.  A full extraction is the set-up plus R times the mean
    column time (the reference solves the R conductors one after another)."""
    import oracle

    sv = oracle.FmmSolver(p["verts"], p["cond"], ncond, order=order, max_level=depth, threads=threads)
    times, its = [], []
    try:
        for j in cols:
            t0 = time.perf_counter()
            _, r = sv.solve_column(j, tol=1e-8, restart=200, max_restarts=50)
            times.append(time.perf_counter() - t0)
            its.append(r["iterations"])
    finally:
        sv.close()
    return sv.t_setup_s, times, its


def config1_cpu(threads_all: int):
    """Config 1 exactly as the reference runs it: two met1 wires on the
    reference bridge mesh (513 panels incl. the substrate plate, so the FMM
    path), FMM order 4 / depth 4, diagonal Jacobi, GMRES 1e-8, every conductor
    (cap/fmm_solver.rs:147-172, bridge.rs:403) -- timed single-thread and on
    all host threads."""
    import oracle
    from gpurify_b200 import layouts

    lay = layouts.two_wires()
    p = oracle.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), lay.net_of_poly, 1.0)
    nc = len(p["nets"]) + 1
    out = {"workload": "two met1 wires 0.14x0.36x20 um, 0.14 um spacing, reference bridge mesh",
           "panels": int(len(p["verts"])), "rhs": nc, "mode": "reference (FMM order 4 depth 4, Jacobi, tol 1e-8)"}
    for th in (1, threads_all):
        reps = []
        for _ in range(3):
            t0 = time.perf_counter()
            oracle.cap_fmm(p["verts"], p["cond"], nc, order=4, max_level=4, tol=1e-8, threads=th)
            reps.append(time.perf_counter() - t0)
        out[f"threads_{th}"] = {"solves_per_s": 1.0 / statistics.median(reps), "ms": 1e3 * statistics.median(reps)}
    return out


def config1_gpu(ctx):
    """Config 1 on the GPU in the reference's own mode (the same mesh, FMM
    order 4 / depth 4, diagonal Jacobi, tol 1e-8, every conductor incl. the
    substrate), FP64: median device-synchronised time of 5 solves after 2
    warm-up solves."""
    import torch

    from gpurify_b200 import _lib, layouts

    lay = layouts.two_wires()
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)
    nc = len(p["nets"]) + 1
    kw = dict(order=4, max_level=4, tol=1e-8, precond=0, far_quad=0, precision=_lib.PREC_FP64)
    for _ in range(2):
        ctx.cap_solve(p["verts"], p["cond"], nc, **kw)
    reps = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, rep = ctx.cap_solve(p["verts"], p["cond"], nc, **kw)
        torch.cuda.synchronize()
        reps.append(time.perf_counter() - t0)
    return {"solves_per_s": 1.0 / statistics.median(reps), "ms": 1e3 * statistics.median(reps),
            "iterations": rep["iterations"]}


def cpu_baseline(p, ncond, R, order, depth, threads, nsample=4):
    """CPU baseline of the GPU arm: the oracle on the same window, set-up plus
    `nsample` conductor columns spread over the nets (about 15-20 s on 16
    host threads), scaled to the R columns of a full extraction."""
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    cols = spread_columns(R, nsample)
    t_setup, times, its = cpu_columns(p, ncond, R, order, depth, cores, cols)
    per = sum(times) / len(times)
    total = t_setup + R * per
    return {"value": 1.0 / total, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"oracle FMM(order {order}, depth {depth}) on the same {len(p['verts'])}-panel window: operator "
                      f"set-up {t_setup:.2f} s, then {len(cols)} of the {R} conductor columns (nets {cols}) "
                      f"{per:.2f} s each ({min(its)}-{max(its)} GMRES iterations); a full extraction = set-up + "
                      f"{R} x the mean column time = {total:.1f} s",
            "panel_rhs_per_s": len(p["verts"]) * R / total, "t_setup_s": t_setup, "t_column_s": times,
            "sample_columns": cols, "measured_s": t_setup + sum(times)}


def run_reference(args, rank, world):
    """Reference arm: the oracle (the reference's CPU field solver restated in
    C++; the reference itself is Rust and cannot be built here) on the bench
    window, all host threads, nothing of the product library loaded.  The
    operator set-up is timed once before the warm-up; every step is then one
    conductor column's GMRES solve (a bounded sample of the full extraction),
    the steps cycling through columns spread over the nets.  value = 1 /
    (set-up + R x mean step time)."""
    if rank != 0:
        return
    import oracle

    lay, p = oracle_window(args.nets, args.side)
    ncond = len(p["nets"]) + 1
    R = len(p["nets"])
    cores = args.cpu_threads if args.cpu_threads > 0 else (os.cpu_count() or 1)
    cols = spread_columns(R, args.warmup + args.steps)
    sv = oracle.FmmSolver(p["verts"], p["cond"], ncond, order=args.order, max_level=args.depth, threads=cores)
    t_setup = sv.t_setup_s
    times, its = [], []
    try:
        for i, j in enumerate(cols):
            t0 = time.perf_counter()
            _, r = sv.solve_column(j, tol=1e-8, restart=200, max_restarts=50)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
                its.append(r["iterations"])
    finally:
        sv.close()
    per = sum(times) / len(times)
    total = t_setup + R * per
    v = 1.0 / total
    timed_cols = cols[args.warmup:]
    sample = (f"oracle FMM(order {args.order}, depth {args.depth}) on the {len(p['verts'])}-panel window, {cores} "
              f"threads: operator set-up {t_setup:.2f} s (timed once), then {len(times)} timed conductor columns "
              f"(nets {timed_cols}) of {per:.2f} s mean ({min(its)}-{max(its)} GMRES iterations); a full extraction "
              f"= set-up + {R} x the mean column = {total:.1f} s")
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded routing window)",
           "config": {"workload": f"routing window {args.nets} nets {args.side:g}x{args.side:g}um 3 layers, "
                                  f"{len(p['verts'])} panels, {R} RHS, GMRES tol 1e-8, FMM order {args.order} "
                                  f"depth {args.depth}",
                      "panels": len(p["verts"]), "rhs": R,
                      "step": "one conductor column's GMRES solve (1/R of an extraction)"},
           "panel_rhs_per_s": len(p["verts"]) * R / total,
           "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
           "extrapolation": {"t_setup_s": t_setup, "t_column_mean_s": per, "columns_timed": len(times),
                             "columns_per_extraction": R},
           "config1": config1_cpu(cores),
           "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def time_solves(ctx, verts, cond, ncond, solve_kw, steps, warmup, stream, dist, local):
    """Warm-up, then EXACTLY `steps` timed solves between a barrier and
    device synchronisation, timed with CUDA events on the context stream
    (operator applies replayed from captured CUDA graphs, no per-kernel
    timing).  Then the same solves once more with per-kernel CUDA-event
    timing on (direct launches) for the kernel breakdown and the roofline."""
    import torch

    reps = []
    for _ in range(warmup):
        ctx.cap_solve(verts, cond, ncond, **solve_kw)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    # let nvidia-smi start up (its first sample) before the timed region: the
    # solver builds its octree on the host, and a process starting beside it
    # would slow the first timed solve
    t_wait = time.perf_counter()
    while sampler.proc and not sampler.lines and time.perf_counter() - t_wait < 3.0:
        time.sleep(0.02)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    C = None
    for _ in range(steps):
        C, rep = ctx.cap_solve(verts, cond, ncond, **solve_kw)
        reps.append(rep)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    ms = max_over_ranks(ms, dist)
    ctx.set_profiling(True)
    ctx.reset_stats()
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.cap_solve(verts, cond, ncond, **solve_kw)
    torch.cuda.synchronize()
    ms_prof = (time.perf_counter() - t0) * 1e3
    ks = ctx.kernel_stats()
    ctx.set_profiling(False)
    launches = sum(r["kernel_launches"] for r in reps)
    return ms, reps, ks, clocks, C, launches, ms_prof


# DRAM bytes per launch measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, one --set full capture of two launches of each
# kernel on this bench window, cold cache) divided by the launch's
# algorithmic bytes as this bench counts them (near apply: 4 B per stored
# near entry plus 16 B per panel and right-hand side; M2L: each box's
# expansion read once and its local expansion written once).  bench scales
# the ratio by the algorithmic bytes of the launches it times.
TRAFFIC_PER_ALGO_BYTE = {"near_apply": 1.163, "m2l": 0.968,
                         # shared-basis M2L: compress + 64 x 64 cores + decompress per apply
                         "m2l_shared": 1.151}


def roofline_of(ks, ms_total, m2l_engine, shared_m2l=False):
    """Roofline of the kernel class with the largest device time, the classes
    split by precision (the mixed path's FP32/TF32 launches apart from its
    FP64 refinement residuals).  M2L is measured as a dense contraction
    against the sustained bf16 tensor peak (the kernel runs inside a solve of
    hundreds of milliseconds; its algorithmic flops are the dense-equivalent
    2 (n^3)^2 R per box pair, counted the same whether or not the operators
    are compressed); every other class as algorithmic bytes against the HBM
    copy peak."""
    pk = load_peaks()
    names = [k for k in ks if k != "total_launches"]
    top = max(names, key=lambda k: ks[k]["ms"])
    k = ks[top]
    per_launch_ms = k["ms"] / max(1, k["launches"])
    src = "measured (MEASURED_PEAKS.json)" if pk["kind"] == "measured" else "fallback"
    algo_bytes = k["bytes"] / max(1, k["launches"])
    traffic = TRAFFIC_PER_ALGO_BYTE.get("m2l_shared" if (top == "m2l" and shared_m2l) else top)
    common = {"kernel": top, "peak_source": src,
              "traffic": traffic * algo_bytes if traffic else None, "launches": k["launches"],
              "ms_per_launch": per_launch_ms, "share_of_step": k["ms"] / ms_total if ms_total > 0 else None}
    if top in ("m2l", "m2l_f64"):
        ach = k["flops"] / max(1, k["launches"]) / (per_launch_ms * 1e-3) / 1e12
        return dict(bound="tensor", achieved=ach, peak=pk["bf16_sustained"], unit="TFLOP/s",
                    frac=ach / pk["bf16_sustained"], peak_kind="bf16 dense, sustained", engine=m2l_engine, **common)
    ach = algo_bytes / (per_launch_ms * 1e-3) / 1e9
    return dict(bound="hbm", achieved=ach, peak=pk["hbm"], unit="GB/s", frac=ach / pk["hbm"],
                flops_per_s=k["flops"] / max(1, k["launches"]) / (per_launch_ms * 1e-3), **common)


def run_workload(args):
    """The other workloads, one JSON line each (not the headline line): two
    wires on a 0.05 um mesh, a batch of uneven windows through
    gpx_cap_solve_batched, the met2-bus sensitivities, and the large block
    (mixed precision; gradients along the 6 layers' thickness and height and
    k, reported for 16 seeded nets)."""
    import numpy as np
    import torch

    from gpurify_b200 import _lib, layouts, pex, sensitivity

    torch.cuda.set_device(0)
    ctx = _lib.Context(0)
    base = dict(order=args.order, max_level=-1, far_quad=args.far_quad, skip_ground_rhs=1, mixed_m2l=args.mixed_m2l)
    out = {"workload": args.workload, "data": "synthetic (seeded layouts)"}

    def timed(fn, reps, warm=True):
        if warm:  # one untimed call first (the large block skips it: one solve takes minutes)
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            r = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps, r

    if args.workload == "twowires":
        lay = layouts.two_wires()
        p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                 mesh_max_edge_m=0.05e-6, max_panels=-1)
        nc = len(p["nets"]) + 1
        Cd, _ = ctx.cap_solve(p["verts"], p["cond"], nc, dense_below=2**31 - 1, skip_ground_rhs=1, tol=1e-10,
                              precond=1)
        out.update(panels=len(p["verts"]), rhs=nc - 1)
        for prec, pc in (("fp64", 2), ("mixed", 1)):
            kw = dict(base, precision=_lib.PREC_MIXED if prec == "mixed" else _lib.PREC_FP64, precond=pc)
            kw, trep = ctx.autotune(p["verts"], p["cond"], nc, target=1e-4, **kw)
            dt, (C, rep) = timed(lambda: ctx.cap_solve(p["verts"], p["cond"], nc, **kw), max(1, args.steps))
            d = np.abs(np.diag(Cd[:2, :2]))
            out[prec] = {"solves_per_s": 1.0 / dt, "ms": dt * 1e3, "iterations": rep["iterations"],
                         "tuned": {k: kw[k] for k in ("order", "max_level", "far_quad", "mixed_near")},
                         "err_vs_all_pairs": float((np.abs(C[:2, :2] - Cd[:2, :2]) / d[:, None]).max()),
                         "cap_af": [float(C[i, i] * 3.9e18) for i in range(2)]}
    elif args.workload == "batch":
        ws = layouts.window_batch(args.windows, seed=7)
        probs = []
        for w in ws:
            p = _lib.bridge_panelize(w.store.arrays(), w.deck.layer_table(), 1.0, w.net_of_poly,
                                     mesh_max_edge_m=EDGE_M, max_panels=-1)
            probs.append((p["verts"], p["cond"], len(p["nets"]) + 1))
        N = sum(len(v) for v, _, _ in probs)
        RR = sum(nc - 1 for _, _, nc in probs)
        NR = sum(len(v) * (nc - 1) for v, _, nc in probs)
        out.update(windows=len(probs), panels=N, rhs=RR, panel_rhs=NR)
        kw = dict(base, precision=_lib.PREC_MIXED, precond=1, batch_streams=8)
        dt, res = timed(lambda: ctx.cap_solve_batched(probs, **kw), 1)
        out["mixed"] = {"windows_per_s": len(probs) / dt, "s": dt, "panel_rhs_per_s": NR / dt,
                        "max_iterations": max(r["iterations"] for _, r in res),
                        "kernel_launches": int(sum(r["kernel_launches"] for _, r in res)),
                        "timing": "wall clock around the synchronous batched call (8 streams)"}
    elif args.workload == "block":
        lay = layouts.large_block(n_nets=args.block_nets, side_um=args.block_side)
        p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                 mesh_max_edge_m=0.8e-6, max_panels=-1)
        nc = len(p["nets"]) + 1
        spans = [sensitivity.layer_span(lay.deck, name) for name, *_ in layouts.BLOCK_LAYERS]
        params = [("thickness", z0, z1) for z0, z1 in spans] + [("height", z0, z1) for z0, z1 in spans] + [("k",)]
        V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
        rows = sorted(int(r) for r in np.random.default_rng(16).choice(nc - 1, min(16, nc - 1), replace=False))
        out.update(panels=len(p["verts"]), rhs=nc - 1, params=len(params), gradient_nets=rows)
        # FP32 inner basis: twice the restart length in the memory left beside
        # the 53 GB of near blocks (GMRES(20) stalls on this problem)
        kw = dict(base, precision=_lib.PREC_MIXED, precond=1, inner_basis32=1)
        free0, total = torch.cuda.mem_get_info(0)
        out["mixed"] = {"device_bytes_total": int(total),
                        "memory_sampling": "free device memory sampled every 20 ms during the call"}
        if args.block_part in ("both", "capacitance"):
            with DeviceMemoryWatch() as mw:
                dt0, (C, rep) = timed(lambda: ctx.cap_solve(p["verts"], p["cond"], nc, **kw), 1, warm=False)
            out["mixed"].update(ms_capacitance_only=dt0 * 1e3, iterations=rep["iterations"],
                                outer_iterations=rep["outer_iterations"], converged=bool(rep["converged"]),
                                restart_used=rep["restart_used"], panel_rhs_per_s=len(p["verts"]) * (nc - 1) / dt0,
                                peak_device_bytes_solve=int(mw.peak_used - (total - free0)),
                                near_pairs=int(rep["nnz_near"]), depth=int(rep["max_level"]))
            print(json.dumps(dict(out, part="capacitance")), flush=True)
        if args.block_part in ("both", "gradients"):
            with DeviceMemoryWatch() as mw:
                dt, (_, dC, rep2) = timed(lambda: ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, grad_rows=rows,
                                                                      **kw), 1, warm=False)
            out["mixed"].update(ms_capacitance_plus_gradients=dt * 1e3,
                                iterations_forward_plus_adjoint=rep2["iterations"],
                                near_pairs=int(rep2["nnz_near"]), depth=int(rep2["max_level"]),
                                max_abs_dC_of_gradient_nets=float(np.abs(dC[:, rows, :nc - 1]).max()),
                                finite_gradient_rows=bool(np.isfinite(dC[:, rows, :nc - 1]).all()),
                                peak_device_bytes_gradients=int(mw.peak_used - (total - free0)))
    else:  # bus
        lay = layouts.bus_crossing()
        z0, z1 = sensitivity.layer_span(lay.deck, "met2")
        params = [("width", b) for b in range(8)] + [("spacing", b) for b in range(7)] + \
                 [("thickness", z0, z1), ("height", z0, z1), ("k",)]
        p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                                 mesh_max_edge_m=0.14e-6, max_panels=-1)
        V = sensitivity.velocity_fields(p["verts"], p["cond"], p["nets"], params)
        nc = len(p["nets"]) + 1
        out.update(panels=len(p["verts"]), rhs=nc - 1, params=len(params))
        grads = {}
        for prec, pc in (("fp64", 2), ("mixed", 1)):
            kw = dict(base, precision=_lib.PREC_MIXED if prec == "mixed" else _lib.PREC_FP64, precond=pc)
            kw, trep = ctx.autotune(p["verts"], p["cond"], nc, target=1e-4, **kw)
            dt, (C, dC, rep) = timed(lambda: ctx.cap_sensitivity(p["verts"], p["cond"], nc, V, **kw),
                                     max(1, args.steps))
            dt0, _ = timed(lambda: ctx.cap_solve(p["verts"], p["cond"], nc, **kw), max(1, args.steps))
            grads[prec] = dC
            out[prec] = {"ms_capacitance_plus_gradients": dt * 1e3, "ms_capacitance_only": dt0 * 1e3,
                         "tuned": {k: kw[k] for k in ("order", "max_level", "far_quad", "mixed_near")},
                         "iterations_forward_plus_adjoint": rep["iterations"]}
        R = nc - 1
        a, b = grads["mixed"][:, :R, :R], grads["fp64"][:, :R, :R]
        out["mixed_vs_fp64_gradient"] = float(np.abs(a - b).max() / np.abs(b).max())
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.workload != "window64":
        run_workload(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from gpurify_b200 import _lib, pex

    ctx = _lib.Context(local)
    base_kw = dict(order=args.order, max_level=args.depth, skip_ground_rhs=1, tol=1e-8, restart=args.restart,
                   far_quad=args.far_quad, precond=args.precond, inner_tol_exp=args.inner_tol_exp,
                   mixed_near=args.mixed_near, m2l_mode=args.m2l_mode, mixed_m2l=args.mixed_m2l,
                   mixed_far_tc=args.mixed_far_tc, no_graphs=1 if args.no_graphs else 0)
    precisions = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    lay = workload(rank, args.nets, args.side)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly,
                             mesh_max_edge_m=EDGE_M, max_panels=-1)
    N = len(p["verts"])
    ncond = len(p["nets"]) + 1
    R = ncond - 1
    verts = torch.from_numpy(p["verts"]).pin_memory().numpy()
    cond = torch.from_numpy(p["cond"]).pin_memory().numpy()
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    runs = {}
    for prec in precisions:
        kw = dict(base_kw, precision=_lib.PREC_MIXED if prec == "mixed" else _lib.PREC_FP64)
        if args.precond < 0:
            kw["precond"] = 1 if prec == "mixed" else 2
        ms, reps, ks, clocks, C, launches, ms_prof = time_solves(ctx, verts, cond, ncond, kw, args.steps,
                                                                 args.warmup, stream, dist, local)
        runs[prec] = dict(ms=ms, reps=reps, ks=ks, clocks=clocks, C=C, kw=kw, launches=launches, ms_prof=ms_prof)
    head = precisions[-1]
    hr = runs[head]
    ms_step = hr["ms"] / args.steps
    value = world * 1e3 / ms_step

    # end to end through the public per-net API (layout polygons -> per-net aF)
    e2e_times, e2e_rep = [], {}
    for _ in range(max(2, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pex.run_pex_by_net_checked(lay.store, lay.deck, lay.net_of_poly, ctx=ctx, report=e2e_rep,
                                   mesh_max_edge_m=EDGE_M, max_panels=-1, **hr["kw"])
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_times) / len(e2e_times)
    e2e_s = max_over_ranks(e2e_s, dist)

    accuracy = None
    if args.accuracy and rank == 0:
        # FP64 all-pairs reference (every entry by the exact Wilton integral),
        # GMRES to 1e-10; errors normalised by the row's diagonal entry.
        Cd, _ = ctx.cap_solve(verts, cond, ncond, dense_below=2**31 - 1, skip_ground_rhs=1, tol=1e-10,
                              precond=max(args.precond, 1))
        Cn = Cd[:R, :R]
        accuracy = {"reference": "FP64 all-pairs Wilton operator (every pair exact), GMRES tol 1e-10",
                    "diag_normalised": "max_ij |C_ij - Cref_ij| / |Cref_ii|",
                    "entrywise": "max_ij |C_ij - Cref_ij| / |Cref_ij|",
                    "entrywise_coupled": "the same over entries with |Cref_ij| >= 1e-3 |Cref_ii|"}
        for prec, rr in runs.items():
            accuracy[prec] = entry_errors(rr["C"][:R, :R], Cn)
        if "mixed" in runs and "fp64" in runs:
            accuracy["mixed_vs_fp64"] = entry_errors(runs["mixed"]["C"][:R, :R], runs["fp64"]["C"][:R, :R])

    if rank == 0:
        shared_m2l = head == "mixed" and args.mixed_m2l == 3 and args.order in (5, 6)
        tc_m2l = head == "mixed" and args.order in (4, 5) and args.mixed_m2l != 1 and (
            args.far_quad == 0 or args.m2l_mode == 1 or args.mixed_m2l >= 2)
        if shared_m2l:
            engine = ("tcgen05 TF32 on the 64 x 64 shared-basis cores, with tcgen05 hi/lo compress and "
                      "decompress; flops counted as the dense-equivalent full operators")
        elif tc_m2l:
            engine = "tcgen05 TF32"
        else:
            engine = ("FP32 CUDA cores, factored low-rank operators" if head == "mixed" else
                      "FP64 CUDA cores, factored low-rank operators")
        roof = roofline_of(hr["ks"], hr["ms_prof"], engine, shared_m2l)
        names = [k for k in hr["ks"] if k != "total_launches"]
        breakdown = {n: {"ms_per_step": hr["ks"][n]["ms"] / args.steps,
                         "launches_per_step": hr["ks"][n]["launches"] / args.steps}
                     for n in names if hr["ks"][n]["launches"]}
        cb = None
        if not args.no_cpu_baseline:
            cb = cpu_baseline(p, ncond, R, args.order, args.depth, args.cpu_threads)
            cb = {k2: cb[k2] for k2 in ("value", "unit", "cores", "kind", "sample", "measured_s")}
            cb["config1"] = config1_cpu(cb["cores"])
            cb["config1"]["gpu_fp64_reference_mode"] = config1_gpu(ctx)
        per_prec = {}
        for prec, rr in runs.items():
            msp = rr["ms"] / args.steps
            per_prec[prec] = {"solves_per_s": world * 1e3 / msp, "ms_per_step": msp,
                              "panel_rhs_per_s": world * N * R / (msp * 1e-3),
                              "iterations": rr["reps"][-1]["iterations"],
                              "outer_iterations": rr["reps"][-1]["outer_iterations"],
                              "max_rel_residual": rr["reps"][-1]["max_rel_residual"]}
        out = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64 (FP64 refinement)",
            "data": "synthetic (seeded 64-net routing window; no public layout used)",
            "config": {"workload": f"routing window {args.nets} nets {args.side:g}x{args.side:g}um 3 layers, 0.25um "
                                   f"panels, {N} panels, {R} RHS, GMRES tol 1e-8",
                       "panels": N, "rhs": R, "precision": head, "order": args.order, "depth": args.depth,
                       "far_quad": args.far_quad, "restart": args.restart,
                       "precond": {pr: runs[pr]["kw"]["precond"] for pr in runs},
                       "mixed_m2l": args.mixed_m2l, "mixed_far_tc": args.mixed_far_tc,
                       "parallelism": f"replicas x{world}", "l2": "working set (Krylov basis > 1 GB) >> L2"},
            "panel_rhs_per_s": world * N * R / (ms_step * 1e-3),
            "precisions": per_prec,
            "speedup_mixed_vs_fp64": (per_prec["mixed"]["solves_per_s"] / per_prec["fp64"]["solves_per_s"]
                                      if "mixed" in per_prec and "fp64" in per_prec else None),
            "accuracy": accuracy,
            "gpu_launches": hr["launches"],
            "roofline": roof, "kernel_breakdown": breakdown,
            "cpu_baseline": cb, "clocks": hr["clocks"],
            "e2e": {"value": world / e2e_s, "unit": "solves/s", "api": "run_pex_by_net_checked",
                    "h2d_bytes_per_step": int(e2e_rep.get("h2d_bytes", 0)),
                    "d2h_bytes_per_step": int(e2e_rep.get("d2h_bytes", 0)),
                    "t_panelize_s": e2e_rep.get("t_panelize_s")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
