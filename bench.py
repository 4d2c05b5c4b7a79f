"""Benchmark: cell-RK-stage updates/s of the DNDS residual-evaluation path on B200.

Workload: the 2-D isentropic vortex on a periodic [0,10]^2 1024x1024 grid whose
interior nodes are jittered by U(-0.2h, 0.2h) (seed 1234), each quad split into
2 triangles (2,097,152 cells); P2 variational reconstruction (one Jacobi sweep
per stage), Roe flux, SSP-RK3 at CFL 0.5 with a global time step.  One "step"
is one SSP-RK3 step = 3 cell-RK-stage updates of every cell.  The headline
`value` is the FP32-bulk path (FP64 cell means, dt and norms); the plain FP64
path is timed beside it.  Synthetic data generated here; no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dnds_b200|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs an independent
replica (the reference partitions the mesh with MPI halos; this implementation runs
one mesh per GPU), and `value` is the sum over ranks (weak scaling).
`--impl reference` times the FP64 CPU restatement of the reference (oracle/)
on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-RK-stage updates/s: FP32+learned VR vs plain FP64 at equal L2 error, 1 B200"
UNIT = "cell-stage updates/s"
WORKLOAD = "isentropic vortex, periodic [0,10]^2, 1024x1024 jittered quads -> 2,097,152 triangles, P2 VR + Roe, SSP-RK3 CFL 0.5"
N_GRID = 1024
# algorithmic bytes per triangle cell of one VR Jacobi sweep: read urec 20s, A^-1B 75s, A^-1b 15s,
# write urec 20s (s = bytes per real), cell means 4x8, 3 neighbour indices 3x4
VR_BYTES_PER_CELL = {4: 130 * 4 + 32 + 12, 8: 130 * 8 + 32 + 12}
KERNELS_PER_STEP = 13  # init, 3 x (VR, flux, update) with dt cell and dt finalize after the first flux, time advance
# algorithmic bytes per triangle cell of one whole SSP-RK3 step: 3 stages x (VR sweep, face flux with
# 1.5 faces per cell (the compact basis record 18s, normal / length / dLambda / indices ~40 B, flux out
# 32 B) plus the cell's coefficients 20s and means 32 B once, cell update 136 B) + EvaluateDt ~74 B.
# FP32 bulk 3 x (564 + 328 + 136) + 74 = 3158 B, FP64 3 x (1084 + 516 + 136) + 74 = 5282 B: at equal
# HBM efficiency the FP32-bulk step can be at most 5282 / 3158 = 1.67 times faster
STEP_BYTES_PER_CELL = {4: 3 * (564 + 328 + 136) + 74, 8: 3 * (1084 + 516 + 136) + 74}
# DRAM bytes (read + write) per launch of the FP32 VR sweep: ncu --metrics dram__bytes_read.sum,
# dram__bytes_write.sum --clock-control none on one k_vr_tma4<float,32,3> launch over the 512x512 version of
# this mesh (524,288 cells; 291.23 MB read + written, 555 B per cell against the 564 B algorithmic), scaled by
# the cell count (x4) to this workload: the working set exceeds L2 at both sizes, so traffic is per cell
VR_TRAFFIC_FP32 = 291.23e6 * 4


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank scalar over all ranks (identity without torch.distributed)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(n_cells: int, steps: int, ms_max: float, world: int) -> float:
    """Whole-job cell-stage updates/s of `world` independent replicas timed by the slowest rank."""
    return n_cells * 3 * steps / (ms_max * 1e-3) * world


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms over the FP32 leg (warm-up, the
    timed steps, the per-kernel timings, the end-to-end loop and the accuracy run): the timed region
    itself is tens of milliseconds, shorter than the sampling interval, and runs the same kernels."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu_index), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(max_seconds=12.0):
    """The FP64 CPU oracle on a bounded sample of the workload (512x512 grid -> 524,288 triangles)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S

    pyoracle.build()
    cores = os.cpu_count() or 1
    m = M.vortex_mesh(512, True, jitter=0.2, seed=1234)
    o = pyoracle.Oracle(m, S.preset("vortex"), n_threads=cores)
    o.set_u(G.isentropic_vortex(m))
    steps = 0
    t = 0.0
    t0 = time.perf_counter()
    while True:
        _, d = o.eval_dt(0.5)
        o.ssprk3_step(d, t)
        t += d
        steps += 1
        el = time.perf_counter() - t0
        if el > max_seconds or steps >= 200:
            break
    v = m.n_cells * 3 * steps / el
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"FP64 oracle, {steps} SSP-RK3 steps on the 512x512 (524,288-triangle) version of the workload, "
                      f"{el:.1f} s, {cores} threads"}


REF_BUDGET_S = 240.0  # wall-clock target of the whole reference arm


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    pyoracle.build()
    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S

    cores = os.cpu_count() or 1
    # each step runs the full workload (1024 x 1024 x 2 = 2,097,152 triangles, about 2 s per step on 16
    # host threads) when the whole --warmup W --steps K run fits in about REF_BUDGET_S, from the cost of one
    # calibration step; with more steps than that the mesh shrinks to a bounded sample of the workload
    cal = M.vortex_mesh(128, True, jitter=0.2, seed=1234)
    oc = pyoracle.Oracle(cal, S.preset("vortex"), n_threads=cores)
    oc.set_u(G.isentropic_vortex(cal))
    _, d = oc.eval_dt(0.5)
    oc.ssprk3_step(d, 0.0)
    t0 = time.perf_counter()
    _, d = oc.eval_dt(0.5)
    oc.ssprk3_step(d, 0.0)
    per_cell = (time.perf_counter() - t0) / cal.n_cells
    del oc
    cells = REF_BUDGET_S / max(args.steps + args.warmup, 1) / max(per_cell, 1e-12)
    n = int(max(32, min(N_GRID, (cells / 2) ** 0.5)))
    m = M.vortex_mesh(n, True, jitter=0.2, seed=1234)
    o = pyoracle.Oracle(m, S.preset("vortex"), n_threads=cores)
    o.set_u(G.isentropic_vortex(m))
    t = 0.0
    for _ in range(args.warmup):
        _, d = o.eval_dt(0.5)
        o.ssprk3_step(d, t)
        t += d
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, d = o.eval_dt(0.5)
        o.ssprk3_step(d, t)
        t += d
    el = time.perf_counter() - t0
    v = m.n_cells * 3 * args.steps / el
    out = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / max(args.steps, 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": m.n_cells, "parallelism": "host threads",
                   "same_mesh_as_gpu_arm": n == N_GRID,
                   "note": "FP64 CPU restatement of the reference (the reference needs Eigen/MPI/METIS, absent here); "
                           f"each step runs the {n}x{n}x2 = {m.n_cells:,}-triangle mesh"
                           + (" of the workload" if n == N_GRID else ", a sample of the workload sized so that the "
                              "run ends within minutes; the metric is per cell")},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} timed SSP-RK3 steps on {m.n_cells:,} triangles, {cores} threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


STEADY_RAMP = dict(cfl=100.0, cfl_ramp_start=100, cfl_ramp_length=1000, cfl_ramp_end=1000.0)
STEADY_PARTS = 16  # the partitioned sweep: the reference on 16 ranks (contiguous blocks of the cell order)


def steady_leg(dev, iters=10000, log=None):
    """The implicit steady RANS-SA path on the 512 x 128 NACA 0012 C-mesh (first spacing 1e-6 chord, far
    field 20 chords, no-slip wall), M 0.15, alpha 10 deg, Re 6e6, SA variable 3x the laminar viscosity in
    the free stream: first-order BDF pseudo time, LU-SGS in the reference's natural scan order
    (level-scheduled), CFL 100 ramped log-linearly to 1000 over iterations 100-1100 (the fstop ramp),
    one C call per run (dndsg_steady_solve).  Reported: ms per pseudo-time iteration (CUDA events),
    the density increment ratio of fstop after `iters` iterations and CL / CD from the wall force, in
    FP64 and FP32 bulk, with the sweep in one part (the reference on one rank) and in STEADY_PARTS
    parts (the reference on that many ranks: each part sweeps its own cells, one level walk per part
    on the GPU); the colour-batched sweep's ms per iteration (it does not converge on these stretched
    cells); the oracle's iteration time on the host cores.  The full convergence to the 1e-8 drop
    takes about 222,000 iterations (python bench.py --steady-full).  Timed outside the headline."""
    import math

    import torch

    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.naca0012_cmesh()
    cfg = S.preset("naca0012_sa")
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    a = math.radians(10.0)
    out = {"workload": "RANS-SA NACA 0012, C-mesh 512x128 (65,536 quads), first spacing 1e-6 chord, M 0.15, "
                       "alpha 10, Re 6e6, BDF1 pseudo time, CFL 100 ramped to 1000, 5 variables",
           "cells": m.n_cells, "iterations": iters}
    from dnds_b200.partition import block_owner

    for prec, name, parts in ((0, "fp64", 1), (1, "fp32", 1), (0, f"fp64_parts{STEADY_PARTS}", STEADY_PARTS),
                              (1, f"fp32_parts{STEADY_PARTS}", STEADY_PARTS)):
        s = Solver(m, cfg, device=dev, precision=prec)
        s.lusgs_set_order(1)
        if parts > 1:
            s.lusgs_set_parts(block_owner(m.n_cells, parts), parts)
        s.set_u(u0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        it, rel, wf, _ = s.steady_run(threshold=1e-8, max_iter=iters, **STEADY_RAMP)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        r = {"iterations": it, "seconds": ms * 1e-3, "ms_per_iteration": ms / it,
             "cell_iterations_per_s": m.n_cells * it / (ms * 1e-3), "rel_residual_rho": float(rel[0]),
             "CL": float((-wf[1] * math.sin(a) + wf[2] * math.cos(a)) / 0.5),
             "CD": float((wf[1] * math.cos(a) + wf[2] * math.sin(a)) / 0.5)}
        s.close()
        if parts > 1:
            out[name] = r
            if log:
                log(name, r)
            continue
        # the colour-batched sweep, timed only
        s = Solver(m, cfg, device=dev, precision=prec)
        nb = s.lusgs_set_order(0)
        s.set_u(u0)
        s.steady_run(cfl=100.0, max_iter=5, threshold=0.0)
        torch.cuda.synchronize()
        e0.record()
        s.steady_run(cfl=100.0, max_iter=30, threshold=0.0)
        e1.record()
        torch.cuda.synchronize()
        r["colour_batches"] = {"batches_per_iteration": nb, "ms_per_iteration": e0.elapsed_time(e1) / 30}
        s.close()
        out[name] = r
        if log:
            log(name, r)
    out["dCL_fp32_vs_fp64"] = abs(out["fp32"]["CL"] - out["fp64"]["CL"])
    out["dCD_fp32_vs_fp64"] = abs(out["fp32"]["CD"] - out["fp64"]["CD"])
    # the oracle's sequential sweep on the host cores, a bounded sample of iterations
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        pyoracle.build()
        o = pyoracle.Oracle(m, cfg, n_threads=0)
        o.set_u(u0)
        o.implicit_iteration(100.0, u0)
        t0 = time.perf_counter()
        n = 5
        for _ in range(n):
            o.implicit_iteration(100.0, u0)
        dt = (time.perf_counter() - t0) / n
        out["cpu_oracle"] = {"ms_per_iteration": dt * 1e3, "cores": os.cpu_count(), "kind": "port",
                             "sample": "5 pseudo-time iterations, natural order"}
    except Exception as e:  # the CPU figure is a side report
        out["cpu_oracle"] = {"error": str(e)[:200]}
    return out


def wall_cp(m, u, far, gamma=1.4):
    """Surface pressure coefficient on the no-slip wall faces from the wall cells' means (first order):
    (x of the face centre, Cp = (p - p_inf) / (rho_inf |v_inf|^2 / 2))."""
    from dnds_b200 import mesh as M

    f = np.nonzero(m.face_bc == M.BC_WALL_NOSLIP)[0]
    c = m.face_cells[f, 0]
    x = 0.5 * (m.node_xy[m.face_nodes[f, 0], 0] + m.node_xy[m.face_nodes[f, 1], 0])

    def p(w):
        return (gamma - 1) * (w[..., 3] - 0.5 * (w[..., 1] ** 2 + w[..., 2] ** 2) / w[..., 0])

    q = 0.5 * (far[1] ** 2 + far[2] ** 2) / far[0]
    return x, (p(u[c]) - p(far)) / q


def steady_full(dev, log=None):
    """The steady RANS-SA run of steady_leg to the configured 1e-8 drop of the density increment ratio:
    the 512 x 128 C-mesh in FP64 (about 222,000 iterations), in FP64 with the sweep in STEADY_PARTS parts,
    and in FP32 bulk (whose rounding floor is near 1e-7: it stops at 150,000 iterations), and the coarse
    128 x 32 C-mesh in FP64.  Time to the residual, iterations, CL, CD and the suction peak of the
    surface Cp; FP32 bulk against FP64: |dCL|, |dCD| and the largest |dCp| over the wall faces."""
    from dnds_b200.partition import block_owner

    import math

    import torch

    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    cfg = S.preset("naca0012_sa")
    far = np.array(cfg["eulerSetting"]["farFieldStaticValue"])
    a = math.radians(10.0)
    out = {"workload": "RANS-SA NACA 0012 C-mesh, M 0.15, alpha 10, Re 6e6, BDF1 pseudo time, LU-SGS natural order, "
                       "CFL 100 ramped to 1000, fstop: density increment ratio < 1e-8"}
    cp = {}
    for key, kw, prec, maxit, parts in (("c512x128_fp64", {}, 0, 300000, 1),
                                        (f"c512x128_fp64_parts{STEADY_PARTS}", {}, 0, 300000, STEADY_PARTS),
                                        ("c512x128_fp32", {}, 1, 150000, 1),
                                        ("c128x32_fp64", dict(n_airfoil=64, n_wake=32, nj=32), 0, 200000, 1)):
        m = M.naca0012_cmesh(**kw)
        s = Solver(m, cfg, device=dev, precision=prec)
        s.lusgs_set_order(1)
        if parts > 1:
            s.lusgs_set_parts(block_owner(m.n_cells, parts), parts)
        s.set_u(np.tile(far, (m.n_cells, 1)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        it, rel, wf, hist = s.steady_run(threshold=1e-8, max_iter=maxit, history=True, **STEADY_RAMP)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        marks = {}
        for lvl in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8):
            hit = np.nonzero(hist <= lvl)[0]
            marks[f"{lvl:.0e}"] = int(hit[0] + 1) if len(hit) else None
        _, cp[key] = wall_cp(m, s.get_u(), far)
        out[key] = {"cells": m.n_cells, "iterations": it, "seconds": sec, "ms_per_iteration": sec * 1e3 / it,
                    "rel_residual_rho": float(rel[0]), "reached_1e-8": bool(rel[0] < 1e-8),
                    "iterations_to": marks,
                    "CL": float((-wf[1] * math.sin(a) + wf[2] * math.cos(a)) / 0.5),
                    "CD": float((wf[1] * math.cos(a) + wf[2] * math.sin(a)) / 0.5),
                    "Cp_min": float(cp[key].min())}
        s.close()
        if log:
            log(key, out[key])
    a64, a32 = out["c512x128_fp64"], out["c512x128_fp32"]
    out["fp32_vs_fp64"] = {"dCL": abs(a32["CL"] - a64["CL"]), "dCD": abs(a32["CD"] - a64["CD"]),
                           "dCp_max": float(np.abs(cp["c512x128_fp32"] - cp["c512x128_fp64"]).max()),
                           "wall_faces": int(cp["c512x128_fp64"].size)}
    return out


# algorithmic bytes per triangle cell of one ReconstructionWBAPLimitFacialV3 pass that limits every cell:
# coefficients read 20s and written 20s, means 32 B, the indicator's face basis rows (1.5 faces x 2 sides
# x 6 x 5 s) and the neighbour mapping matrices (1.5 faces x 2 sides x 25 s): 205s + 32 B
WBAP_BYTES_PER_CELL = {4: 205 * 4 + 32, 8: 205 * 8 + 32}


def riemann_leg(dev, steps=20, grid=2048, log=None):
    """The four-quadrant 2-D Riemann problem at its configured size (2048 x 2048 quads on [0,1]^2,
    interior nodes jittered by U(-0.15h, 0.15h), seed 4321, split into 8,388,608 triangles; P2 VR,
    CWBAP limiter, HLLC, SSP-RK3 at CFL 0.4 towards t = 0.3): cell-RK-stage updates/s in FP32 bulk and
    FP64, and the limiter alone (ReconstructionWBAPLimitFacialV3) with the smooth-indicator gate and
    with every cell limited, against its algorithmic bytes.  Timed outside the headline."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.riemann_mesh(grid)
    cfg = S.preset("riemann")
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    peak, peak_kind = measured_peak()
    out = {"workload": f"2-D Riemann, [0,1]^2, {grid}x{grid} jittered quads -> {m.n_cells:,} triangles, P2 VR + "
                       "CWBAP + HLLC, SSP-RK3 CFL 0.4", "cells": m.n_cells, "steps": steps}
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
    for prec, name in ((1, "fp32"), (0, "fp64")):
        s = Solver(m, cfg, device=dev, precision=prec)
        s.set_u(u0)
        for _ in range(3):
            s.ssprk3_step(0.4, 0.3)
        e0, e1 = ev()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            s.ssprk3_step(0.4, 0.3)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        r = {"ms_per_step": ms, "value": m.n_cells * 3 / (ms * 1e-3), "unit": UNIT, "t": s.time}
        nk = 10
        for if_all, key in ((False, "limiter_ms"), (True, "limiter_all_cells_ms")):
            e0, e1 = ev()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(nk):
                s.ReconstructionWBAPLimitFacialV3(if_all)
            e1.record()
            torch.cuda.synchronize()
            r[key] = e0.elapsed_time(e1) / nk
        sz = 4 if prec == 1 else 8
        ach = WBAP_BYTES_PER_CELL[sz] * m.n_cells / (r["limiter_all_cells_ms"] * 1e-3) / 1e9
        r["limiter_roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                 "peak_kind": f"{peak_kind} hbm_gbs", "alg_bytes_per_cell": WBAP_BYTES_PER_CELL[sz]}
        flags, nred = s.status()
        r["flags"] = flags
        r["reduced_order_points"] = nred
        out[name] = r
        s.close()
        if log:
            log(name, r)
    out["speedup_fp32_over_fp64"] = out["fp64"]["ms_per_step"] / out["fp32"]["ms_per_step"]
    return out


def riemann_to_end_leg(dev, grid=512, t_end=0.3, log=None):
    """The 2-D Riemann problem run to its configured end time t = 0.3 (SSP-RK3, CFL 0.4, P2 VR, CWBAP,
    HLLC) in FP32 bulk and in FP64 on a grid x grid jittered mesh (2 grid^2 triangles): steps, device
    time of the whole run, cell-RK-stage updates/s over it, and the density difference of the two
    precisions at t = 0.3 (L2 volume-weighted and Linf, absolute and relative to the density's own L2).
    The configured 2048 x 2048 mesh takes about 47,000 steps per precision (python bench.py
    --riemann-full); the default run uses a coarser grid so that the bench ends within minutes."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.riemann_mesh(grid)
    cfg = S.preset("riemann")
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    vol = G.cell_quadrature(m)[1].sum(1)
    out = {"workload": f"2-D Riemann, [0,1]^2, {grid}x{grid} jittered quads -> {m.n_cells:,} triangles, P2 VR + "
                       f"CWBAP + HLLC, SSP-RK3 CFL 0.4 to t = {t_end}", "cells": m.n_cells}
    us = {}
    for prec, name in ((1, "fp32"), (0, "fp64")):
        s = Solver(m, cfg, device=dev, precision=prec)
        s.set_u(u0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        steps = s.run_to(t_end, 0.4)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        us[name] = s.get_u()
        flags, nred = s.status()
        out[name] = {"steps": steps, "t": s.time, "seconds": sec, "ms_per_step": sec * 1e3 / steps,
                     "value": m.n_cells * 3 * steps / sec, "unit": UNIT, "flags": flags,
                     "reduced_order_points": nred}
        s.close()
        if log:
            log(name, out[name])
    d = us["fp32"][:, 0] - us["fp64"][:, 0]
    l2 = float(np.sqrt((d * d * vol).sum() / vol.sum()))
    rho_l2 = float(np.sqrt((us["fp64"][:, 0] ** 2 * vol).sum() / vol.sum()))
    out["rho_fp32_vs_fp64"] = {"l2": l2, "linf": float(np.abs(d).max()), "l2_relative": l2 / rho_l2,
                               "l1": float((np.abs(d) * vol).sum() / vol.sum())}
    out["speedup_fp32_over_fp64"] = out["fp64"]["seconds"] / out["fp32"]["seconds"]
    return out


def dual_time_leg(dev, grid=N_GRID, steps=20, dt=0.005, log=None):
    """The reference's implicit unsteady driver on the headline vortex (2,097,152 triangles): SDIRK4 and
    BDF2 dual time (ImplicitSDIRK4DualTimeStep / ImplicitBDFDualTimeStep, DNDS_ODE.hpp:269-497) with
    LU-SGS in colour batches, pseudo-time CFL 100, at most 20 internal iterations per stage to a density
    increment ratio of 1e-4, physical dt 0.005 (about 1.2 times the explicit step at CFL 0.5: on this fine
    mesh larger steps leave the stages unconverged after 30 iterations, and SDIRK4 then diverges),
    `steps` steps to t = 0.1; and SDIRK4 with GMRES(LU-SGS) (5 Krylov vectors, one restart).  ms per
    physical step, internal iterations per stage, and the density L2 error against the exact advected
    vortex at the end, FP64 and FP32 bulk.  The oracle's SDIRK4 step on the 128 x 128 x 2 version on the
    host cores gives the CPU figure."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(grid, True, jitter=0.2, seed=1234)
    u0 = G.isentropic_vortex(m)
    vol = G.cell_quadrature(m)[1].sum(1)
    exact = G.isentropic_vortex(m, t=steps * dt)[:, 0]
    out = {"workload": f"isentropic vortex, {grid}x{grid}x2 = {m.n_cells:,} triangles, physical dt {dt}, "
                       f"{steps} steps to t = {steps * dt:.3g}, pseudo-time CFL 100, LU-SGS colour batches, "
                       "internal iterations <= 20 to 1e-4"}
    variants = (("sdirk4", dict(scheme="sdirk4"), 1), ("sdirk4", dict(scheme="sdirk4"), 0),
                ("bdf2", dict(scheme="bdf", bdf_order=2), 1),
                ("sdirk4_gmres", dict(scheme="sdirk4", gmres_code=1, n_gmres_space=5, n_gmres_iter=1), 1))
    for name, kw, prec in variants:
        s = Solver(m, S.preset("vortex"), device=dev, precision=prec)
        s.set_u(u0)
        its = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for k in range(steps):
            it, _ = s.dual_step(dt, k * dt, cfl=100.0, max_iter=20, threshold=1e-4, **kw)
            its.append([int(x) for x in it])
        e1.record()
        torch.cuda.synchronize()
        d = s.get_u()[:, 0] - exact
        key = f"{name}_{'fp32' if prec else 'fp64'}"
        out[key] = {"ms_per_step": e0.elapsed_time(e1) / steps, "iterations_per_stage": its,
                    "l2_rho_vs_exact": float(np.sqrt((d * d * vol).sum() / vol.sum()))}
        s.close()
        if log:
            log(key, out[key])
    try:  # the oracle's SDIRK4 step on a bounded sample of the workload, host cores
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        pyoracle.build()
        mc = M.vortex_mesh(128, True, jitter=0.2, seed=1234)
        o = pyoracle.Oracle(mc, S.preset("vortex"), n_threads=0)
        o.set_u(G.isentropic_vortex(mc))
        t0 = time.perf_counter()
        o.dual_step(dt, 0.0, scheme="sdirk4", cfl=100.0, max_iter=20, threshold=1e-4)
        sec = time.perf_counter() - t0
        out["cpu_oracle"] = {"ms_per_step": sec * 1e3, "cells": mc.n_cells, "cores": os.cpu_count(), "kind": "port",
                             "cell_steps_per_s": mc.n_cells / sec, "sample": "one SDIRK4 step, 128x128x2 triangles"}
    except Exception as e:  # the CPU figure is a side report
        out["cpu_oracle"] = {"error": str(e)[:200]}
    return out


def partition_leg(dev, grid=512, steps=20, log=None):
    """Partitioned runs on one GPU (dnds_b200.partition.PartitionedRun: one context per part with its
    ghost layer, halo pack / unpack after every VR sweep and stage update, dt reduced over the parts on
    the host) against the whole mesh, FP32 bulk, the vortex on grid x grid x 2 triangles: ms per
    SSP-RK3 step (wall time over `steps` steps; the partitioned step synchronises once for dt) and the
    largest difference of the owned means from the whole-mesh run.  On several GPUs the pack / unpack
    pairs become NCCL send / receive; that run is not available on one GPU."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.partition import PartitionedRun
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(grid, True, jitter=0.2, seed=1234)
    u0 = G.isentropic_vortex(m)
    cfg = S.preset("vortex")
    out = {"workload": f"isentropic vortex, {grid}x{grid}x2 = {m.n_cells:,} triangles, FP32 bulk, SSP-RK3 CFL 0.5"}
    s = Solver(m, cfg, device=dev, precision=1)
    s.set_u(u0)
    s.ssprk3_step(0.5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        s.ssprk3_step(0.5)
    torch.cuda.synchronize()
    out["whole_mesh_ms_per_step"] = (time.perf_counter() - t0) / steps * 1e3
    ref = s.get_u()
    s.close()
    for nparts in (2, 4):
        t0 = time.perf_counter()
        pr = PartitionedRun(m, cfg, nparts, precision=1, device=dev)
        t_setup = time.perf_counter() - t0
        pr.set_u(u0)
        pr.ssprk3_step(0.5)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            pr.ssprk3_step(0.5)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) / steps * 1e3
        diff = float(np.abs(pr.get_u() - ref).max() / np.abs(ref).max())
        pr.close()
        out[f"parts{nparts}"] = {"ms_per_step": ms, "max_rel_diff_vs_whole": diff, "setup_s": t_setup}
        if log:
            log(f"parts{nparts}", out[f"parts{nparts}"])
    return out


def renumber_leg(dev, grid=N_GRID, steps=20, log=None):
    """The METIS-free renumbering on the headline workload (FP32 bulk): the VR sweep, the RHS and the
    SSP-RK3 step on the generator's cell order, on a random permutation of it (a mesh file whose
    element order carries no locality), and on that permutation renumbered along a Hilbert curve
    (mesh.renumber).  CUDA-event times; the results of all three are the same, permuted."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m0 = M.vortex_mesh(grid, True, jitter=0.2, seed=1234)
    u0 = G.isentropic_vortex(m0)
    shuffled, sh = M.renumber(m0, np.random.default_rng(7).permutation(m0.n_cells))
    t0 = time.perf_counter()
    hil, order = M.renumber(shuffled)
    t_renumber = time.perf_counter() - t0
    out = {"workload": f"isentropic vortex, {grid}x{grid}x2 = {m0.n_cells:,} triangles, FP32 bulk",
           "renumber_host_s": t_renumber}
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
    for key, m, u in (("generator_order", m0, u0), ("random_order", shuffled, u0[sh]),
                      ("random_then_hilbert", hil, u0[sh][order])):
        L, R = m.face_cells[:, 0], m.face_cells[:, 1]
        inner = R >= 0
        s = Solver(m, S.preset("vortex"), device=dev, precision=1)
        s.set_u(u)
        for _ in range(3):
            s.ssprk3_step(0.5)
        r = {"mean_face_index_gap": float(np.abs(L[inner] - R[inner]).mean())}
        for name, fn in (("vr_ms", lambda: s.ReconstructionJacobiStep(1)), ("rhs_ms", lambda: s.EvaluateRHS(0.0, copy=False)),
                         ("step_ms", lambda: s.ssprk3_step(0.5))):
            e0, e1 = ev()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            r[name] = e0.elapsed_time(e1) / steps
        s.close()
        out[key] = r
        if log:
            log(key, r)
    return out


def small_mesh_leg(dev, steps=2000):
    """The launch-bound small case: the isentropic vortex on 40 x 40 periodic quads (1,600 cells), P2 VR +
    Roe, SSP-RK3 CFL 0.5: ms per step with one kernel launch per kernel (dndsg_ssprk3_step) and with
    pairs of steps replayed from a CUDA graph (dndsg_ssprk3_steps).  Timed outside the headline."""
    import torch

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(40, False)
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    out = {"workload": "isentropic vortex, periodic [0,10]^2, 40x40 quads (1,600 cells), P2 VR + Roe, SSP-RK3 CFL 0.5",
           "cells": m.n_cells, "steps": steps}
    for prec, name in ((1, "fp32"), (0, "fp64")):
        s = Solver(m, cfg, device=dev, precision=prec)
        s.set_u(u0)
        s.ssprk3_steps(0.5, 10)
        r = {}
        for mode in ("launches", "graph"):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if mode == "graph":
                s.ssprk3_steps(0.5, steps)
            else:
                for _ in range(steps):
                    s.ssprk3_step(0.5)
            e1.record()
            torch.cuda.synchronize()
            r[f"ms_per_step_{mode}"] = e0.elapsed_time(e1) / steps
        r["value_graph"] = m.n_cells * 3 / (r["ms_per_step_graph"] * 1e-3)
        out[name] = r
        s.close()
    return out


def learned_leg(dev, grid, tol=1e-7, log=None):
    """The learned VR warm start (BF16 MLP on tcgen05), both input designs: each is harvested from
    tolerance-mode runs of the three explicit workloads (the vortex on 40 x 40 quads and on two
    256 x 256 x 2 jittered triangle meshes, the Riemann problem with the limiter on 256 x 256 x 2), trained
    on the GPU (pairs whose targets exceed +-10 left out: learned.bounded_pairs), and evaluated as
    Jacobi sweeps per SSP-RK3 step to the same rms-increment tolerance,
    with and without the network, on fresh-seed (9999) 1448 x 1448 x 2 = 4,193,408-triangle vortex and
    Riemann meshes.  Design 0 extrapolates two plain sweeps; design 1 is the configured input (neighbour
    mean differences and the previous-step coefficients).  Plus the tensor-core forward's throughput.
    Timed outside the headline."""
    import torch

    from dnds_b200.learned import WarmStartNet, bounded_pairs, evaluate, train, training_set

    out = {"tolerance_rms_increment": tol, "evaluation_grid": 1448}
    nets = {}
    for design in (0, 1):
        t0 = time.perf_counter()
        X, T = training_set(tol, steps=8, n=256, features=design)
        n_harvested = int(X.shape[0])
        X, T, kept = bounded_pairs(X, T)
        torch.cuda.synchronize()
        t_harvest = time.perf_counter() - t0
        net = WarmStartNet(dev, seed=7, features=design)
        t0 = time.perf_counter()
        _, val = train(net, X, T, epochs=20)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        out[f"design{design}_training"] = {"pairs_harvested": n_harvested, "pairs": int(X.shape[0]),
                                           "kept_fraction": kept, "harvest_s": t_harvest, "train_s": t_train,
                                           "train_samples_per_s": 20 * X.shape[0] / t_train, "val_loss": val,
                                           "target_mean_square": float((T ** 2).mean())}
        del X, T
        nets[f"design{design}"] = net
    out["evaluation"] = evaluate(nets, tol, grid=1448, steps=3, seed=9999, log=log)
    # inference throughput of the tensor-core forward: 4,194,304 rows of 64 features
    rows = 4_194_304
    net = nets["design0"]
    Xf = torch.randn((rows, 64), device=dev, dtype=torch.float32)
    Yf = net.forward(Xf)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        Yf = net.forward(Xf)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    flop = 2 * (64 * 64 * 3 + 64 * 20) * rows
    out["forward_tc"] = {"rows": rows, "ms": ms, "rows_per_s": rows / (ms * 1e-3),
                         "tflops": flop / (ms * 1e-3) / 1e12, "gbs": rows * (64 * 4 + 20 * 4) / (ms * 1e-3) / 1e9,
                         "note": "tcgen05.mma kind::f16, BF16 operands, FP32 accumulator in tensor memory; "
                                 "bytes are the FP32 features read and outputs written"}
    del Xf, Yf
    for n in nets.values():
        n.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="dnds_b200", choices=["dnds_b200", "reference"])
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy-t", type=float, default=2.0, help="end time of the accuracy runs (the config's t=2)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid", type=int, default=N_GRID, help="grid size n (n x n quads -> 2 n^2 triangles)")
    ap.add_argument("--precisions", default="fp32,fp64")
    ap.add_argument("--no-steady", action="store_true", help="skip the implicit steady RANS-SA NACA 0012 report")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start report")
    ap.add_argument("--no-renumber", action="store_true", help="skip the cell-renumbering (locality) report")
    ap.add_argument("--no-dual", action="store_true", help="skip the implicit unsteady (dual time) report")
    ap.add_argument("--no-riemann", action="store_true", help="skip the 8.4M-triangle Riemann / CWBAP report")
    ap.add_argument("--riemann-grid", type=int, default=2048, help="grid size of the Riemann / CWBAP report")
    ap.add_argument("--riemann-end-grid", type=int, default=512,
                    help="grid size of the Riemann run to t = 0.3 in the default bench")
    ap.add_argument("--steady-full", action="store_true",
                    help="only the steady RANS-SA NACA 0012 runs to the 1e-8 drop (about 10 minutes); one JSON line")
    ap.add_argument("--riemann-full", action="store_true",
                    help="only the Riemann problem to t = 0.3 on the configured 2048 x 2048 mesh (both precisions, "
                         "about 17 minutes); prints one JSON line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch

    if args.steady_full:
        torch.cuda.set_device(0)
        clk = ClockSampler(0)
        r = steady_full(0, log=lambda *a: print(*a, file=sys.stderr, flush=True))
        r["clocks"] = clk.stop()
        r["command"] = "python bench.py --steady-full"
        print(json.dumps(r))
        return
    if args.riemann_full:
        torch.cuda.set_device(0)
        clk = ClockSampler(0)
        r = riemann_to_end_leg(0, grid=2048, log=lambda *a: print(*a, file=sys.stderr, flush=True))
        r["clocks"] = clk.stop()
        r["command"] = "python bench.py --riemann-full"
        print(json.dumps(r))
        return

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(args.grid, True, jitter=0.2, seed=1234)
    N = m.n_cells
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def time_steps(solver, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        for _ in range(k):
            solver.ssprk3_step(0.5, 1e300)
        e1.record()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1), device="cuda")

    results = {}
    wanted = args.precisions.split(",")
    for prec, name in ((1, "fp32"), (0, "fp64")):
        if name not in wanted:
            continue
        s = Solver(m, cfg, device=dev, precision=prec)
        s.set_u(u0)
        clk = ClockSampler(dev) if name == "fp32" else None
        for _ in range(args.warmup):
            s.ssprk3_step(0.5, 1e300)
        ms = time_steps(s, args.steps)
        # per-kernel: the VR sweep alone, and the RHS (face flux + gather)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nk = 20
        barrier()
        e0.record()
        for _ in range(nk):
            s.ReconstructionJacobiStep(1)
        e1.record()
        torch.cuda.synchronize()
        vr_ms = e0.elapsed_time(e1) / nk
        s.EvaluateDt(0.5)
        e0.record()
        for _ in range(nk):
            s.EvaluateRHS(0.0, copy=False)
        e1.record()
        torch.cuda.synchronize()
        rhs_ms = e0.elapsed_time(e1) / nk
        flags, nred = s.status()
        results[name] = dict(ms=ms, vr_ms=vr_ms, rhs_ms=rhs_ms, clocks=None, flags=flags, nred=nred)
        # end-to-end through the public API with host buffers: per step h2d of the
        # state u (pinned), one SSP-RK3 step, d2h of the new state
        if name == "fp32" and not args.no_e2e:
            host = torch.empty((N, 4), dtype=torch.float64, pin_memory=True)
            host.copy_(torch.from_numpy(u0))
            hnp = host.numpy()
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                s.set_u(hnp)
                s.ssprk3_step(0.5, 1e300)
                s.get_u(out=hnp)
            barrier()
            results[name]["e2e_s"] = max_over_ranks(time.perf_counter() - t0, device="cuda")
        # accuracy at t = 2 against the exact advected vortex (density)
        if not args.no_accuracy:
            s.set_u(u0)
            s.set_urec(np.zeros((N, 5, 4)))
            s.time = 0.0
            steps = s.run_to(args.accuracy_t, 0.5)
            u = s.get_u()
            ex = G.isentropic_vortex(m, t=args.accuracy_t)
            vol = G.cell_quadrature(m)[1].sum(1)
            d = u[:, 0] - ex[:, 0]
            results[name]["l2_rho"] = float(np.sqrt((d * d * vol).sum() / vol.sum()))
            results[name]["linf_rho"] = float(np.abs(d).max())
            results[name]["steps_to_t2"] = steps
            results[name]["u_t2"] = u
        if clk:
            results[name]["clocks"] = clk.stop()
        s.close()

    if len(results) == 2 and "u_t2" in results["fp32"]:
        d = results["fp32"]["u_t2"][:, 0] - results["fp64"]["u_t2"][:, 0]
        vol = G.cell_quadrature(m)[1].sum(1)
        l2_vs64 = float(np.sqrt((d * d * vol).sum() / vol.sum()))
    else:
        l2_vs64 = None
    for r in results.values():
        r.pop("u_t2", None)

    r32 = results.get("fp32") or results["fp64"]
    r64 = results.get("fp64") or r32
    value = replica_throughput(N, args.steps, r32["ms"], ws)
    value64 = replica_throughput(N, args.steps, r64["ms"], ws)
    peak, peak_kind = measured_peak()
    vr_bytes = VR_BYTES_PER_CELL[4] * N
    achieved = vr_bytes / (r32["vr_ms"] * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r32["ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 bulk (f64 means, dt, norms)", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.grid == N_GRID else f"{WORKLOAD} (grid {args.grid})", "cells": N, "faces": m.n_faces, "precision": "fp32-bulk",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                   "l2_flush": "no flush: per-step working set ~1.3 GB > 126 MB L2"},
        "value_fp64": value64,
        "fp64_path": {"value": value64, "ms_per_step": r64["ms"] / args.steps, "vr_ms": r64["vr_ms"],
                      "rhs_ms": r64["rhs_ms"]},
        "speedup_fp32_over_fp64": value / value64,
        "step_roofline": {
            name: {"alg_bytes_per_cell": STEP_BYTES_PER_CELL[sz],
                   "achieved": STEP_BYTES_PER_CELL[sz] * N / (r["ms"] / args.steps * 1e-3) / 1e9,
                   "frac": STEP_BYTES_PER_CELL[sz] * N / (r["ms"] / args.steps * 1e-3) / 1e9 / peak,
                   "unit": "GB/s"}
            for name, r, sz in (("fp32", r32, 4), ("fp64", r64, 8))},
        "speedup_bound_by_bytes": STEP_BYTES_PER_CELL[8] / STEP_BYTES_PER_CELL[4],
        "kernels_ms": {"vr_sweep_fp32": r32["vr_ms"], "rhs_fp32": r32["rhs_ms"]},
        "roofline": {"kernel": "vr_sweep (FP32)", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                     "traffic": VR_TRAFFIC_FP32,
                     "alg_bytes_per_launch": vr_bytes},
        "gpu_launches": KERNELS_PER_STEP * args.steps,
        "clocks": r32["clocks"],
        "status": {"flags": r32["flags"] | r64["flags"], "reduced_order_points": r32["nred"] + r64["nred"]},
    }
    if "e2e_s" in r32:
        out["e2e"] = {"value": replica_throughput(N, args.steps, r32["e2e_s"] * 1e3, ws), "unit": UNIT,
                      "h2d_bytes_per_step": N * 4 * 8, "d2h_bytes_per_step": N * 4 * 8}
    if "l2_rho" in r32:
        out["accuracy"] = {"t_end": args.accuracy_t, "l2_rho_fp32": r32["l2_rho"], "l2_rho_fp64": r64["l2_rho"],
                           "linf_rho_fp32": r32["linf_rho"], "linf_rho_fp64": r64["linf_rho"],
                           "l2_rho_fp32_vs_fp64": l2_vs64, "steps": r32["steps_to_t2"],
                           "l2_ratio_fp32_over_fp64": r32["l2_rho"] / r64["l2_rho"],
                           "equal_l2_within_1pct": abs(r32["l2_rho"] / r64["l2_rho"] - 1.0) <= 0.01,
                           "reference": "exact advected vortex (cell averages), density"}
    if rank == 0 and ws == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline()
    if rank == 0 and ws == 1 and not args.no_steady:
        out["steady_naca0012_sa"] = steady_leg(dev)
        rec = os.path.join(ROOT, "profiles", "steady_naca0012_sa_full.json")
        if os.path.exists(rec):  # the runs to the 1e-8 drop, recorded by --steady-full (too long for here)
            with open(rec) as fh:
                out["steady_naca0012_sa_full_recorded"] = json.load(fh)
    if rank == 0 and ws == 1 and not args.no_riemann:
        out["small_mesh_c1"] = small_mesh_leg(dev)
    if rank == 0 and ws == 1 and not args.no_riemann:
        out["riemann_cwbap"] = riemann_leg(dev, grid=args.riemann_grid)
        out["riemann_to_t03"] = riemann_to_end_leg(dev, grid=args.riemann_end_grid)
        rec = os.path.join(ROOT, "profiles", "riemann_full_tri2048_t0.3.json")
        if os.path.exists(rec):  # the configured mesh to t = 0.3, recorded by --riemann-full (too long for here)
            with open(rec) as fh:
                out["riemann_to_t03_2048_recorded"] = json.load(fh)
    def side(fn, *a):  # a side report that fails leaves an error in its place, not a missing line
        try:
            return fn(*a)
        except Exception as e:
            return {"error": f"{type(e).__name__}: {str(e)[:300]}"}

    if rank == 0 and ws == 1 and not args.no_dual:
        out["dual_time_vortex"] = side(dual_time_leg, dev, args.grid)
    if rank == 0 and ws == 1 and not args.no_renumber:
        out["renumber_locality"] = side(renumber_leg, dev, args.grid)
        out["partitioned_one_gpu"] = side(partition_leg, dev)
    if rank == 0 and ws == 1 and not args.no_learned:
        out["learned_vr"] = learned_leg(dev, args.grid)
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
