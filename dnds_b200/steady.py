"""Steady NACA 0012 runs on the implicit path (the role of the reference's EulerSolver run with
`ifSteadyQuit`, DNDS_FV_EulerSolver.hpp:609-615 and :984-1061): first-order BDF pseudo time with
colour-batched or scan-order LU-SGS (optionally partitioned, --parts), stopping on the relative
density increment (fstop).

    python -m dnds_b200.steady --case sa --iters 2000 --cfl 100

Cases: `euler` (inviscid, M 0.15, alpha 10), `laminar` (M 0.5, Re 5000, alpha 0), `sa` (RANS-SA,
M 0.15, alpha 10, Re 6e6).  Prints the increment history every --every iterations and CL / CD from
the wall force (per unit chord, free-stream dynamic pressure 0.5); --plt writes the final state in
the reference's Tecplot binary layout.
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np

from . import mesh as M
from . import settings as S
from .solver import Solver

CASES = {
    # name: (preset, wall BC, mesh keyword arguments, alpha in degrees)
    "euler": ("naca0012", M.BC_WALL_EULER, {}, 10.0),
    "laminar": ("naca0012_laminar", M.BC_WALL_NOSLIP, dict(n_airfoil=128, n_wake=64, nj=64, first=1e-4, far=20.0), 0.0),
    "sa": ("naca0012_sa", M.BC_WALL_NOSLIP, {}, 10.0),
}


def force_coefficients(wall_flux, alpha_deg: float, q: float = 0.5):
    a = math.radians(alpha_deg)
    fx, fy = wall_flux[1], wall_flux[2]
    return (-fx * math.sin(a) + fy * math.cos(a)) / q, (fx * math.cos(a) + fy * math.sin(a)) / q


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--case", choices=sorted(CASES), default="sa")
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--cfl", type=float, default=100.0)
    ap.add_argument("--threshold", type=float, default=1e-8, help="relative density increment to stop at")
    ap.add_argument("--order", choices=["natural", "colour", "lines"], default="natural")
    ap.add_argument("--parts", type=int, default=1,
                    help="sweep the scan order in this many parts, as the reference on that many ranks")
    ap.add_argument("--precision", type=int, default=0, help="0 FP64, 1 FP32 bulk")
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--plt", default=None, help="write the final state as a Tecplot binary file (PrintData)")
    a = ap.parse_args(argv)
    preset, wall, mkw, alpha = CASES[a.case]
    m = M.naca0012_cmesh(wall_bc=wall, **mkw)
    cfg = S.preset(preset)
    s = Solver(m, cfg, precision=a.precision)
    nb = s.lusgs_set_order(0) if a.order == "colour" else s.lusgs_set_order(
        1, M.line_scan_order(m) if a.order == "lines" else None)
    if a.parts > 1 and a.order != "colour":
        from .partition import block_owner

        nb = s.lusgs_set_parts(block_owner(m.n_cells, a.parts), a.parts)
    s.set_u(np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1)))
    s.bdf_begin()
    print(f"{m.name}: {m.n_cells} cells, case {a.case}, {nb} LU-SGS batches per iteration")
    base = None
    t0 = time.perf_counter()
    it, wf, rel = 0, np.zeros(s.nv), 1.0
    for it in range(1, a.iters + 1):
        res, wf = s.implicit_iteration(a.cfl)
        base = res[0] if base is None else max(base, res[0])
        rel = res[0] / base
        if it % a.every == 0 or rel < a.threshold:
            cl, cd = force_coefficients(wf, alpha)
            print(f"iter {it:6d}  rel {rel:.3e}  CL {cl:.5f}  CD {cd:.5f}  {time.perf_counter() - t0:.1f} s", flush=True)
        if rel < a.threshold:
            break
    cl, cd = force_coefficients(wf, alpha)
    flags, nred = s.status()
    if a.plt:
        from .tecplot import print_data

        print_data(a.plt, m, s.get_u(), cfg, rhs=s.EvaluateRHS(0.0))
        print(f"wrote {a.plt}")
    print(f"done: {it} iterations, rel {rel:.3e}, CL {cl:.5f}, CD {cd:.5f}, flags {flags}")
    return 0 if flags == 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
