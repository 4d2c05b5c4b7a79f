"""Explicit SSP-RK3 runs of the vortex and 2-D Riemann workloads (the role of the reference's explicit
solver loop, DNDS_FV_EulerSolver.hpp:713-837 with ExplicitSSPRK3LocalDt::Step, DNDS_ODE.hpp:131-177).

    python -m dnds_b200.explicit --case riemann --grid 2048 --steps 5 --precision 1

Cases: `vortex` (periodic [0,10]^2, isentropic vortex, Roe, no limiter, CFL 0.5) and `riemann`
([0,1]^2, four quadrant states, HLLC, CWBAP limiter, CFL 0.4), both on grid x grid jittered quads
split into triangles.  Runs --warmup untimed steps, then --steps steps timed with CUDA events, and
prints ms per step and cell-stage updates per second; --limiter-all N then times N calls of the limiter
with every cell limited (ReconstructionWBAPLimitFacialV3 with ifAll).
"""
from __future__ import annotations

import argparse

from . import geometry as G
from . import mesh as M
from . import settings as S
from .solver import Solver


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--case", choices=["vortex", "riemann"], default="riemann")
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", type=int, default=1, help="0 FP64, 1 FP32 bulk")
    ap.add_argument("--limiter-all", type=int, default=0, help="then time this many every-cell limiter calls")
    a = ap.parse_args(argv)
    import torch

    if a.case == "vortex":
        m, cfl, t_end = M.vortex_mesh(a.grid, True, jitter=0.2, seed=1234), 0.5, 1e300
        u0 = G.isentropic_vortex(m)
    else:
        m, cfl, t_end = M.riemann_mesh(a.grid), 0.4, 0.3
        u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    s = Solver(m, S.preset(a.case), precision=a.precision)
    s.set_u(u0)
    for _ in range(a.warmup):
        s.ssprk3_step(cfl, t_end)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        s.ssprk3_step(cfl, t_end)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(a.steps, 1)
    print(f"{m.name}: {m.n_cells} cells, precision {a.precision}: {ms:.3f} ms per step, "
          f"{3 * m.n_cells / (ms * 1e-3):.3e} cell-stage updates/s, t = {s.time:.4e}")
    if a.limiter_all > 0:
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.limiter_all):
            s.ReconstructionWBAPLimitFacialV3(True)
        e1.record()
        torch.cuda.synchronize()
        print(f"limiter, every cell: {e0.elapsed_time(e1) / a.limiter_all:.3f} ms per call")
    flags, _ = s.status()
    s.close()
    return 0 if flags == 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
