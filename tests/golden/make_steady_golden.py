"""Converged steady RANS-SA states of the oracle on coarse NACA 0012 C-meshes (tests/golden/sa_steady_*.npz).

The oracle's restatement of the reference's steady implicit run (RunImplicitEuler with ifSteadyQuit,
DNDS_FV_EulerSolver.hpp:852-1061): first-order BDF pseudo time, LU-SGS in the natural scan order,
CFL 100 ramped log-linearly to 1000 over iterations 100-1100 (the fstop ramp, :1047-1052), until the
L1 norm of the density increment falls below 1e-8 of its largest value so far.  Stored: the mesh
arguments, the converged state [N][5], the iteration count, the first iteration whose ratio falls
below 1e-3, ..., 1e-8, and the wall force of the final state's residual.  Runs on the host cores
(about 4 minutes for c64x16 and half an hour for c128x32 on 8 threads).

usage: python tests/golden/make_steady_golden.py c64x16 [c128x32] [--threads N]
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = {"c64x16": dict(n_airfoil=32, n_wake=16, nj=16), "c128x32": dict(n_airfoil=64, n_wake=32, nj=32)}
RAMP = dict(cfl=100.0, cfl_ramp_start=100, cfl_ramp_length=1000, cfl_ramp_end=1000.0)
THRESHOLD = 1e-8


def ramp_cfl(it: int) -> float:
    """The CFL after iteration it (fstop: log-linear from cfl to cfl_ramp_end over the ramp)."""
    s, n = RAMP["cfl_ramp_start"], RAMP["cfl_ramp_length"]
    if s <= it <= s + n:
        return math.exp(math.log(RAMP["cfl"]) + math.log(RAMP["cfl_ramp_end"] / RAMP["cfl"]) * (it - s) / n)
    return None


def converge(name: str, threads: int, max_iter: int = 400000):
    import pyoracle

    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S

    pyoracle.build()
    m = M.naca0012_cmesh(**CASES[name])
    cfg = S.preset("naca0012_sa")
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    o = pyoracle.Oracle(m, cfg, n_threads=threads)
    o.set_u(u0)
    cfl, base, hist = RAMP["cfl"], None, []
    t0 = time.time()
    for it in range(1, max_iter + 1):
        inc = o.implicit_iteration(cfl, u0)
        r = np.abs(inc[:, 0]).sum()
        base = r if base is None else max(base, r)
        hist.append(r / base)
        if hist[-1] < THRESHOLD:
            break
        c = ramp_cfl(it)
        cfl = c if c is not None else cfl
    _, wall = o.eval_rhs(0.0)
    print(f"{name}: {it} iterations, ratio {hist[-1]:.3e}, {time.time() - t0:.0f} s", flush=True)
    h = np.array(hist)
    marks = np.array([int(np.argmax(h <= 10.0 ** -k)) + 1 for k in range(3, 9)])
    np.savez_compressed(os.path.join(HERE, f"sa_steady_{name}.npz"), u=o.get_u(), iterations=it, marks=marks,
                        wall=wall, **{k: v for k, v in CASES[name].items()})


if __name__ == "__main__":
    args = sys.argv[1:]
    threads = 8
    if "--threads" in args:
        k = args.index("--threads")
        threads = int(args[k + 1])
        del args[k:k + 2]
    for name in args or ["c64x16"]:
        converge(name, threads)
