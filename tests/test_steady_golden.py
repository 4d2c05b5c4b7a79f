"""Steady RANS-SA solves to the configured 1e-8 drop against the oracle's converged runs.

The fixtures (tests/golden/make_steady_golden.py) hold the oracle's steady run on coarse NACA 0012
C-meshes: first-order BDF pseudo time, LU-SGS in the natural scan order, CFL 100 ramped to 1000 over
iterations 100-1100, stopped when the L1 norm of the density increment falls below 1e-8 of its largest
value so far (RunImplicitEuler with ifSteadyQuit, DNDS_FV_EulerSolver.hpp:852-1061).  The GPU runs the
same solver through one C call (dndsg_steady_solve).  FP64: the same number of iterations to within
0.5% (the runs differ in summation order only, and the ratio crosses each decade at the same iteration
to within a few), the converged state within 1e-6 relative and the lift and drag coefficients within
1e-6.  FP32 bulk stops at its rounding floor; its CL and CD must agree with the oracle's within the
configured 1e-4.
"""
import math
import os

import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RAMP = dict(cfl=100.0, cfl_ramp_start=100, cfl_ramp_length=1000, cfl_ramp_end=1000.0)
ALPHA = math.radians(10.0)

pytestmark = pytest.mark.gpu


def _fixture(name):
    path = os.path.join(GOLDEN, f"sa_steady_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated")
    return np.load(path)


def _coefficients(wf):
    """CL, CD from the wall force (the free stream has unit density and speed: q = 1/2, chord 1)."""
    cl = (-wf[1] * math.sin(ALPHA) + wf[2] * math.cos(ALPHA)) / 0.5
    cd = (wf[1] * math.cos(ALPHA) + wf[2] * math.sin(ALPHA)) / 0.5
    return cl, cd


def _solve(g, precision, max_iter):
    from dnds_b200.solver import Solver

    m = M.naca0012_cmesh(n_airfoil=int(g["n_airfoil"]), n_wake=int(g["n_wake"]), nj=int(g["nj"]))
    cfg = S.preset("naca0012_sa")
    s = Solver(m, cfg, precision=precision)
    s.lusgs_set_order(1)
    s.set_u(np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1)))
    it, rel, wf, hist = s.steady_run(threshold=1e-8, max_iter=max_iter, history=True, **RAMP)
    u = s.get_u()
    flags, _ = s.status()
    s.close()
    return it, rel, wf, hist, u, flags


@pytest.mark.parametrize("name", ["c64x16", "c128x32"])
def test_fp64_steady_solve_matches_the_converged_oracle(name):
    g = _fixture(name)
    n_ref = int(g["iterations"])
    it, rel, wf, hist, u, flags = _solve(g, 0, int(1.2 * n_ref))
    marks = [int(np.argmax(hist <= 10.0 ** -k)) + 1 for k in range(3, 9)]
    print(f"\n{name}: GPU {it} iterations (oracle {n_ref}); decades at {marks} (oracle {list(g['marks'])})")
    assert flags == 0
    assert rel[0] < 1e-8
    assert abs(it - n_ref) <= 0.005 * n_ref
    assert np.abs(u - g["u"]).max() < 1e-6 * np.abs(g["u"]).max()
    cl, cd = _coefficients(wf)
    cl_o, cd_o = _coefficients(g["wall"])
    assert abs(cl - cl_o) < 1e-6 and abs(cd - cd_o) < 1e-6


def test_fp32_bulk_steady_forces_within_the_configured_bound():
    g = _fixture("c64x16")
    n_ref = int(g["iterations"])
    it, rel, wf, _, u, flags = _solve(g, 1, n_ref)
    assert flags == 0
    assert rel[0] < 1e-6
    cl, cd = _coefficients(wf)
    cl_o, cd_o = _coefficients(g["wall"])
    print(f"\nFP32 bulk: {it} iterations, ratio {rel[0]:.2e}, |dCL| {abs(cl - cl_o):.2e}, |dCD| {abs(cd - cd_o):.2e}")
    assert abs(cl - cl_o) < 1e-4 and abs(cd - cd_o) < 1e-4
