"""GPU against the oracle at the configured sizes (the oracle runs on the host cores; about 14 GB and a
minute at 2,097,152 cells).

C2: the 1024 x 1024 x 2 = 2,097,152-triangle jittered vortex, one FP64 SSP-RK3 step from the
cell-averaged vortex (each stage a VR sweep, EvaluateDt, EvaluateRHS and the update), within 1e-12.
C3: the Riemann problem on 1024 x 1024 x 2 triangles (a quarter of the configured 2048 x 2048, whose
oracle would need about 56 GB), from the quadrant states times a smooth perturbation: two VR sweeps,
the CWBAP indicator and the exact set of cells it lists, the limited face states, dt and the RHS, FP64,
within 1e-11.  C4: the 512 x 128 RANS-SA C-mesh at the configured spacing, three pseudo-time
iterations in the natural order and with the sweep in 16 parts, within 1e-9 (the single-iteration
tolerance of tests/test_sa.py).
"""
import importlib.util
import os

import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_c2_vortex_full_size_step_matches_oracle(oracle_lib):
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(1024, True, jitter=0.2, seed=1234)
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    o = oracle_lib.Oracle(m, cfg, n_threads=0)
    o.set_u(u0)
    _, d = o.eval_dt(0.5)
    o.ssprk3_step(d, 0.0)
    ref = o.get_u()
    del o
    s = Solver(m, cfg, precision=0)
    s.set_u(u0)
    s.ssprk3_step(0.5)
    assert abs(s.time - d) < 1e-13 * d
    assert _rel(s.get_u() - u0, ref - u0) < 1e-10  # the one-step change, relative to its own size
    assert _rel(s.get_u(), ref) < 1e-14
    flags, _ = s.status()
    assert flags == 0
    s.close()


def test_c3_riemann_large_single_evaluations_match_oracle(oracle_lib):
    from dnds_b200.solver import Solver

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    m = M.riemann_mesh(1024)
    cfg = S.preset("riemann")
    u = mg.perturbed_quadrants(m)
    z = np.zeros((m.n_cells, 5, 4))
    o = oracle_lib.Oracle(m, cfg, n_threads=0)
    o.set_u(u)
    o.set_urec(z)
    o.vr_step(2)
    s = Solver(m, cfg, precision=0)
    s.set_u(u)
    s.set_urec(z)
    s.ReconstructionJacobiStep(2)
    assert _rel(s.face_values(0.0), o.face_values(0.0)) < 1e-11
    ind_o = o.limiter(False)
    ind_s = s.ReconstructionWBAPLimitFacialV3(False, indicator=True)
    scale = cfg["vfvSetting"]["WBAP_SmoothIndicatorScale"]
    assert (ind_o >= scale).sum() > 1000
    assert np.array_equal(ind_o >= scale, ind_s >= scale)
    assert _rel(s.face_values(0.0), o.face_values(0.0)) < 1e-11
    _, dmin_o = o.eval_dt(0.4)
    assert abs(s.EvaluateDt(0.4) - dmin_o) < 1e-13 * dmin_o
    rhs_o, _ = o.eval_rhs(0.0)
    del o
    assert _rel(s.EvaluateRHS(0.0), rhs_o) < 1e-11
    s.close()


@pytest.mark.parametrize("parts", [1, 16])
def test_c4_sa_full_size_iterations_match_oracle(oracle_lib, parts):
    from dnds_b200.partition import block_owner
    from dnds_b200.solver import Solver

    m = M.naca0012_cmesh()
    cfg = S.preset("naca0012_sa")
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    o = oracle_lib.Oracle(m, cfg, n_threads=0)
    s = Solver(m, cfg, precision=0)
    s.lusgs_set_order(1)
    if parts > 1:
        p = block_owner(m.n_cells, parts)
        o.set_lusgs_parts(p)
        s.lusgs_set_parts(p, parts)
    o.set_u(u0)
    s.set_u(u0)
    s.bdf_begin()
    for _ in range(3):
        res, _ = s.implicit_iteration(100.0)
        inc = o.implicit_iteration(100.0, u0)
        assert abs(res[0] - np.abs(inc[:, 0]).sum()) < 1e-9 * res[0]
    assert _rel(s.get_u(), o.get_u()) < 1e-9
    flags, _ = s.status()
    assert flags == 0
    s.close()
