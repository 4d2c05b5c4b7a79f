"""The 2-D four-quadrant Riemann configuration (P2 VR, CWBAP limiter in every stage, HLLC flux,
SSP-RK3 at CFL 0.4, run to t = 0.3) through the C ABI against the FP64 oracle, on a 64 x 64
jittered grid (8,192 triangles) from the configured quadrant states.

The oracle restates ReconstructionWBAPLimitFacialV3 (DNDS_FV_VR.hpp:2053-2329), HLLCFlux_IdealGas
(DNDS_Gas.hpp:312-403) and the Special_2DRiemannFar boundary state (DNDS_FV_EulerEvaluator.hpp:
1126-1243).  Compared: the density and the whole state after 50 steps and at t = 0.3 (both runs take
the same number of steps), relative to the field's largest magnitude.  Tolerances: FP64 1e-10 after
50 steps and 1e-8 at t = 0.3 (the runs differ in summation order and FMA contraction, and the
limiter's switch si >= 0.1 and the positivity fallbacks amplify rounding differences near shocks over
about 1,100 steps); FP32 bulk 2e-4 after 50 steps and 2e-2 at t = 0.3 (L2 of the density difference
relative to the density's L2 within 2e-3).
"""
import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S

pytestmark = pytest.mark.gpu

T_END = 0.3
CFL = 0.4
N_EARLY = 50


@pytest.fixture(scope="module")
def oracle_run(oracle_lib):
    """The oracle's trajectory: the state after N_EARLY steps and at T_END, and the step count."""
    m = M.riemann_mesh(64)
    cfg = S.preset("riemann")
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    o = oracle_lib.Oracle(m, cfg, n_threads=0)
    o.set_u(u0)
    t, steps, early = 0.0, 0, None
    while t < T_END - 1e-12:
        _, d = o.eval_dt(CFL)
        d = min(d, T_END - t)
        o.ssprk3_step(d, t)
        t += d
        steps += 1
        if steps == N_EARLY:
            early = o.get_u()
    return m, cfg, u0, early, o.get_u(), steps, t


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("precision,tol_early,tol_end", [(0, 1e-10, 1e-8), (1, 2e-4, 2e-2)])
def test_riemann_cwbap_hllc_against_oracle(oracle_run, precision, tol_early, tol_end):
    from dnds_b200.solver import Solver

    m, cfg, u0, early, end, steps, t_end = oracle_run
    s = Solver(m, cfg, precision=precision)
    s.set_u(u0)
    for _ in range(N_EARLY):
        s.ssprk3_step(CFL, T_END)
    e_early = _rel(s.get_u(), early)
    n = N_EARLY + s.run_to(T_END, CFL)
    u = s.get_u()
    e_end = _rel(u, end)
    vol = G.cell_quadrature(m)[1].sum(1)
    d = u[:, 0] - end[:, 0]
    l2_rel = np.sqrt((d * d * vol).sum() / (end[:, 0] ** 2 * vol).sum())
    print(f"precision {precision}: after {N_EARLY} steps {e_early:.3e}; at t = {T_END} ({n} steps, oracle "
          f"{steps}) max {e_end:.3e}, density L2 {l2_rel:.3e}")
    assert n == steps
    assert abs(s.time - t_end) < 1e-14
    assert e_early < tol_early
    assert e_end < tol_end
    if precision == 1:
        assert l2_rel < 2e-3
    flags, _ = s.status()
    assert flags & 1 == 0  # no NaN or non-positive state reached a flux
    s.close()
