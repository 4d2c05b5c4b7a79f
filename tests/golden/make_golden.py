"""Generates the golden fixtures of the parity tests from the FP64 oracle.

Run from the repository root:  python tests/golden/make_golden.py
Each case: a small synthetic mesh, its initial state, and the oracle's
outputs (face Gauss-point states after 3 VR Jacobi sweeps, EvaluateDt,
EvaluateRHS, and the state after 2 SSP-RK3 steps).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import pyoracle  # noqa: E402
from dnds_b200 import geometry as G  # noqa: E402
from dnds_b200 import mesh as M  # noqa: E402
from dnds_b200 import settings as S  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def smooth_state(m):
    return G.cell_average(m, lambda x, y: np.stack(
        [1 + 0.1 * np.sin(x) * np.cos(y), 0.3 + 0.05 * x, -0.2 + 0.05 * y, 2.5 + 0.1 * np.cos(x)], -1))


CASES = {
    "vortex_quad10": (lambda: M.vortex_mesh(10, False), "vortex", lambda m: G.isentropic_vortex(m)),
    "vortex_tri8_jitter": (lambda: M.vortex_mesh(8, True, jitter=0.2, seed=1234), "vortex",
                           lambda m: G.isentropic_vortex(m)),
    "riemann_tri8": (lambda: M.riemann_mesh(8, jitter=0.15, seed=4321), "riemann",
                     lambda m: G.quadrant_states(m, S.RIEMANN_2D_STATES)),
    "eulerwall_quad6x5": (lambda: M.structured_grid(6, 5, 2.0, 1.0, triangles=False, jitter=0.2, periodic=False,
                                                     bc=M.BC_WALL_EULER), "vortex", smooth_state),
    "farfield_tri6x5": (lambda: M.structured_grid(6, 5, 2.0, 1.0, triangles=True, jitter=0.2, periodic=False,
                                                   bc=M.BC_FARFIELD), "vortex", smooth_state),
}


def perturbed_quadrants(m):
    """Four-quadrant Riemann states times a smooth perturbation, so that no
    reconstruction coefficient is zero up to rounding: the WBAP biway of the
    reference uses sign(u2), which jumps at u2 = 0, so on exactly constant
    regions the limiter's decision depends on rounding noise."""
    q = np.array(S.RIEMANN_2D_STATES)

    def f(x, y):
        k = np.where(x > 0.8, np.where(y > 0.8, 0, 3), np.where(y > 0.8, 1, 2))
        pert = 1.0 + 0.05 * np.sin(6.3 * x + 1.1) * np.cos(5.1 * y + 0.3)
        rho, u, v, p = q[k, 0] * pert, q[k, 1] + 0.02 * pert, q[k, 2] - 0.01 * pert, q[k, 3] * pert
        return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], -1)

    return G.cell_average(m, f)


def make_limiter_case(procedure=1):
    """2-D Riemann mesh with the CWBAP limiter (procedure 1, ReconstructionWBAPLimitFacialV3) or the
    3WBAP limiter (procedure 0, ReconstructionWBAPLimitFacialV2): indicator and limited face states
    after 3 VR sweeps, the same with every cell limited (from a fresh reconstruction), then 2 SSP-RK3
    steps with the limiter in every stage."""
    m = M.riemann_mesh(16, jitter=0.15, seed=4321)
    cfg = S.preset("riemann", limiterProcedure=procedure)
    o = pyoracle.Oracle(m, cfg, n_threads=1)
    lim = o.limiter if procedure == 1 else o.limiter_v2
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    o.set_u(u0)
    o.vr_step(3)
    ind = lim(False)
    fv = o.face_values(0.0)
    # every cell limited, from the same unlimited reconstruction
    o.set_urec(np.zeros((m.n_cells, 5, 4)))
    o.vr_step(3)
    lim(True)
    fv_all = o.face_values(0.0)
    up = perturbed_quadrants(m)
    o.set_u(up)
    o.set_urec(np.zeros((m.n_cells, 5, 4)))
    t = 0.0
    for _ in range(2):
        _, d = o.eval_dt(0.4)
        o.ssprk3_step(d, t)
        t += d
    return dict(u0=u0, indicator=ind, face_values_lim=fv, face_values_limall=fv_all, u0_perturbed=up,
                u_rk2=o.get_u(), t_rk2=t)


def make_case(name):
    if name == "riemann_tri16_limiter":
        return make_limiter_case(1)
    if name == "riemann_tri16_limiter_v2":
        return make_limiter_case(0)
    mk, pre, init = CASES[name]
    m = mk()
    cfg = S.preset(pre, useLimiter=False)
    o = pyoracle.Oracle(m, cfg, n_threads=1)
    u0 = init(m)
    o.set_u(u0)
    o.vr_step(3)
    fv = o.face_values(0.1)
    dt, dtmin = o.eval_dt(0.5)
    rhs, _ = o.eval_rhs(0.1)
    # two SSP-RK3 steps from u0 with a fresh reconstruction
    o.set_u(u0)
    o.set_urec(np.zeros((m.n_cells, 5, 4)))
    t = 0.0
    for _ in range(2):
        _, d = o.eval_dt(0.5)
        o.ssprk3_step(d, t)
        t += d
    u2 = o.get_u()
    return dict(u0=u0, face_values=fv, dt=dt, dtmin=dtmin, rhs=rhs, u_rk2=u2, t_rk2=t)


LIMITER_CASES = ["riemann_tri16_limiter", "riemann_tri16_limiter_v2"]

if __name__ == "__main__":
    pyoracle.build()
    for name in list(CASES) + LIMITER_CASES:
        d = make_case(name)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **d)
        print(name, {k: np.shape(v) for k, v in d.items()})
