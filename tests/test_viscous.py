"""The Navier-Stokes viscous flux (NS_2D with mu > 0): the oracle's restatement of
fluxFace's viscous part and of EvaluateRHS's face gradient, and the GPU path against it.

Tolerances: FP64 GPU vs FP64 oracle 1e-11 relative for one evaluation and 1e-10 after
20 implicit iterations in the same (natural) sweep order; FP32 bulk 2e-5 on the RHS.
"""
import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S


def _mesh():
    return M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0)  # no-slip wall


def _cfg():
    return S.preset("naca0012_laminar")


def _free_stream(m, cfg):
    return np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# ---------------------------------------------------------------------- CPU
def test_gas_settings_from_reference_keys():
    s = S.make_settings(_cfg())
    assert s.mu_gas == pytest.approx(1 / 5000.0) and s.pr_gas == pytest.approx(0.72)
    assert s.cp_gas == pytest.approx(1.4 / 0.4)  # Rgas gamma / (gamma - 1)
    assert S.make_settings(S.preset("naca0012")).mu_gas == 0.0  # no muGas: inviscid


def test_oracle_viscous_free_stream_preserved(oracle_lib):
    """A uniform state has zero gradients and zero jumps: the viscous flux vanishes and the
    periodic free stream stays a steady state."""
    m = M.vortex_mesh(8, True, jitter=0.2)
    cfg = S.preset("vortex", eulerSetting={"riemannSolverType": "Roe",
                                           "idealGasProperty": S.laminar_gas(0.5, 100.0),
                                           "farFieldStaticValue": [1.0, 1.0, 1.0, 3.5]})
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    o.set_u(np.tile([1.0, 0.3, -0.2, 3.0], (m.n_cells, 1)))
    o.vr_step(3)
    rhs, _ = o.eval_rhs(0.0)
    assert np.abs(rhs).max() < 1e-12


def test_oracle_laminar_naca_is_symmetric_with_positive_drag(oracle_lib):
    """Laminar NACA 0012 at alpha 0: the converged wall force has no lift and a drag of the
    size a Re 5000 airfoil has (skin friction plus pressure drag, ~0.05-0.07 on this mesh)."""
    m, cfg = _mesh(), _cfg()
    u0 = _free_stream(m, cfg)
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    base = None
    for it in range(4000):
        r = np.abs(o.implicit_iteration(50.0, u0)[:, 0]).sum()
        base = r if base is None else max(base, r)
        if r / base < 1e-6:
            break
    _, wf = o.eval_rhs(0.0)
    cd, cl = wf[1] / 0.5, wf[2] / 0.5
    assert abs(cl) < 1e-4 and 0.04 < cd < 0.09


# ---------------------------------------------------------------------- GPU
def _state(oracle_lib, m, cfg, n=15):
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    u0 = _free_stream(m, cfg)
    o.set_u(u0)
    for _ in range(n):
        o.implicit_iteration(50.0, u0)
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 2e-5)])
def test_viscous_dt_and_rhs_match_oracle(oracle_lib, precision, tol):
    from dnds_b200.solver import Solver

    m, cfg = _mesh(), _cfg()
    o = _state(oracle_lib, m, cfg)
    u, urec = o.get_u(), o.get_urec()
    s = Solver(m, cfg, precision=precision)
    s.set_u(u)
    s.set_urec(urec)
    dmin = s.EvaluateDt(50.0, use_local_dt=True)
    dt_ref, dmin_ref = o.eval_dt(50.0, use_local_dt=True)
    assert _rel(s.get_dt(), dt_ref) < 1e-13 and abs(dmin - dmin_ref) < 1e-13 * dmin_ref
    rhs = s.EvaluateRHS(0.0)
    ref, _ = o.eval_rhs(0.0)
    assert _rel(rhs, ref) < tol
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.gpu
def test_viscous_implicit_iterations_match_oracle(oracle_lib):
    from dnds_b200.solver import Solver

    m, cfg = _mesh(), _cfg()
    u0 = _free_stream(m, cfg)
    s = Solver(m, cfg, precision=0)
    s.lusgs_set_order(1)  # the reference's natural sweep order
    s.set_u(u0)
    s.bdf_begin()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    for _ in range(20):
        s.implicit_iteration(50.0)
        o.implicit_iteration(50.0, u0)
    ref = o.get_u()
    assert _rel(s.get_u(), ref) < 1e-10


@pytest.mark.gpu
def test_viscous_steady_force_fp32_within_1e4_of_fp64():
    from dnds_b200.solver import Solver

    m, cfg = _mesh(), _cfg()
    u0 = _free_stream(m, cfg)
    forces = {}
    for prec in (0, 1):
        s = Solver(m, cfg, precision=prec)
        s.lusgs_set_order(1)
        s.set_u(u0)
        it, rel, wf = s.steady_solve(50.0, 1e-6, 6000)
        assert rel[0] < 1e-6
        forces[prec] = wf
    cd64, cd32 = forces[0][1] / 0.5, forces[1][1] / 0.5
    assert 0.04 < cd64 < 0.09
    assert abs(cd32 - cd64) < 1e-4 * abs(cd64)
