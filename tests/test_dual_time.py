"""Dual time stepping, the reference's implicit driver: ImplicitSDIRK4DualTimeStep and
ImplicitBDFDualTimeStep (DNDS_ODE.hpp:269-497) with the EulerSolver's fdtau / frhs / fsolve /
fstop, and fsolve's GMRES over LUSGSMatrixVec with the LU-SGS sweeps as preconditioner
(DNDS_Linear.hpp:12-107, DNDS_FV_EulerEvaluator.cpp:1062-1143).

The oracle is pinned by properties the schemes must have: one BDF1 step is the first-order
pseudo-time iteration already checked against the reference; the temporal orders of BDF1 / BDF2 /
SDIRK4 on the periodic isentropic vortex (self-convergence in dt on a fixed mesh, so the spatial
error cancels); GMRES and LU-SGS inner solvers reach the same converged step.  The GPU path is then
held to the oracle at a fixed number of internal iterations: FP64 1e-10 relative on u (the dot
products and Givens rotations of GMRES sum in a different order than the oracle's Householder
least squares).
"""
import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S


def _vortex(n=10):
    return M.vortex_mesh(n, False, jitter=0.1)


def _vortex_cfg():
    return S.preset("vortex")


def _naca_small():
    return M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0, wall_bc=M.BC_WALL_EULER)


def _naca_cfg():
    return S.preset("naca0012", eulerSetting={"riemannSolverType": "Roe", "idealGasProperty": {"gamma": 1.4},
                                              "farFieldStaticValue": S.free_stream(0.5, 2.0)})


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# ---------------------------------------------------------------------- CPU
def test_oracle_bdf1_step_is_the_pseudo_time_iteration(oracle_lib):
    m, cfg = _vortex(8), _vortex_cfg()
    a = oracle_lib.Oracle(m, cfg, n_threads=2)
    a.init_vortex()
    u0 = a.get_u()
    b = oracle_lib.Oracle(m, cfg, n_threads=2)
    b.set_u(u0)
    its, _ = a.dual_step(0.3, scheme="bdf", bdf_order=1, cfl=20.0, max_iter=6)
    assert its[0] == 6
    for _ in range(6):
        b.implicit_iteration(20.0, u0, dt=0.3)
    assert _rel(a.get_u(), b.get_u()) < 1e-12


def _self_convergence(oracle_lib, scheme, order, dts, t_end=0.4):
    m, cfg = _vortex(10), _vortex_cfg()
    sol = []
    for dt in dts:
        o = oracle_lib.Oracle(m, cfg, n_threads=2)
        o.init_vortex()
        t = 0.0
        for _ in range(int(round(t_end / dt))):
            o.dual_step(dt, t, scheme=scheme, bdf_order=order, cfl=100.0, max_iter=80, threshold=1e-12)
            t += dt
        sol.append(o.get_u())
    ref = sol[-1]
    return [np.abs(u - ref).max() for u in sol[:-1]]


@pytest.mark.parametrize("scheme,order,lo,hi", [("bdf", 1, 1.6, 2.6), ("bdf", 2, 3.0, 5.5), ("sdirk4", 0, 9.0, 40.0)])
def test_oracle_temporal_order(oracle_lib, scheme, order, lo, hi):
    """Halving dt divides the error by about 2^p: p = 1 (BDF1), 2 (BDF2, started by a BDF1 step),
    4 (SDIRK4).  The finest dt is the reference solution."""
    e = _self_convergence(oracle_lib, scheme, order, [0.2, 0.1, 0.0125])
    assert lo < e[0] / e[1] < hi, e


def test_oracle_gmres_and_lusgs_reach_the_same_step(oracle_lib):
    m, cfg = _vortex(8), _vortex_cfg()
    out, its = {}, {}
    for code in (0, 1, 2):
        o = oracle_lib.Oracle(m, cfg, n_threads=2)
        o.init_vortex()
        i, _ = o.dual_step(0.5, scheme="bdf", bdf_order=2, cfl=100.0, max_iter=200, threshold=1e-11,
                           gmres_code=code, n_gmres_space=6, n_gmres_iter=1)
        out[code], its[code] = o.get_u(), i[0]
    assert _rel(out[1], out[0]) < 1e-8 and _rel(out[2], out[0]) < 1e-8
    assert its[1] <= its[0] and its[2] <= its[0]  # never more outer iterations than with LU-SGS alone


def _linear_system(o, m, cfg, alpha=0.6, dt=0.1):
    """A non-uniform state, its LU-SGS diagonal, and LUSGSMatrixVec assembled column by column."""
    o.init_vortex()
    o.eval_dt(30.0, use_local_dt=True)
    o.lusgs_matrix_init(dt, alpha)
    n = m.n_cells * 4
    A = np.empty((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        A[:, k] = o.lusgs_matvec(e.reshape(-1, 4), alpha).ravel()
    return A


def test_oracle_gmres_solves_the_lusgs_matrix_system(oracle_lib):
    """GMRES over LUSGSMatrixVec, LU-SGS preconditioned, against a dense solve of the same matrix
    (assembled from the matrix-vector product): enough Krylov vectors and restarts reach it."""
    m, cfg = _vortex(6), _vortex_cfg()
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    A = _linear_system(o, m, cfg)
    b = np.random.default_rng(7).standard_normal(A.shape[0])
    ref = np.linalg.solve(A, b)
    x = o.gmres_lusgs(b.reshape(-1, 4), alpha=0.6, n_space=20, n_restart=6).ravel()
    assert np.abs(x - ref).max() < 1e-9 * np.abs(ref).max()
    # one short cycle already beats the preconditioner alone
    x1 = o.gmres_lusgs(b.reshape(-1, 4), alpha=0.6, n_space=4, n_restart=1).ravel()
    m0 = np.zeros_like(b).reshape(-1, 4)
    o.lusgs_forward(b.reshape(-1, 4), m0, 0.6)
    o.lusgs_backward(b.reshape(-1, 4), m0, 0.6)
    assert np.linalg.norm(A @ x1 - b) < np.linalg.norm(A @ m0.ravel() - b)


def test_oracle_bdf_history_needs_a_constant_dt(oracle_lib):
    m, cfg = _vortex(8), _vortex_cfg()
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    o.init_vortex()
    o.dual_step(0.2, scheme="bdf", bdf_order=2, max_iter=2)
    with pytest.raises(RuntimeError):
        o.dual_step(0.1, scheme="bdf", bdf_order=2, max_iter=2)
    o.dual_reset()
    o.dual_step(0.1, scheme="bdf", bdf_order=2, max_iter=2)


# ---------------------------------------------------------------------- GPU
def _pair(oracle_lib, m, cfg, u0):
    from dnds_b200.solver import Solver

    s = Solver(m, cfg, precision=0)
    s.lusgs_set_order(1)  # the reference's natural sweep order
    s.set_u(u0)
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    return s, o


def _vortex_state(oracle_lib, m, cfg):
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    o.init_vortex()
    return o.get_u()


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,order", [("bdf", 2), ("sdirk4", 0), ("bdf", 3)])
@pytest.mark.parametrize("gmres_code", [0, 1, 2])
def test_dual_step_matches_oracle(oracle_lib, scheme, order, gmres_code):
    """The isentropic vortex on 16 x 16 x 2 jittered periodic triangles, natural sweep order, a
    fixed number of internal iterations (3 per stage); BDF runs 3 steps so the history is used."""
    m, cfg = M.vortex_mesh(16, True, jitter=0.2), _vortex_cfg()
    s, o = _pair(oracle_lib, m, cfg, _vortex_state(oracle_lib, m, cfg))
    kw = dict(scheme=scheme, bdf_order=max(order, 1), cfl=50.0, max_iter=3, threshold=1e-100, gmres_code=gmres_code,
              n_gmres_space=4, n_gmres_iter=1)
    nsteps = 3 if scheme == "bdf" else 1
    for k in range(nsteps):
        its, res = s.dual_step(0.1, 0.1 * k, **kw)
        rits, rres = o.dual_step(0.1, 0.1 * k, **kw)
        assert list(its) == list(rits)
        assert abs(res[0] - rres[0]) < 1e-8 * abs(rres[0])
    u, ref = s.get_u(), o.get_u()
    assert np.isfinite(ref).all() and _rel(u, ref) < 1e-10
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.gpu
def test_dual_step_with_walls_matches_oracle(oracle_lib):
    """BDF2 with GMRES on the NACA 0012 C-mesh (Euler wall, far field), impulsive start, a small
    physical step; the threshold ends the internal loops (fstop)."""
    m, cfg = _naca_small(), _naca_cfg()
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    s, o = _pair(oracle_lib, m, cfg, u0)
    kw = dict(scheme="bdf", bdf_order=2, cfl=20.0, max_iter=30, threshold=1e-3, gmres_code=2, n_gmres_space=5,
              n_gmres_iter=1)
    for k in range(2):
        its, _ = s.dual_step(2e-3, 2e-3 * k, **kw)
        rits, _ = o.dual_step(2e-3, 2e-3 * k, **kw)
        assert its[0] == rits[0] and its[0] < 30
    u, ref = s.get_u(), o.get_u()
    assert np.isfinite(ref).all() and _rel(u, ref) < 1e-10


@pytest.mark.gpu
def test_dual_step_colour_batches_match_oracle_in_colour_order(oracle_lib):
    from dnds_b200.solver import Solver

    m, cfg = M.vortex_mesh(16, True, jitter=0.2), _vortex_cfg()
    u0 = _vortex_state(oracle_lib, m, cfg)
    s = Solver(m, cfg, precision=0)
    col, _ = s.lusgs_colours()
    scan = np.argsort(col, kind="stable")
    s.set_u(u0)
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    kw = dict(scheme="sdirk4", cfl=50.0, max_iter=4, threshold=1e-100, gmres_code=2, n_gmres_space=5, n_gmres_iter=1)
    s.dual_step(0.1, 0.0, **kw)
    o.dual_step(0.1, 0.0, scan2cell=scan, **kw)
    u, ref = s.get_u(), o.get_u()
    assert np.isfinite(ref).all() and _rel(u, ref) < 1e-10


def _sa_case():
    m = M.naca0012_cmesh(32, 16, 16, first=1e-3, far=10.0)  # no-slip wall
    return m, S.naca0012_sa(0.15, 10.0, 1e5)


def test_oracle_sa_bdf1_step_is_the_pseudo_time_iteration(oracle_lib):
    m, cfg = _sa_case()
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    a = oracle_lib.Oracle(m, cfg, n_threads=4)
    a.set_u(u0)
    a.dual_step(0.01, scheme="bdf", bdf_order=1, cfl=20.0, max_iter=4)
    b = oracle_lib.Oracle(m, cfg, n_threads=4)
    b.set_u(u0)
    for _ in range(4):
        b.implicit_iteration(20.0, u0, dt=0.01)
    assert _rel(a.get_u(), b.get_u()) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,gmres_code", [("bdf", 0), ("bdf", 2), ("sdirk4", 1)])
def test_sa_dual_step_matches_oracle(oracle_lib, scheme, gmres_code):
    """RANS-SA (5 variables, no-slip wall) in dual time: the U5 rhs and increment pass through
    CompressInc; BDF2 runs 2 steps so the history is used."""
    m, cfg = _sa_case()
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    s, o = _pair(oracle_lib, m, cfg, u0)
    kw = dict(scheme=scheme, bdf_order=2, cfl=20.0, max_iter=3, threshold=1e-100, gmres_code=gmres_code,
              n_gmres_space=4, n_gmres_iter=1)
    for k in range(2 if scheme == "bdf" else 1):
        its, res = s.dual_step(1e-3, 1e-3 * k, **kw)
        rits, rres = o.dual_step(1e-3, 1e-3 * k, **kw)
        assert list(its) == list(rits) and len(res) == 5
    u, ref = s.get_u(), o.get_u()
    assert np.isfinite(ref).all() and ref[:, 4].min() > 0
    assert _rel(u[:, :4], ref[:, :4]) < 1e-9 and _rel(u[:, 4], ref[:, 4]) < 1e-9
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.gpu
def test_dual_step_with_the_limiter_matches_oracle(oracle_lib):
    """The 2-D Riemann problem with the CWBAP limiter in frhs (HLLC, far-field Riemann boundary states):
    BDF2 with LU-SGS in the natural order, 2 steps of 2 internal iterations."""
    from dnds_b200 import geometry as G

    m, cfg = M.riemann_mesh(24), S.preset("riemann")
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    s, o = _pair(oracle_lib, m, cfg, u0)
    kw = dict(scheme="bdf", bdf_order=2, cfl=5.0, max_iter=2, threshold=1e-100, gmres_code=0)
    for k in range(2):
        s.dual_step(2e-3, 2e-3 * k, **kw)
        o.dual_step(2e-3, 2e-3 * k, **kw)
    u, ref = s.get_u(), o.get_u()
    assert np.isfinite(ref).all() and _rel(u, ref) < 1e-10


@pytest.mark.gpu
def test_dual_step_fp32_bulk_close_to_fp64():
    """FP32-bulk contexts (FP32 coefficients, FP64 means and increments) in dual time: SDIRK4 with
    GMRES on the vortex agrees with the FP64 context to 1e-5 relative."""
    from dnds_b200 import geometry as G
    from dnds_b200.solver import Solver

    m, cfg = M.vortex_mesh(16, True, jitter=0.2), _vortex_cfg()
    out = []
    for prec in (0, 1):
        s = Solver(m, cfg, precision=prec)
        s.set_u(G.isentropic_vortex(m))
        s.dual_step(0.1, 0.0, scheme="sdirk4", cfl=50.0, max_iter=4, threshold=1e-100, gmres_code=2, n_gmres_space=4,
                    n_gmres_iter=1)
        out.append(s.get_u())
    assert _rel(out[1], out[0]) < 1e-5


@pytest.mark.gpu
def test_sdirk4_step_conserves_at_full_size():
    """The SDIRK4 update x = xLast + dt sum b_j R_j is conservative whatever the inner convergence:
    on the periodic 2,097,152-triangle vortex the volume-weighted totals of all four conserved
    variables stay put to round-off after one step of 2 internal iterations per stage."""
    from dnds_b200 import geometry as G
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(1024, True, jitter=0.2)
    s = Solver(m, _vortex_cfg(), precision=0)
    u0 = G.isentropic_vortex(m)
    s.set_u(u0)
    vol = G.cell_quadrature(m)[1].sum(1)
    before = (u0 * vol[:, None]).sum(0)
    its, _ = s.dual_step(0.05, 0.0, scheme="sdirk4", cfl=50.0, max_iter=2, threshold=1e-100)
    assert list(its) == [2, 2, 2]
    u = s.get_u()
    after = (u * vol[:, None]).sum(0)
    assert np.isfinite(u).all() and np.abs(u - u0).max() > 1e-8  # it moved
    assert np.all(np.abs(after - before) < 1e-11 * np.abs(before).max())


@pytest.mark.gpu
def test_lusgs_matvec_matches_oracle(oracle_lib):
    import torch

    m, cfg = _naca_small(), _naca_cfg()
    u0 = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    for _ in range(20):  # a non-uniform state
        o.implicit_iteration(50.0, u0)
    u, urec = o.get_u(), o.get_urec()
    s, _ = _pair(oracle_lib, m, cfg, u)
    s.set_urec(urec)
    s.EvaluateDt(50.0, use_local_dt=True)
    s.LUSGSMatrixInit(0.1, 0.6)
    o.eval_dt(50.0, use_local_dt=True)
    o.lusgs_matrix_init(0.1, 0.6)
    x = np.random.default_rng(3).standard_normal((m.n_cells, 4))
    xd = torch.tensor(x, device="cuda:0")
    ax = torch.empty_like(xd)
    s.LUSGSMatrixVec(0.6, xd.data_ptr(), ax.data_ptr())
    ref = o.lusgs_matvec(x, 0.6)
    assert _rel(ax.cpu().numpy(), ref) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("order", [0, 1])
def test_gmres_lusgs_matches_oracle(oracle_lib, order):
    import torch

    m, cfg = _vortex(16), _vortex_cfg()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.init_vortex()
    u = o.get_u()
    from dnds_b200.solver import Solver

    s = Solver(m, cfg, precision=0)
    nb = s.lusgs_set_order(order)
    scan = np.argsort(s.lusgs_colours()[0], kind="stable") if order == 0 else None
    s.set_u(u)
    s.EvaluateDt(30.0, use_local_dt=True)
    s.LUSGSMatrixInit(0.1, 0.6)
    o.eval_dt(30.0, use_local_dt=True)
    o.lusgs_matrix_init(0.1, 0.6)
    b = np.random.default_rng(11).standard_normal((m.n_cells, 4))
    bd = torch.tensor(b, device="cuda:0")
    xd = torch.zeros_like(bd)
    s.gmres_lusgs(0.6, 8, 2, bd.data_ptr(), xd.data_ptr())
    ref = o.gmres_lusgs(b, alpha=0.6, n_space=8, n_restart=2, scan2cell=scan)
    assert _rel(xd.cpu().numpy(), ref) < 1e-10


@pytest.mark.gpu
def test_dual_step_rejects_bad_settings():
    from dnds_b200.solver import DndsgError, Solver

    m, cfg = _naca_small(), _naca_cfg()
    s = Solver(m, cfg, precision=0)
    s.set_u(np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1)))
    with pytest.raises(DndsgError):
        s.dual_step(0.1, scheme="bdf", bdf_order=5)
    with pytest.raises(DndsgError):
        s.dual_step(0.1, gmres_code=1, n_gmres_space=40)
    s.dual_step(0.1, scheme="bdf", bdf_order=2, max_iter=1)
    with pytest.raises(DndsgError):
        s.dual_step(0.2, scheme="bdf", bdf_order=2, max_iter=1)
