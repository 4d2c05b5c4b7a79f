"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances: FP64 GPU path vs FP64 oracle, relative to the field's max
magnitude, 1e-11 for one evaluation and 1e-10 after a few RK steps (the two
differ only in summation order, FMA contraction and the 5x5 solver).  The
FP32-bulk path is held to 2e-6 (relative) on single evaluations.
"""
import os

import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def _solver(m, cfg, precision=0):
    from dnds_b200.solver import Solver

    return Solver(m, cfg, precision=precision)


def _golden_case(name):
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mk, pre, _ = mg.CASES[name]
    return mk(), S.preset(pre, useLimiter=False), np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


CASES = ["vortex_quad10", "vortex_tri8_jitter", "riemann_tri8", "eulerwall_quad6x5", "farfield_tri6x5"]


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_golden(name):
    m, cfg, ref = _golden_case(name)
    s = _solver(m, cfg, 0)
    s.set_u(ref["u0"])
    s.ReconstructionJacobiStep(3)
    assert _rel(s.face_values(0.1), ref["face_values"]) < 1e-11
    dtmin = s.EvaluateDt(0.5, use_local_dt=False)
    assert abs(dtmin - float(ref["dtmin"])) < 1e-13 * float(ref["dtmin"])
    assert _rel(s.get_dt(), ref["dt"]) < 1e-13
    rhs = s.EvaluateRHS(0.1)
    assert _rel(rhs, ref["rhs"]) < 1e-11
    flags, _ = s.status()
    assert flags == 0
    # two SSP-RK3 steps from u0 and a zero reconstruction
    s.set_u(ref["u0"])
    s.set_urec(np.zeros((m.n_cells, 5, 4)))
    s.time = 0.0
    for _ in range(2):
        s.ssprk3_step(0.5, 1e300)
    assert _rel(s.get_u(), ref["u_rk2"]) < 1e-12
    assert abs(s.time - float(ref["t_rk2"])) < 1e-14


@pytest.mark.parametrize("name", ["vortex_tri8_jitter", "riemann_tri8", "eulerwall_quad6x5"])
def test_fp32_bulk_close_to_golden(name):
    m, cfg, ref = _golden_case(name)
    s = _solver(m, cfg, 1)
    s.set_u(ref["u0"])
    s.ReconstructionJacobiStep(3)
    assert _rel(s.face_values(0.1), ref["face_values"]) < 2e-6
    s.EvaluateDt(0.5, use_local_dt=True)
    rhs = s.EvaluateRHS(0.1)
    assert _rel(rhs, ref["rhs"]) < 2e-5


@pytest.mark.parametrize("procedure", [1, 0])
@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-4)])
def test_limiter_matches_golden(precision, tol, procedure):
    """The WBAP limiters and SSP-RK3 with the limiter in every stage, 2-D Riemann mesh: CWBAP
    (limiterProcedure 1, ReconstructionWBAPLimitFacialV3) and 3WBAP (limiterProcedure 0,
    ReconstructionWBAPLimitFacialV2)."""
    m = M.riemann_mesh(16, jitter=0.15, seed=4321)
    name = "riemann_tri16_limiter" if procedure == 1 else "riemann_tri16_limiter_v2"
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    s = _solver(m, S.preset("riemann", limiterProcedure=procedure), precision)
    limit = s.ReconstructionWBAPLimitFacialV3 if procedure == 1 else s.ReconstructionWBAPLimitFacialV2
    s.set_u(ref["u0"])
    s.ReconstructionJacobiStep(3)
    ind = limit(False, indicator=True)
    assert _rel(ind, ref["indicator"]) < tol
    assert _rel(s.face_values(0.0), ref["face_values_lim"]) < tol
    s.set_urec(np.zeros((m.n_cells, 5, 4)))
    s.ReconstructionJacobiStep(3)
    limit(True)
    assert _rel(s.face_values(0.0), ref["face_values_limall"]) < tol
    # multi-step parity on a smoothly perturbed state (no coefficient is zero up to rounding,
    # where the reference's sign(u2) in the biway WBAP is discontinuous)
    s.set_u(ref["u0_perturbed"])
    s.set_urec(np.zeros((m.n_cells, 5, 4)))
    s.time = 0.0
    for _ in range(2):
        s.ssprk3_step(0.4, 1e300)
    assert _rel(s.get_u(), ref["u_rk2"]) < (1e-11 if precision == 0 else 1e-5)
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.parametrize("precision", [0, 1])
def test_limiter_changes_only_the_cells_it_lists(precision):
    """The indicator pass lists the cells with si >= WBAP_SmoothIndicatorScale and only those are
    limited: every other cell keeps its coefficients bit for bit.  A free stream lists no cell at all."""
    m = M.riemann_mesh(48, jitter=0.15, seed=4321)
    cfg = S.preset("riemann")
    scale = cfg["vfvSetting"]["WBAP_SmoothIndicatorScale"]
    s = _solver(m, cfg, precision)
    s.set_u(G.quadrant_states(m, S.RIEMANN_2D_STATES))
    s.ReconstructionJacobiStep(3)
    before = s.get_urec()
    ind = s.ReconstructionWBAPLimitFacialV3(False, indicator=True)
    after = s.get_urec()
    keep = ind < scale
    assert keep.any() and (~keep).any()
    assert np.array_equal(after[keep], before[keep])
    assert not np.array_equal(after[~keep], before[~keep])
    # a free stream: the reconstruction vanishes, no indicator reaches the scale, nothing changes
    s.set_u(np.tile(G.quadrant_states(m, S.RIEMANN_2D_STATES)[:1], (m.n_cells, 1)))
    s.set_urec(np.zeros((m.n_cells, 5, 4)))
    s.ReconstructionJacobiStep(2)
    before = s.get_urec()
    ind = s.ReconstructionWBAPLimitFacialV3(False, indicator=True)
    assert (ind < scale).all()
    assert np.array_equal(s.get_urec(), before)
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replayed_steps_equal_single_steps(precision):
    """dndsg_ssprk3_steps (pairs of steps from a CUDA graph) computes what the same number of
    dndsg_ssprk3_step calls computes, bit for bit: odd counts, a coefficient-buffer parity flipped by a
    lone VR sweep in between, a new cfl (a second capture), and the limiter on the Riemann mesh."""
    cases = [(M.vortex_mesh(16, True, jitter=0.2), S.preset("vortex"), None, 0.5),
             (M.riemann_mesh(16, jitter=0.15, seed=4321), S.preset("riemann"), S.RIEMANN_2D_STATES, 0.4)]
    for m, cfg, states, cfl in cases:
        u0 = G.isentropic_vortex(m) if states is None else G.quadrant_states(m, states)
        a, b = _solver(m, cfg, precision), _solver(m, cfg, precision)
        for s in (a, b):
            s.set_u(u0)
        for k in range(5):
            a.ssprk3_step(cfl)
        b.ssprk3_steps(cfl, 5)
        assert np.array_equal(a.get_u(), b.get_u()) and a.time == b.time
        for s in (a, b):
            s.ReconstructionJacobiStep(1)
        for k in range(4):
            a.ssprk3_step(0.8 * cfl)
        b.ssprk3_steps(0.8 * cfl, 4)
        assert np.array_equal(a.get_u(), b.get_u()) and np.array_equal(a.get_urec(), b.get_urec())
        b.ssprk3_steps(cfl, 0)
        for s in (a, b):
            flags, _ = s.status()
            assert flags == 0
            s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_steps_follow_a_new_owned_mask(precision):
    """An owned-cell mask set after the step graph was captured takes effect in the graph steps: the
    cell with the smallest dt is left out of the dt minimum, the steps equal single steps with the
    same mask and differ from steps without it."""
    import ctypes as C

    m, cfg = M.vortex_mesh(16, True, jitter=0.2), S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    a, b, c = (_solver(m, cfg, precision) for _ in range(3))
    for s in (a, b, c):
        s.set_u(u0)
        s.ssprk3_steps(0.5, 2)
    a.EvaluateDt(0.5, use_local_dt=True)
    mask = np.ones(m.n_cells, dtype=np.uint8)
    mask[int(np.argmin(a.get_dt()))] = 0
    for s in (a, b):
        s._check(s.L.dndsg_set_owned(s.h, mask.ctypes.data_as(C.c_void_p)))
    t0 = a.time
    a.ssprk3_steps(0.5, 2)
    for _ in range(2):
        b.ssprk3_step(0.5)
    c.ssprk3_steps(0.5, 2)
    assert np.array_equal(a.get_u(), b.get_u()) and a.time == b.time
    assert a.time - t0 > c.time - t0
    for s in (a, b, c):
        s.close()


def test_vortex_c1_against_oracle(oracle_lib):
    """40x40 periodic quads, P2 VR + Roe, SSP-RK3 CFL 0.5: 20 steps GPU vs oracle."""
    m = M.vortex_mesh(40, False)
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    o = oracle_lib.Oracle(m, cfg)
    o.set_u(u0)
    s = _solver(m, cfg, 0)
    s.set_u(u0)
    t = 0.0
    for _ in range(20):
        _, d = o.eval_dt(0.5)
        o.ssprk3_step(d, t)
        t += d
        s.ssprk3_step(0.5, 1e300)
    assert abs(s.time - t) < 1e-13 * t
    assert _rel(s.get_u(), o.get_u()) < 1e-10
    s.EvaluateRHS(s.time)
    ro, _ = o.eval_rhs(t)
    for p in (1, 2, 3):
        np.testing.assert_allclose(s.EvaluateResidual(p, p == 2), o.residual(ro, p, p == 2), rtol=1e-9)


def test_vr_increment_and_buffers():
    m = M.vortex_mesh(16, True, jitter=0.2)
    s = _solver(m, S.preset("vortex"), 0)
    s.set_u(G.isentropic_vortex(m))
    inc = [s.ReconstructionJacobiStep(1, with_increment=True) for _ in range(30)]
    assert inc[0] > 0 and inc[-1] < inc[0] * 1e-2
    p, nbytes = s.device_buffer(0)
    assert p and nbytes == m.n_cells * 32


def test_full_size_vortex_properties():
    """The 2,097,152-triangle jittered periodic vortex mesh: free-stream
    preservation and discrete conservation of one RHS evaluation, both precisions."""
    m = M.vortex_mesh(1024, True, jitter=0.2, seed=1234)
    for prec in (0, 1):
        s = _solver(m, S.preset("vortex"), prec)
        s.set_u(np.tile([1.0, 1.0, 1.0, 3.5], (m.n_cells, 1)))
        s.ReconstructionJacobiStep(2)
        s.EvaluateDt(0.5)
        rhs = s.EvaluateRHS(0.0)
        assert np.abs(rhs).max() < (1e-9 if prec == 0 else 2e-3)
        s.set_u(G.isentropic_vortex(m))
        s.ReconstructionJacobiStep(2)
        s.EvaluateDt(0.5)
        rhs = s.EvaluateRHS(0.0)
        vol = np.zeros(m.n_cells)
        pts, wts = G.cell_quadrature(m)
        vol = wts.sum(1)
        tot = (rhs * vol[:, None]).sum(0)
        assert np.abs(tot).max() < 1e-10 * np.abs(rhs * vol[:, None]).sum()
        flags, nred = s.status()
        assert flags == 0 and nred == 0
        s.close()


def test_bad_arguments_fail_loudly():
    from dnds_b200.solver import DndsgError

    m = M.vortex_mesh(4, False)
    cfg = S.preset("vortex")
    bad = M.Mesh(m.node_xy, m.cell_nodes, m.face_nodes, m.face_cells.copy(), m.face_bc, m.face_shift)
    bad.face_cells[0, 0] = m.n_cells + 5
    with pytest.raises(DndsgError):
        _solver(bad, cfg)
    with pytest.raises(DndsgError):
        _solver(m, S.preset("vortex", recOrder=3))
