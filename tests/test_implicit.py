"""The implicit steady path: colour-batched LU-SGS and first-order BDF pseudo time.

The reference sweeps LU-SGS cell by cell in a scan order
(UpdateLUSGSForward / Backward, DNDS_FV_EulerEvaluator.cpp:1149-1357); the GPU
sweeps colour by colour, which is the same computation in the colour-sorted
scan order.  So, against the oracle run in that order, one sweep pair and a
sequence of pseudo-time iterations agree to FP64 summation order (1e-12 and
1e-10 relative); against the oracle in the natural order only the converged
steady state is comparable (to the convergence level, 1e-6 relative).
"""
import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S


def _naca_small():
    return M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0, wall_bc=M.BC_WALL_EULER)


def _cfg(mach=0.5, alpha=2.0):
    return S.preset("naca0012", eulerSetting={"riemannSolverType": "Roe", "idealGasProperty": {"gamma": 1.4},
                                              "farFieldStaticValue": S.free_stream(mach, alpha)})


def _oracle(oracle_lib, m, cfg):
    return oracle_lib.Oracle(m, cfg, n_threads=4)


def _free_stream(m, cfg):
    return np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))


def _run_oracle(o, x_last, cfl, threshold, max_iter, scan=None):
    base = None
    for it in range(1, max_iter + 1):
        inc = o.implicit_iteration(cfl, x_last, scan2cell=scan)
        r = np.abs(inc).sum(0)
        base = r if base is None else np.maximum(base, r)
        if r[0] / base[0] < threshold:
            break
    return it, r[0] / base[0]


# ---------------------------------------------------------------------- CPU
def test_naca_cmesh_topology():
    m = M.naca0012_cmesh(64, 32, 24, first=1e-4, far=20.0)
    xy = m.node_xy[m.cell_nodes]
    area = 0.5 * sum(xy[:, k, 0] * xy[:, (k + 1) % 4, 1] - xy[:, (k + 1) % 4, 0] * xy[:, k, 1] for k in range(4))
    assert area.min() > 0
    for k in range(4):  # every corner convex
        a, b = xy[:, (k + 1) % 4] - xy[:, k], xy[:, (k + 2) % 4] - xy[:, (k + 1) % 4]
        assert (a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]).min() > 0
    ni, nj = 2 * 32 + 64, 24
    assert m.n_cells == ni * nj
    assert (m.face_bc == M.BC_WALL_NOSLIP).sum() == 64
    assert (m.face_bc == M.BC_FARFIELD).sum() == ni + 2 * nj
    # wall faces lie on the airfoil, and the whole boundary closes: sum of area-weighted normals is zero
    wall = m.face_nodes[m.face_bc == M.BC_WALL_NOSLIP]
    mid = 0.5 * (m.node_xy[wall[:, 0]] + m.node_xy[wall[:, 1]])
    assert mid[:, 0].min() >= 0 and mid[:, 0].max() <= 1 and np.abs(mid[:, 1]).max() < 0.07
    bnd = m.face_nodes[m.face_bc != M.BC_INNER]
    d = m.node_xy[bnd[:, 1]] - m.node_xy[bnd[:, 0]]
    assert np.abs(d.sum(0)).max() < 1e-12
    # first wall-normal spacing
    j1 = m.cell_nodes[: ni * nj: nj][32 + 32]  # first cell row above the mid-chord lower surface
    h = np.linalg.norm(m.node_xy[j1[3]] - m.node_xy[j1[0]])
    assert 0.9e-4 < h < 1.5e-4


def test_line_scan_order_is_a_permutation_with_independent_lines():
    m = _naca_small()
    scan = M.line_scan_order(m)
    assert np.array_equal(np.sort(scan), np.arange(m.n_cells))
    nj = m.meta["nj"]
    line = np.arange(m.n_cells) // nj
    L, R = m.face_cells[:, 0], m.face_cells[:, 1]
    inner = R >= 0
    cross = line[L[inner]] != line[R[inner]]
    # faces between different lines always join lines of opposite parity
    assert np.all((line[L[inner]][cross] - line[R[inner]][cross]) % 2 == 1)


def test_oracle_free_stream_is_a_fixed_point(oracle_lib):
    m = M.vortex_mesh(8, True, jitter=0.2)
    cfg = S.preset("vortex")
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    u = np.tile([1.0, 0.3, -0.2, 3.0], (m.n_cells, 1))
    o.set_u(u)
    inc = o.implicit_iteration(50.0, u)
    assert np.abs(inc).max() < 1e-12


def test_oracle_steady_state_does_not_depend_on_the_scan_order(oracle_lib):
    """Colour-batched LU-SGS changes the sweep order; the converged steady state must not move."""
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    res = []
    for scan in (None, np.arange(m.n_cells)[::-1].copy()):
        o = _oracle(oracle_lib, m, cfg)
        o.set_u(u0)
        it, rel = _run_oracle(o, u0, 100.0, 1e-8, 20000, scan)
        assert rel < 1e-8
        res.append((o.get_u(), o.eval_rhs(0.0)[1]))
    (ua, wa), (ub, wb) = res
    assert np.abs(ua - ub).max() < 1e-6 * np.abs(ua).max()
    assert np.abs(wa - wb).max() < 1e-6 * np.abs(wa).max()


# ---------------------------------------------------------------------- GPU
def _gpu(m, cfg, precision=0):
    from dnds_b200.solver import Solver

    return Solver(m, cfg, precision=precision)


def _colour_scan(s):
    col, n = s.lusgs_colours()
    assert n >= 2
    return np.argsort(col, kind="stable")


@pytest.mark.gpu
def test_colouring_is_proper():
    m = _naca_small()
    s = _gpu(m, _cfg())
    col, n = s.lusgs_colours()
    L, R = m.face_cells[:, 0], m.face_cells[:, 1]
    inner = R >= 0
    assert np.all(col[L[inner]] != col[R[inner]])
    assert col.min() == 0 and col.max() == n - 1 and n <= 6


@pytest.mark.gpu
def test_lusgs_sweeps_match_oracle(oracle_lib):
    import torch

    from dnds_b200.solver import BUF_RHS

    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    _run_oracle(o, u0, 100.0, 0.0, 30)  # a non-uniform state
    u, urec = o.get_u(), o.get_urec()
    s = _gpu(m, cfg)
    s.set_u(u)
    s.set_urec(urec)
    s.EvaluateDt(100.0, use_local_dt=True)
    rhs = s.EvaluateRHS(0.0)
    s.LUSGSMatrixInit(1e100, 1.0)
    rptr, _ = s.device_buffer(BUF_RHS)
    inc = torch.zeros((m.n_cells, 4), dtype=torch.float64, device="cuda:0")
    s.UpdateLUSGSForward(1.0, rptr, inc.data_ptr())
    fwd = inc.cpu().numpy().copy()
    s.UpdateLUSGSBackward(1.0, rptr, inc.data_ptr())
    both = inc.cpu().numpy()

    scan = _colour_scan(s)
    o.set_u(u)
    o.set_urec(urec)
    o.eval_dt(100.0, use_local_dt=True)
    o.lusgs_matrix_init(1e100, 1.0)
    ref = np.zeros((m.n_cells, 4))
    o.lusgs_forward(rhs, ref, 1.0, scan)
    assert np.abs(fwd - ref).max() < 1e-12 * np.abs(ref).max()
    o.lusgs_backward(rhs, ref, 1.0, scan)
    assert np.abs(both - ref).max() < 1e-12 * np.abs(ref).max()
    # the natural order gives a different (equally valid) increment
    nat = np.zeros((m.n_cells, 4))
    o.lusgs_forward(rhs, nat, 1.0)
    o.lusgs_backward(rhs, nat, 1.0)
    assert np.abs(nat - ref).max() > 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
def test_implicit_iterations_match_oracle(oracle_lib):
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    s = _gpu(m, cfg)
    s.set_u(u0)
    s.bdf_begin()
    scan = _colour_scan(s)
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    for it in range(20):
        res, wf = s.implicit_iteration(100.0)
        inc = o.implicit_iteration(100.0, u0, scan2cell=scan)
        assert abs(res[0] - np.abs(inc[:, 0]).sum()) < 1e-9 * res[0]
    u = s.get_u()
    ref = o.get_u()
    assert np.abs(u - ref).max() < 1e-10 * np.abs(ref).max()
    _, wref = o.eval_rhs(0.0)
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.gpu
def test_level_scheduled_natural_order_matches_sequential_oracle(oracle_lib):
    """Mode 1 runs the reference's own sequential sweep order (natural cell order) as dependency
    levels: sweeps and iterations agree with the oracle's sequential sweep to summation order."""
    import torch

    from dnds_b200.solver import BUF_RHS

    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    s = _gpu(m, cfg)
    nb = s.lusgs_set_order(1)
    assert nb >= 2 * (32 + 16)  # levels follow i + j on the structured C-mesh
    s.set_u(u0)
    s.bdf_begin()
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    for it in range(20):
        res, _ = s.implicit_iteration(100.0)
        inc = o.implicit_iteration(100.0, u0)
        assert abs(res[0] - np.abs(inc[:, 0]).sum()) < 1e-9 * res[0]
    ref = o.get_u()
    assert np.abs(s.get_u() - ref).max() < 1e-10 * np.abs(ref).max()
    # one sweep pair on the current state, against the oracle in the natural order
    s.EvaluateDt(100.0, use_local_dt=True)
    rhs = s.EvaluateRHS(0.0)
    s.LUSGSMatrixInit(1e100, 1.0)
    rptr, _ = s.device_buffer(BUF_RHS)
    inc = torch.zeros((m.n_cells, 4), dtype=torch.float64, device="cuda:0")
    s.UpdateLUSGSForward(1.0, rptr, inc.data_ptr())
    s.UpdateLUSGSBackward(1.0, rptr, inc.data_ptr())
    o.set_u(s.get_u())
    o.set_urec(s.get_urec())
    o.eval_dt(100.0, use_local_dt=True)
    o.lusgs_matrix_init(1e100, 1.0)
    nat = np.zeros((m.n_cells, 4))
    o.lusgs_forward(rhs, nat, 1.0)
    o.lusgs_backward(rhs, nat, 1.0)
    assert np.abs(inc.cpu().numpy() - nat).max() < 1e-12 * np.abs(nat).max()
    # back to colour batches
    assert s.lusgs_set_order(0) == 2 * s.lusgs_colours()[1]


@pytest.mark.gpu
def test_scan_order_beyond_the_shared_level_table_matches_oracle(oracle_lib):
    """A 2200 x 2 channel in the natural order has 2201 levels per sweep; a scan order that walks the
    channel back and forth (rows alternately forward and reversed) makes more than 4095 levels
    (the level table one block keeps in shared memory), so the sweep runs on the general
    level-by-level path.  Both agree with the oracle's sequential sweep."""
    from dnds_b200.solver import DndsgError

    m = M.structured_grid(2200, 2, 440.0, 0.4, periodic=False)
    cfg = S.preset("naca0012", eulerSetting={"riemannSolverType": "Roe", "idealGasProperty": {"gamma": 1.4},
                                             "farFieldStaticValue": S.free_stream(0.5, 2.0)})
    rng = np.random.default_rng(2)
    u0 = _free_stream(m, cfg) * (1 + 0.02 * rng.uniform(size=(m.n_cells, 1)))
    s = _gpu(m, cfg)
    with pytest.raises(DndsgError):
        s.lusgs_set_order(1, np.zeros(m.n_cells, dtype=np.int64))  # not a permutation
    assert s.lusgs_set_order(1) == 2 * 2201  # natural order: levels i + j
    order = np.concatenate([np.arange(2200), np.arange(4399, 2199, -1)])  # row 1 walked backwards
    assert s.lusgs_set_order(1, order) == 2 * 4400
    s.set_u(u0)
    s.bdf_begin()
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    for _ in range(3):
        s.implicit_iteration(20.0)
        o.implicit_iteration(20.0, u0, scan2cell=order)
    ref = o.get_u()
    assert np.abs(s.get_u() - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.gpu
def test_line_scan_order_matches_oracle(oracle_lib):
    """A caller-given scan order (wall-normal lines, even then odd) runs as nj + 1 levels per
    sweep (the odd lines follow the even ones one level behind) and computes what the oracle's
    sequential sweep in that order computes."""
    m, cfg = _naca_small(), _cfg()
    scan = M.line_scan_order(m)
    u0 = _free_stream(m, cfg)
    s = _gpu(m, cfg)
    assert s.lusgs_set_order(1, scan) == 2 * (16 + 1)
    s.set_u(u0)
    s.bdf_begin()
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    for it in range(10):
        s.implicit_iteration(100.0)
        o.implicit_iteration(100.0, u0, scan2cell=scan)
    ref = o.get_u()
    assert np.abs(s.get_u() - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.gpu
def test_wide_levels_read_records_and_increments_from_global_memory(oracle_lib):
    """The line order on a C-mesh 300 cells around makes levels of about 300 positions: a level
    holds more positions than the walk buffers records for (128; the rest are read from global
    memory), and a neighbour one level back is sometimes more than the 256 positions of the
    increment ring behind (read from global memory), sometimes not.  The sweep still computes what
    the oracle's sequential sweep in that order computes."""
    m = M.naca0012_cmesh(200, 50, 8, first=2e-3, far=10.0, wall_bc=M.BC_WALL_EULER)
    cfg = _cfg()
    scan = M.line_scan_order(m)
    u0 = _free_stream(m, cfg)
    s = _gpu(m, cfg)
    assert s.lusgs_set_order(1, scan) == 2 * (8 + 1)
    s.set_u(u0)
    s.bdf_begin()
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    for it in range(5):
        s.implicit_iteration(100.0)
        o.implicit_iteration(100.0, u0, scan2cell=scan)
    ref = o.get_u()
    assert np.abs(s.get_u() - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.gpu
def test_steady_state_matches_natural_order_oracle(oracle_lib):
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    o = _oracle(oracle_lib, m, cfg)
    o.set_u(u0)
    it_o, rel_o = _run_oracle(o, u0, 100.0, 1e-8, 20000)
    uo = o.get_u()
    _, wo = o.eval_rhs(0.0)
    s = _gpu(m, cfg)
    s.set_u(u0)
    it_g, rel_g, wg = s.steady_solve(100.0, 1e-8, 20000)
    assert rel_g[0] < 1e-8
    ug = s.get_u()
    assert np.abs(ug - uo).max() < 1e-6 * np.abs(uo).max()
    # wall force: the GPU's is from its last iteration's RHS, the oracle's from the converged state
    assert np.abs(wg - wo)[1:3].max() < 1e-6 * np.abs(wo[1:3]).max()
    # FP32-bulk reconstruction and flux: the force within 1e-4 of the FP64 one
    s32 = _gpu(m, cfg, precision=1)
    s32.set_u(u0)
    it32, rel32, w32 = s32.steady_solve(100.0, 1e-5, 20000)
    assert rel32[0] < 1e-5
    assert np.abs(w32 - wo)[1:3].max() < 1e-4 * np.abs(wo[1:3]).max()


@pytest.mark.gpu
def test_full_size_naca_iterations_reduce_the_residual():
    """The 512 x 128 C-mesh (first spacing 1e-6 chord, far field 20 chords) at M 0.15,
    alpha 10 degrees, in the reference's natural sweep order: 300 pseudo-time iterations run
    clean and lower the increment norm (in the colour order the same start grows at first)."""
    m = M.naca0012_cmesh(wall_bc=M.BC_WALL_EULER)
    cfg = S.preset("naca0012")
    s = _gpu(m, cfg)
    s.lusgs_set_order(1)
    s.set_u(_free_stream(m, cfg))
    hist = []
    it, rel, wf = s.steady_solve(100.0, 1e-12, 300, history=hist)
    h = np.array(hist)
    assert np.isfinite(h).all() and np.isfinite(wf).all()
    assert h[-1, 0] < 0.5 * h[:, 0].max()
    assert s.get_u()[:, 0].min() > 0
    flags, _ = s.status()
    assert flags == 0
