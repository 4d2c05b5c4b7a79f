"""Edge cases of the mesh and setup paths: ragged (mixed triangle / quadrilateral) cells, the
smallest meshes, rejected inputs, and the largest workload of the explicit configs.

Tolerances as in test_gpu_parity.py: FP64 GPU vs FP64 oracle 1e-11 relative, FP32 bulk 2e-5.
"""
import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S


def _mixed_mesh(n=8, seed=3):
    """[0,1]^2, n x n nodes jittered; the left half quadrilaterals, the right half split into
    triangles, far field all round: cells with 3 and 4 faces side by side (ragged face slots)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    xs, ys = np.meshgrid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1), indexing="ij")
    xy = np.stack([xs.ravel(), ys.ravel()], 1)
    inner = (xy[:, 0] > 0) & (xy[:, 0] < 1) & (xy[:, 1] > 0) & (xy[:, 1] < 1)
    xy[inner] += rng.uniform(-0.2 * h, 0.2 * h, (inner.sum(), 2))
    nid = lambda i, j: i * (n + 1) + j
    cells = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if i < n // 2:
                cells.append([a, b, c, d])
            else:
                cells.append([a, b, c, -1])
                cells.append([a, c, d, -1])
    cells = np.array(cells)
    faces = M.faces_from_cells(xy, cells, lambda a, b: M.BC_FARFIELD)
    return M._as_mesh(xy, cells, faces, "mixed", {})


def _cfg():
    return S.preset("naca0012", eulerSetting={"riemannSolverType": "Roe", "idealGasProperty": {"gamma": 1.4},
                                              "farFieldStaticValue": S.free_stream(0.4, 20.0)})


def _state(m, seed=5):
    rng = np.random.default_rng(seed)
    x = m.node_xy[np.where(m.cell_nodes >= 0, m.cell_nodes, m.cell_nodes[:, :1])].mean(1)
    rho = 1.0 + 0.2 * np.sin(4 * x[:, 0]) * np.cos(3 * x[:, 1])
    u = 0.3 + 0.1 * np.cos(5 * x[:, 1])
    v = -0.2 + 0.1 * np.sin(4 * x[:, 0])
    p = 1.0 + 0.1 * rng.uniform(size=len(x))
    return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], 1)


# ---------------------------------------------------------------------- CPU
def test_faces_from_cells_mixed_and_rejects_misoriented():
    m = _mixed_mesh()
    nf = np.where(m.cell_nodes[:, 3] < 0, 3, 4)
    assert set(np.unique(nf)) == {3, 4}
    assert (m.face_bc == M.BC_FARFIELD).sum() == 4 * 8
    bad = m.cell_nodes.copy()
    bad[0, [1, 3]] = bad[0, [3, 1]]  # clockwise
    with pytest.raises(AssertionError):
        M.faces_from_cells(m.node_xy, bad, lambda a, b: M.BC_FARFIELD)


# ---------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 2e-5)])
def test_mixed_cells_match_oracle(oracle_lib, precision, tol):
    from dnds_b200.solver import Solver

    m, cfg = _mixed_mesh(), _cfg()
    u = _state(m)
    s = Solver(m, cfg, precision=precision)
    s.set_u(u)
    s.ReconstructionJacobiStep(3)
    o = oracle_lib.Oracle(m, cfg, n_threads=2)
    o.set_u(u)
    o.vr_step(3)
    fv, ref = s.face_values(0.0), o.face_values(0.0)
    assert np.abs(fv - ref).max() < tol * np.abs(ref).max()
    s.EvaluateDt(0.5)
    o.eval_dt(0.5)
    rhs, (rref, _) = s.EvaluateRHS(0.0), o.eval_rhs(0.0)
    assert np.abs(rhs - rref).max() < tol * np.abs(rref).max()


@pytest.mark.gpu
def test_single_cell_mesh(oracle_lib):
    """One quadrilateral with four far-field faces: a VR with no neighbours and no interior face."""
    from dnds_b200.solver import Solver

    xy = np.array([[0.0, 0.0], [1.0, 0.1], [1.1, 1.0], [0.0, 0.9]])
    cells = np.array([[0, 1, 2, 3]])
    m = M._as_mesh(xy, cells, M.faces_from_cells(xy, cells, lambda a, b: M.BC_FARFIELD), "one", {})
    cfg = _cfg()
    u = np.array([[1.1, 0.3, 0.1, 2.9]])
    s = Solver(m, cfg, precision=0)
    s.set_u(u)
    s.ReconstructionJacobiStep(2)
    s.EvaluateDt(0.5)
    rhs = s.EvaluateRHS(0.0)
    o = oracle_lib.Oracle(m, cfg, n_threads=1)
    o.set_u(u)
    o.vr_step(2)
    o.eval_dt(0.5)
    ref, _ = o.eval_rhs(0.0)
    assert np.abs(rhs - ref).max() < 1e-11 * np.abs(ref).max()


@pytest.mark.gpu
def test_clockwise_cell_is_rejected():
    from dnds_b200.solver import DndsgError, Solver

    m = _mixed_mesh()
    flipped = m.cell_nodes.copy()
    flipped[0, [1, 3]] = flipped[0, [3, 1]]
    bad = M.Mesh(m.node_xy, flipped, m.face_nodes, m.face_cells, m.face_bc, m.face_shift)
    with pytest.raises(DndsgError):
        Solver(bad, _cfg(), precision=0)


@pytest.mark.gpu
def test_largest_explicit_workload_runs_clean():
    """The four-quadrant Riemann problem at its configured size: 2048 x 2048 x 2 = 8,388,608
    jittered triangles, CWBAP limiter, HLLC, FP32 bulk.  Two SSP-RK3 steps: positive density and
    pressure everywhere, no kernel flags."""
    from dnds_b200.solver import Solver

    m = M.riemann_mesh(2048)
    assert m.n_cells == 8_388_608
    s = Solver(m, S.preset("riemann"), precision=1)
    s.set_u(G.quadrant_states(m, S.RIEMANN_2D_STATES))
    for _ in range(2):
        s.ssprk3_step(0.4, 0.3)
    u = s.get_u()
    p = 0.4 * (u[:, 3] - 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2) / u[:, 0])
    assert np.isfinite(u).all() and u[:, 0].min() > 0 and p.min() > 0
    flags, _ = s.status()
    assert flags == 0
