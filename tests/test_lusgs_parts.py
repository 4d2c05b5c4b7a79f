"""Partitioned LU-SGS sweeps: the scan-order sweep as the reference runs it on several MPI ranks.

On a rank, UpdateLUSGSForward / Backward (DNDS_FV_EulerEvaluator.cpp:1149-1357) loop over the rank's
own cells in its scan order; a neighbour on another rank is a ghost whose scan position counts as
after every local cell (iScanOther = iScan + 1, :1177-1181 and :1313-1317).  So a ghost never enters
the forward sweep, and enters the backward sweep with the increment pulled between the two sweeps
(the other rank's forward result).  The oracle restates that with a part index per cell
(Oracle.set_lusgs_parts); dndsg_lusgs_set_parts runs it on the GPU with one level walk per part.

CPU: one part is the unpartitioned sweep, bit for bit; the partitioned forward sweep on the whole
mesh equals each part's own forward sweep on its local mesh (owned cells, then the ghost layer, as
partition_mesh builds it for a multi-rank run).  GPU: sweeps and pseudo-time iterations against the
partitioned oracle (FP64, to summation order: 1e-12 for a sweep pair, 1e-10 after iterations), in
the natural order and in a caller-given scan order, Euler and RANS-SA.
"""
import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S
from dnds_b200.partition import block_owner, partition_mesh


def _naca_small():
    return M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0, wall_bc=M.BC_WALL_EULER)


def _cfg():
    return S.preset("naca0012", eulerSetting={"riemannSolverType": "Roe", "idealGasProperty": {"gamma": 1.4},
                                              "farFieldStaticValue": S.free_stream(0.5, 2.0)})


def _free_stream(m, cfg):
    return np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _developed(oracle_lib, m, cfg, iters=30):
    """A non-uniform state: iterations of the unpartitioned oracle from the free stream."""
    u0 = _free_stream(m, cfg)
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_u(u0)
    for _ in range(iters):
        o.implicit_iteration(100.0, u0)
    return o.get_u(), o.get_urec()


# ---------------------------------------------------------------------- CPU
def test_block_owner_is_contiguous_and_balanced():
    p = block_owner(1000, 7)
    assert p.dtype == np.int32 and p[0] == 0 and p[-1] == 6
    assert (np.diff(p) >= 0).all()
    n = np.bincount(p)
    assert n.max() - n.min() <= 1


def test_oracle_one_part_is_the_unpartitioned_sweep(oracle_lib):
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    a = oracle_lib.Oracle(m, cfg, n_threads=1)
    b = oracle_lib.Oracle(m, cfg, n_threads=1)
    b.set_lusgs_parts(np.zeros(m.n_cells, dtype=np.int32))
    for o in (a, b):
        o.set_u(u0)
        for _ in range(3):
            o.implicit_iteration(100.0, u0)
    assert np.array_equal(a.get_u(), b.get_u())


def test_oracle_partitioned_forward_is_each_part_on_its_own_mesh(oracle_lib):
    """Each part's local mesh lists its owned cells in global order followed by the ghosts, so in the
    local natural order every ghost comes after every owned cell: the unpartitioned sweep on that
    mesh is what the reference's rank computes.  Its forward increments of the owned cells equal the
    partitioned forward sweep on the whole mesh."""
    m, cfg = _naca_small(), _cfg()
    u, urec = _developed(oracle_lib, m, cfg)
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((m.n_cells, 4))
    nparts = 3
    o = oracle_lib.Oracle(m, cfg, n_threads=1)
    o.set_lusgs_parts(block_owner(m.n_cells, nparts))
    o.set_u(u)
    o.set_urec(urec)
    o.eval_dt(100.0, use_local_dt=True)
    o.lusgs_matrix_init(1e100, 1.0)
    whole = np.zeros((m.n_cells, 4))
    o.lusgs_forward(rhs, whole, 1.0)
    for part in partition_mesh(m, nparts):
        q = oracle_lib.Oracle(part.mesh, cfg, n_threads=1)
        q.set_u(u[part.cells])
        q.set_urec(urec[part.cells])
        q.eval_dt(100.0, use_local_dt=True)
        q.lusgs_matrix_init(1e100, 1.0)
        loc = np.zeros((len(part.cells), 4))
        q.lusgs_forward(rhs[part.cells], loc, 1.0)
        own = part.cells[:part.n_owned]
        assert _rel(loc[:part.n_owned], whole[own]) < 1e-14


def test_oracle_partitioned_backward_differs_from_the_unpartitioned_one(oracle_lib):
    """The parts decouple: a partitioned sweep pair is a different (block-Jacobi across parts)
    approximation of the same system, not the sequential sweep."""
    m, cfg = _naca_small(), _cfg()
    u, urec = _developed(oracle_lib, m, cfg)
    rhs = np.random.default_rng(6).standard_normal((m.n_cells, 4))
    out = []
    for parts in (None, block_owner(m.n_cells, 4)):
        o = oracle_lib.Oracle(m, cfg, n_threads=1)
        o.set_lusgs_parts(parts)
        o.set_u(u)
        o.set_urec(urec)
        o.eval_dt(100.0, use_local_dt=True)
        o.lusgs_matrix_init(1e100, 1.0)
        inc = np.zeros((m.n_cells, 4))
        o.lusgs_forward(rhs, inc, 1.0)
        o.lusgs_backward(rhs, inc, 1.0)
        out.append(inc)
    assert np.isfinite(out[1]).all()
    assert _rel(out[1], out[0]) > 1e-6


# ---------------------------------------------------------------------- GPU
def _gpu(m, cfg):
    from dnds_b200.solver import Solver

    return Solver(m, cfg, precision=0)


@pytest.mark.gpu
@pytest.mark.parametrize("nparts,scan", [(4, None), (3, "lines"), (64, None)])
def test_partitioned_sweep_pair_matches_oracle(oracle_lib, nparts, scan):
    import torch

    from dnds_b200.solver import BUF_RHS

    m, cfg = _naca_small(), _cfg()
    u, urec = _developed(oracle_lib, m, cfg)
    order = M.line_scan_order(m) if scan == "lines" else None
    parts = block_owner(m.n_cells, nparts)
    s = _gpu(m, cfg)
    full = s.lusgs_set_order(1, order)
    nb = s.lusgs_set_parts(parts, nparts)
    assert nb < full or scan == "lines"
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
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_lusgs_parts(parts)
    o.set_u(u)
    o.set_urec(urec)
    o.eval_dt(100.0, use_local_dt=True)
    o.lusgs_matrix_init(1e100, 1.0)
    ref = np.zeros((m.n_cells, 4))
    o.lusgs_forward(rhs, ref, 1.0, order)
    assert _rel(fwd, ref) < 1e-12
    o.lusgs_backward(rhs, ref, 1.0, order)
    assert _rel(both, ref) < 1e-12
    flags, _ = s.status()
    assert flags == 0
    s.close()


@pytest.mark.gpu
def test_partitioned_iterations_match_oracle(oracle_lib):
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg)
    parts = block_owner(m.n_cells, 4)
    s = _gpu(m, cfg)
    # 64 x 16 cells: natural-order levels i + j (79 per sweep); 4 parts of 16 columns: 31 per sweep
    assert s.lusgs_set_order(1) == 2 * 79
    assert s.lusgs_set_parts(parts, 4) == 2 * 31
    s.set_u(u0)
    s.bdf_begin()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_lusgs_parts(parts)
    o.set_u(u0)
    for _ in range(20):
        res, _ = s.implicit_iteration(100.0)
        inc = o.implicit_iteration(100.0, u0)
        assert abs(res[0] - np.abs(inc[:, 0]).sum()) < 1e-9 * res[0]
    assert _rel(s.get_u(), o.get_u()) < 1e-10
    # back to one part: the natural-order schedule again
    assert s.lusgs_set_parts(None) == 2 * 79
    s.close()


@pytest.mark.gpu
def test_partitioned_sa_iterations_match_oracle(oracle_lib):
    m = M.naca0012_cmesh(32, 16, 16, first=1e-3, far=10.0)
    cfg = S.naca0012_sa(0.15, 10.0, 1e5)
    u0 = _free_stream(m, cfg)
    parts = block_owner(m.n_cells, 4)
    s = _gpu(m, cfg)
    s.lusgs_set_order(1)
    s.lusgs_set_parts(parts, 4)
    s.set_u(u0)
    s.bdf_begin()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_lusgs_parts(parts)
    o.set_u(u0)
    for _ in range(20):
        res, _ = s.implicit_iteration(20.0)
        inc = o.implicit_iteration(20.0, u0)
        assert abs(res[4] - np.abs(inc[:, 4]).sum()) < 1e-8 * max(res[4], 1e-300)
    assert _rel(s.get_u(), o.get_u()) < 1e-9
    flags, _ = s.status()
    assert flags == 0
    s.close()


@pytest.mark.gpu
def test_bad_parts_are_refused_and_change_nothing():
    from dnds_b200.solver import DndsgError

    m, cfg = _naca_small(), _cfg()
    s = _gpu(m, cfg)
    nb = s.lusgs_set_order(1)
    bad = block_owner(m.n_cells, 4)
    bad[7] = 4
    with pytest.raises(DndsgError, match="out of range"):
        s.lusgs_set_parts(bad, 4)
    assert s.lusgs_set_order(1) == nb
    s.close()


@pytest.mark.gpu
def test_partitioned_sweeps_on_mixed_cells_match_oracle(oracle_lib):
    """Ragged face slots (quadrilaterals and triangles side by side, far field all round) in 3 parts."""
    import importlib.util
    import os

    spec = importlib.util.spec_from_file_location(
        "edge_cases", os.path.join(os.path.dirname(os.path.abspath(__file__)), "test_edge_cases.py"))
    ec = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ec)
    m = ec._mixed_mesh(12)
    cfg = _cfg()
    far = np.array(cfg["eulerSetting"]["farFieldStaticValue"])
    x = m.node_xy[m.cell_nodes.clip(0)].mean(1)
    u0 = far[None, :] * (1 + 0.05 * np.sin(6.0 * x[:, :1]) * np.cos(5.0 * x[:, 1:]))
    parts = block_owner(m.n_cells, 3)
    s = _gpu(m, cfg)
    s.lusgs_set_order(1)
    s.lusgs_set_parts(parts, 3)
    s.set_u(u0)
    s.bdf_begin()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_lusgs_parts(parts)
    o.set_u(u0)
    for _ in range(10):
        res, _ = s.implicit_iteration(50.0)
        inc = o.implicit_iteration(50.0, u0)
        assert abs(res[0] - np.abs(inc[:, 0]).sum()) < 1e-9 * res[0]
    assert _rel(s.get_u(), o.get_u()) < 1e-10
    s.close()


@pytest.mark.gpu
def test_an_empty_part_is_walked_as_nothing(oracle_lib):
    """Parts 0 and 2 of 3 (part 1 holds no cell): its block has no level and returns at once."""
    m, cfg = _naca_small(), _cfg()
    u0 = _free_stream(m, cfg) * (1 + 0.01 * np.sin(np.arange(m.n_cells))[:, None])
    parts = 2 * block_owner(m.n_cells, 2)
    s = _gpu(m, cfg)
    s.lusgs_set_order(1)
    s.lusgs_set_parts(parts, 3)
    s.set_u(u0)
    s.bdf_begin()
    o = oracle_lib.Oracle(m, cfg, n_threads=4)
    o.set_lusgs_parts(parts)
    o.set_u(u0)
    for _ in range(5):
        s.implicit_iteration(100.0)
        o.implicit_iteration(100.0, u0)
    assert _rel(s.get_u(), o.get_u()) < 1e-10
    flags, _ = s.status()
    assert flags == 0
    s.close()
