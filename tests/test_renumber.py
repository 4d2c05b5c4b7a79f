"""METIS-free renumbering for locality (mesh.renumber, mesh.hilbert_order): cells along a Hilbert curve
through their centroids, faces by their lower cell.  The discretisation does not depend on the
numbering (every cell keeps its nodes and element-local face order, every face its geometry), so the
results on a renumbered mesh are those of the original, permuted: checked on the oracle (CPU) and on
the GPU path, FP64 and FP32 bulk.
"""
import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S


def _locality(m):
    L, R = m.face_cells[:, 0], m.face_cells[:, 1]
    inner = R >= 0
    return np.abs(L[inner] - R[inner]).mean() / m.n_cells


def _shuffled(n=32, seed=7):
    m = M.vortex_mesh(n, True, jitter=0.2, seed=1234)
    return m, M.renumber(m, np.random.default_rng(seed).permutation(m.n_cells))


def test_hilbert_order_steps_between_neighbours():
    k = 5
    xs, ys = np.meshgrid(np.arange(1 << k), np.arange(1 << k), indexing="ij")
    pts = np.stack([xs.ravel(), ys.ravel()], 1).astype(float)
    o = M.hilbert_order(pts, bits=k)
    assert np.array_equal(np.sort(o), np.arange(len(pts)))
    steps = np.abs(np.diff(pts[o], axis=0)).sum(1)
    assert steps.min() == 1 and steps.max() == 1  # every step of the curve goes to a neighbouring point


def test_renumber_keeps_the_mesh_and_restores_locality():
    m, (ms, sh) = _shuffled(64)
    mh, order = M.renumber(ms)
    for mm, o in ((ms, sh), (mh, order)):
        assert mm.n_cells == m.n_cells and mm.n_faces == m.n_faces
    # the same cells (node lists) and the same faces (nodes, boundary type, shift), renumbered
    assert np.array_equal(mh.cell_nodes, ms.cell_nodes[order])
    key = lambda mm: sorted(map(tuple, np.concatenate([mm.face_nodes, mm.face_bc[:, None], mm.face_shift], 1)))
    assert key(mh) == key(m)
    # adjacency: face (L, R) of the original maps to (new L, new R) of the renumbered mesh
    new_of_old = np.empty(m.n_cells, dtype=np.int64)
    new_of_old[sh[order]] = np.arange(m.n_cells)
    pairs = lambda mm, f: set(map(tuple, np.sort(f(mm.face_cells[mm.face_cells[:, 1] >= 0]), 1)))
    assert pairs(m, lambda fc: new_of_old[fc]) == pairs(mh, lambda fc: fc)
    assert _locality(ms) > 0.3 and _locality(mh) < 0.05
    with pytest.raises(ValueError, match="permutation"):
        M.renumber(m, np.zeros(m.n_cells, dtype=np.int64))


def test_oracle_results_are_permuted_by_the_renumbering(oracle_lib):
    m, (ms, sh) = _shuffled(16)
    mh, order = M.renumber(ms)
    perm = sh[order]  # new cell k of mh is cell perm[k] of m
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    out = []
    for mm, u in ((m, u0), (mh, u0[perm])):
        o = oracle_lib.Oracle(mm, cfg, n_threads=1)
        o.set_u(u)
        o.vr_step(3)
        _, dmin = o.eval_dt(0.5)
        rhs, _ = o.eval_rhs(0.0)
        out.append((dmin, rhs))
    assert out[1][0] == out[0][0]
    assert np.abs(out[1][1] - out[0][1][perm]).max() <= 1e-13 * np.abs(out[0][1]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_results_are_permuted_by_the_renumbering(precision):
    from dnds_b200.solver import Solver

    m, (ms, sh) = _shuffled(32)
    mh, order = M.renumber(ms)
    perm = sh[order]
    cfg = S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    res = []
    for mm, u in ((m, u0), (mh, u0[perm])):
        s = Solver(mm, cfg, precision=precision)
        s.set_u(u)
        s.ReconstructionJacobiStep(3)
        dmin = s.EvaluateDt(0.5)
        rhs = s.EvaluateRHS(0.0)
        s.set_u(u)
        s.set_urec(np.zeros((mm.n_cells, 5, 4)))
        s.time = 0.0
        for _ in range(2):
            s.ssprk3_step(0.5)
        res.append((dmin, rhs, s.get_u()))
        s.close()
    (d0, r0, u0s), (d1, r1, u1s) = res
    assert d1 == d0
    assert np.abs(r1 - r0[perm]).max() <= 1e-13 * np.abs(r0).max()
    assert np.abs(u1s - u0s[perm]).max() <= 1e-14 * np.abs(u0s).max()
