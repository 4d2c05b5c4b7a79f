"""CPU tests of the FP64 oracle: pinned against the reference's known answers
and the properties its algorithms guarantee, and against the committed
golden fixtures (which the GPU parity tests also use)."""
import os

import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_roe_flux_known_answer(oracle_lib):
    # test/testGas.cpp:22-27,68: Roe flux of UL=(1,0.5916,0,0,2.675), UR=(1,0,0,0,2.5), gamma 1.4
    f = oracle_lib.riemann_flux(1, [1.0, 0.5916, 0.0, 2.675], [1.0, 0.0, 0.0, 2.5], 1.4, 0.0)
    ref = np.array([0.369291683630373, 1.54891136111009, 0.0, 1.45489148963839])
    np.testing.assert_allclose(f, ref, rtol=0, atol=5e-14)


def test_hllc_consistency(oracle_lib):
    # F(U, U) = physical flux for both Riemann solvers
    U = np.array([1.3, 0.4, -0.2, 3.1])
    p = 0.4 * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0])
    phys = np.array([U[1], U[1] ** 2 / U[0] + p, U[1] * U[2] / U[0], (U[3] + p) * U[1] / U[0]])
    for kind in (1, 2):
        np.testing.assert_allclose(oracle_lib.riemann_flux(kind, U, U), phys, rtol=1e-14, atol=1e-14)


def _single_cell_mesh(xy):
    n = len(xy)
    fn = np.array([[k, (k + 1) % n] for k in range(n)], dtype=np.int32)
    cn = np.full((1, 4), -1, dtype=np.int32)
    cn[0, :n] = np.arange(n)
    return M.Mesh(np.array(xy, dtype=np.float64), cn, fn, np.array([[0, -1]] * n, dtype=np.int32),
                  np.full(n, M.BC_FARFIELD, dtype=np.int32), np.zeros((n, 2)))


def test_element_volumes(oracle_lib):
    # test/elemtest.cpp: Tri3 equilateral triangle, Quad4 on the unit circle
    tri = _single_cell_mesh([[0, 0], [1, 0], [0.5, np.sqrt(3) * 0.5]])
    q = [[np.cos(np.pi * k / 2), np.sin(np.pi * k / 2)] for k in range(4)]
    quad = _single_cell_mesh(q)
    cfg = S.preset("vortex", vfvSetting={"farWeight": 1.0})  # a lone cell needs the far-field value term
    for m, v in ((tri, np.sqrt(3) / 4), (quad, 2.0)):
        o = oracle_lib.Oracle(m, cfg, n_threads=1)
        vol, bary, area = o.geometry()
        assert abs(vol[0] - v) < 1e-14


def _quadratic(x, y):
    a = 1 + 0.3 * x - 0.2 * y + 0.05 * x * x + 0.07 * x * y - 0.04 * y * y
    return np.stack([a, 0.5 * a, -0.3 * a, 10 + a], -1)


@pytest.mark.parametrize("tri", [False, True])
@pytest.mark.parametrize("preset", ["vortex", "riemann"])
def test_vr_reproduces_quadratics(oracle_lib, tri, preset):
    """The VR functional vanishes on a common quadratic, so converged Jacobi
    sweeps reproduce cell averages of any quadratic exactly."""
    m = M.structured_grid(12, 10, 3.0, 2.0, triangles=tri, jitter=0.2, periodic=False, bc=M.BC_FARFIELD)
    o = oracle_lib.Oracle(m, S.preset(preset), n_threads=2)
    o.set_u(G.cell_average(m, _quadratic))
    for _ in range(3000):
        inc = o.vr_step(1)
        if inc < 1e-30:
            break
    fv = o.face_values()
    L3 = np.array([-np.sqrt(0.6), 0, np.sqrt(0.6)])
    a = m.node_xy[m.face_nodes[:, 0]]
    b = m.node_xy[m.face_nodes[:, 1]]
    gp = a[:, None, :] * (1 - L3[None, :, None]) / 2 + b[:, None, :] * (1 + L3[None, :, None]) / 2
    ex = _quadratic(gp[..., 0], gp[..., 1])
    inner = m.face_cells[:, 1] >= 0
    assert np.abs(fv[:, :, 0, :] - ex).max() < 1e-11
    assert np.abs(fv[inner][:, :, 1, :] - ex[inner]).max() < 1e-11


def test_vr_convergence_order(oracle_lib):
    """Static reconstruction (test/staticReconstructionTest.cpp:38-55) of
    (1-cos 2pi x)(1-cos 2pi y) on periodic meshes: third order in the point values."""

    def f(x, y):
        v = (1 - np.cos(2 * np.pi * x)) * (1 - np.cos(2 * np.pi * y))
        return np.stack([2 + v, v, v, 5 + v], -1)

    errs = []
    for n in (8, 16, 32):
        m = M.structured_grid(n, n, 1.0, 1.0, triangles=True, jitter=0.1, periodic=True)
        o = oracle_lib.Oracle(m, S.preset("vortex"), n_threads=4)
        o.set_u(G.cell_average(m, f))
        for _ in range(4000):
            if o.vr_step(1) < 1e-28:
                break
        fv = o.face_values()
        L3 = np.array([-np.sqrt(0.6), 0, np.sqrt(0.6)])
        a = m.node_xy[m.face_nodes[:, 0]]
        b = m.node_xy[m.face_nodes[:, 1]]
        gp = a[:, None, :] * (1 - L3[None, :, None]) / 2 + b[:, None, :] * (1 + L3[None, :, None]) / 2
        ex = f(gp[..., 0], gp[..., 1])
        errs.append(np.sqrt(np.mean((fv[:, :, 0, 0] - ex[..., 0]) ** 2)))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > 2.7, (errs, rates)


def test_freestream_and_conservation(oracle_lib):
    m = M.vortex_mesh(12, True, jitter=0.2)
    o = oracle_lib.Oracle(m, S.preset("vortex"), n_threads=2)
    o.set_u(np.tile([1.0, 1.0, 1.0, 3.5], (m.n_cells, 1)))
    o.vr_step(2)
    o.eval_dt(0.5)
    rhs, _ = o.eval_rhs()
    assert np.abs(rhs).max() < 1e-12
    o.set_u(G.isentropic_vortex(m))
    o.vr_step(2)
    o.eval_dt(0.5)
    rhs, _ = o.eval_rhs()
    vol, _, _ = o.geometry()
    total = (rhs * vol[:, None]).sum(0)
    assert np.abs(total).max() < 1e-12 * np.abs(rhs * vol[:, None]).sum()


@pytest.mark.parametrize("name", ["vortex_quad10", "vortex_tri8_jitter", "riemann_tri8", "eulerwall_quad6x5",
                                  "farfield_tri6x5", "riemann_tri16_limiter"])
def test_oracle_matches_golden(oracle_lib, name):
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    d = mg.make_case(name)
    keys = ("indicator", "face_values_lim", "face_values_limall", "u_rk2") if "limiter" in name else \
        ("face_values", "dt", "rhs", "u_rk2")
    for k in keys:
        sc = max(np.abs(ref[k]).max(), 1e-300)
        assert np.abs(d[k] - ref[k]).max() <= 1e-12 * sc, k
