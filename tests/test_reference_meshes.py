"""The reference's own Gmsh meshes through the Gmsh 2.2 reader and the GPU path.

Fixtures (tests/golden/make_reference_meshes.py): data/mesh/Uniform128.msh (128 x 128 quads on the
unit square, "bc-3" = Wall_Euler) and data/mesh/NACA0012_WIDE_H3_NS.msh (14,280 quads around a
NACA 0012, "bc-4" = Wall_NoSlip on the airfoil, "bc-2" = Farfield), stored as the parsed file
content.  The boundary names map to BoundaryType as in DNDS_Mesh.hpp:801-829.

CPU: the fixtures equal a fresh parse of the reference's files (where the reference is present),
the meshes build with the expected counts and closed, counter-clockwise cells, and an unknown
boundary name is an error.  GPU (FP64 through the C ABI against the oracle): three VR sweeps, the
face Gauss-point states, EvaluateDt and EvaluateRHS; Uniform128 within 1e-11 (single evaluations, as
the golden tests); the NACA 0012 mesh with the laminar Navier-Stokes model and with RANS-SA within
1e-10 (faces) and 1e-9 (RHS), its wall cells of aspect ratio up to 3.7e4 amplifying rounding.
"""
import importlib.util
import os

import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _mrm():
    spec = importlib.util.spec_from_file_location("make_reference_meshes", os.path.join(GOLDEN, "make_reference_meshes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _mesh(name):
    return M.gmsh_mesh(_mrm().load_fixture(name), name)


@pytest.mark.parametrize("name", ["gmsh_uniform128", "gmsh_naca0012_wide_h3_ns"])
def test_fixture_is_the_reference_file(name):
    mod = _mrm()
    path = os.path.join(mod.reference_mesh_dir(), mod.MESHES[name])
    if not os.path.exists(path):
        pytest.skip("the reference checkout is not on this machine")
    g, f = M.parse_gmsh2(path), mod.load_fixture(name)
    assert np.array_equal(g["nodes"], f["nodes"])
    assert np.array_equal(g["cells"], f["cells"]) and np.array_equal(g["bnd"], f["bnd"])
    assert g["names"] == f["names"]


def test_reference_meshes_build():
    u = _mesh("gmsh_uniform128")
    assert (u.n_cells, u.n_faces) == (16384, 33024)
    assert np.sum(u.face_bc == M.BC_WALL_EULER) == 512 and np.sum(u.face_bc == M.BC_INNER) == 32512
    n = _mesh("gmsh_naca0012_wide_h3_ns")
    assert (n.n_cells, n.n_faces) == (14280, 28728)
    assert np.sum(n.face_bc == M.BC_WALL_NOSLIP) == 168 and np.sum(n.face_bc == M.BC_FARFIELD) == 168
    for m in (u, n):
        # counter-clockwise cells, and every cell closed: the sum of its outward face normals vanishes
        xy = m.node_xy[m.cell_nodes[:, :4].clip(0)]
        a = 0.5 * np.sum(xy[:, :, 0] * np.roll(xy[:, :, 1], -1, 1) - np.roll(xy[:, :, 0], -1, 1) * xy[:, :, 1], 1)
        assert (a > 0).all()
        d = m.node_xy[m.face_nodes[:, 1]] - m.node_xy[m.face_nodes[:, 0]]
        nrm = np.stack([d[:, 1], -d[:, 0]], 1)
        clo = np.zeros((m.n_cells, 2))
        np.add.at(clo, m.face_cells[:, 0], nrm)
        inner = m.face_cells[:, 1] >= 0
        np.add.at(clo, m.face_cells[inner, 1], -nrm[inner])
        assert np.abs(clo).max() < 1e-12 * np.abs(nrm).max()


def test_unknown_boundary_name_is_an_error():
    g = _mrm().load_fixture("gmsh_uniform128")
    g["names"] = {k: ("bc-unknown" if v == "bc-3" else v) for k, v in g["names"].items()}
    with pytest.raises(ValueError, match="not a DNDS boundary name"):
        M.gmsh_mesh(g)


def _smooth_uniform(m):
    from dnds_b200 import geometry as G

    return G.cell_average(m, lambda x, y: np.stack(
        [1 + 0.2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y), 0.3 + 0.1 * np.cos(2 * np.pi * y),
         -0.2 + 0.1 * np.sin(2 * np.pi * x), 2.5 + 0.1 * np.cos(2 * np.pi * x)], -1))


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _compare(oracle_lib, m, cfg, u0, t=0.0, cfl=0.5, faces=True, tol_faces=1e-11, tol_dt=1e-13, tol_rhs=1e-11):
    from dnds_b200.solver import Solver

    o = oracle_lib.Oracle(m, cfg, n_threads=0)
    o.set_u(u0)
    o.vr_step(3)
    s = Solver(m, cfg, precision=0)
    s.set_u(u0)
    s.ReconstructionJacobiStep(3)
    if faces:
        assert _rel(s.face_values(t), o.face_values(t)) < tol_faces
    dt_o, dmin_o = o.eval_dt(cfl, 1e100, True)
    dmin_s = s.EvaluateDt(cfl, 1e100, True)
    assert abs(dmin_s - dmin_o) < tol_dt * dmin_o
    assert _rel(s.get_dt(), dt_o) < 1e-12
    rhs_o, _ = o.eval_rhs(t)
    rhs_s = s.EvaluateRHS(t)
    assert _rel(rhs_s, rhs_o) < tol_rhs
    flags, _ = s.status()
    assert flags == 0
    s.close()


@pytest.mark.gpu
def test_uniform128_euler_walls_against_oracle(oracle_lib):
    m = _mesh("gmsh_uniform128")
    _compare(oracle_lib, m, S.preset("vortex"), _smooth_uniform(m))


@pytest.mark.gpu
def test_naca0012_wide_h3_laminar_against_oracle(oracle_lib):
    m = _mesh("gmsh_naca0012_wide_h3_ns")
    cfg = S.preset("naca0012_laminar")
    far = np.array(cfg["eulerSetting"]["farFieldStaticValue"])
    x = m.node_xy[m.cell_nodes[:, :4].clip(0)].mean(1)
    pert = 1 + 0.05 * np.exp(-((x[:, 0] - 0.5) ** 2 + x[:, 1] ** 2))
    u0 = far[None, :] * pert[:, None]
    # boundary-layer cells of aspect ratio up to 3.7e4 under a flow started impulsively at a no-slip
    # wall: the VR systems' conditioning lifts the rounding difference of the two implementations
    # (Cholesky against Gauss-Jordan) to 2e-11 in the face states, and the viscous terms of the
    # thinnest cells at the trailing edge (right-hand sides of 3e7) to 1.4e-10 in the RHS (measured);
    # dt through the viscous spectral radius 3e-13
    _compare(oracle_lib, m, cfg, u0, cfl=5.0, tol_faces=1e-10, tol_dt=1e-12, tol_rhs=1e-9)


@pytest.mark.gpu
def test_naca0012_wide_h3_sa_against_oracle(oracle_lib):
    m = _mesh("gmsh_naca0012_wide_h3_ns")
    cfg = S.preset("naca0012_sa")
    far = np.array(cfg["eulerSetting"]["farFieldStaticValue"])
    x = m.node_xy[m.cell_nodes[:, :4].clip(0)].mean(1)
    pert = 1 + 0.05 * np.exp(-((x[:, 0] - 0.5) ** 2 + x[:, 1] ** 2))
    u0 = far[None, :] * pert[:, None]
    # as the laminar case; dt also goes through the SA eddy viscosity (pow / exp of two math
    # libraries): 4e-13 measured
    _compare(oracle_lib, m, cfg, u0, cfl=5.0, faces=False, tol_dt=1e-12, tol_rhs=1e-9)
