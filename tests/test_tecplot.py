"""Tecplot binary output (PrintSerialPartPltBinaryDataArray, DNDS_Mesh.hpp:1639-1817, and the
quantities of EulerSolver::PrintData, DNDS_FV_EulerSolver.hpp:1436-1492): the file layout read back
field by field, triangles as degenerate quadrilaterals, and the derived quantities."""
import struct

import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S
from dnds_b200 import tecplot as P


def test_plt_round_trip_and_layout(tmp_path):
    m = M.vortex_mesh(4, True, jitter=0.1)
    data = np.random.default_rng(1).standard_normal((2, m.n_cells))
    f = tmp_path / "a.plt"
    P.write_plt(str(f), m.node_xy, m.cell_nodes, ["A", "B"], data, t=0.25)
    raw = f.read_bytes()
    assert raw[:8] == b"#!TDV112" and struct.unpack_from("<ii", raw, 8) == (1, 0)
    r = P.read_plt(str(f))
    assert r["names"] == ["X", "Y", "Z", "A", "B", "iPart"] and r["t"] == 0.25
    assert np.array_equal(r["xyz"][:, :2], m.node_xy) and not r["xyz"][:, 2].any()
    assert np.array_equal(r["data"]["A"], data[0]) and np.array_equal(r["data"]["B"], data[1])
    assert not r["data"]["iPart"].any()
    tri = m.cell_nodes[:, 3] < 0
    assert tri.all() and np.array_equal(r["conn"][:, :3], m.cell_nodes[:, :3])
    assert np.array_equal(r["conn"][:, 3], m.cell_nodes[:, 2])  # last node repeated
    # size: header + 3 node arrays + (2 data + iPart) cell arrays + 4 ints per cell
    assert len(raw) > 8 * (3 * len(m.node_xy) + 3 * m.n_cells) + 16 * m.n_cells


def test_print_data_quantities(tmp_path):
    m = M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0)
    cfg = S.preset("naca0012_sa")
    rng = np.random.default_rng(2)
    u = np.tile(np.array(cfg["eulerSetting"]["farFieldStaticValue"]), (m.n_cells, 1))
    u[:, 0] *= 1 + 0.1 * rng.uniform(size=m.n_cells)
    rhs = rng.standard_normal((m.n_cells, 5))
    f = tmp_path / "sa.plt"
    P.print_data(str(f), m, u, cfg, rhs=rhs)
    r = P.read_plt(str(f))
    assert r["names"][3:] == ["R", "U", "V", "W", "P", "T", "M", "ifUseLimiter", "RHSr", "iPart"]
    d = r["data"]
    rho = u[:, 0]
    p = 0.4 * (u[:, 3] - 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2) / rho)
    assert np.allclose(d["R"], rho) and np.allclose(d["U"], u[:, 1] / rho)
    assert np.allclose(d["W"], p)  # the reference's 2-D labels: pressure under "W"
    assert np.allclose(d["P"], p / rho)  # temperature with Rgas 1 under "P"
    assert np.allclose(d["T"], np.sqrt((u[:, 1] ** 2 + u[:, 2] ** 2) / rho ** 2 / (1.4 * p / rho)))  # Mach
    assert not d["M"].any()  # the limiter indicator (none given)
    assert np.allclose(d["ifUseLimiter"], rhs[:, 0])  # the RHS density entry (8th output)
    assert np.allclose(d["RHSr"], u[:, 4] / rho)  # the SA variable over rho (9th output)


@pytest.mark.gpu
def test_print_data_from_the_solver(tmp_path):
    from dnds_b200 import geometry as G
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(16, True, jitter=0.2)
    cfg = S.preset("vortex")
    s = Solver(m, cfg, precision=0)
    s.set_u(G.isentropic_vortex(m))
    s.ssprk3_step(0.5, 0.2)
    u = s.get_u()
    f = tmp_path / "v.plt"
    P.print_data(str(f), m, u, cfg)
    r = P.read_plt(str(f))
    assert np.array_equal(r["data"]["R"], u[:, 0])
