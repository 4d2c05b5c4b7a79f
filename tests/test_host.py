"""CPU tests of the host side: mesh builders, settings layout, and the C ABI
library (loads without a GPU and exports every symbol include/dndsg.h declares)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from dnds_b200 import mesh as M
from dnds_b200 import settings as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _signed_area(m):
    xy = m.node_xy
    cn = m.cell_nodes
    nn = np.where(cn[:, 3] < 0, 3, 4)
    a = np.zeros(m.n_cells)
    for k in range(4):
        i = cn[:, k]
        j = np.where(k + 1 < nn, cn[:, (k + 1) % 4], cn[:, 0])
        valid = k < nn
        a += np.where(valid, xy[np.maximum(i, 0), 0] * xy[np.maximum(j, 0), 1] - xy[np.maximum(j, 0), 0] * xy[np.maximum(i, 0), 1], 0)
    return 0.5 * a


@pytest.mark.parametrize("tri", [False, True])
@pytest.mark.parametrize("periodic", [False, True])
def test_structured_grid_topology(tri, periodic):
    m = M.structured_grid(7, 5, 3.0, 2.0, triangles=tri, jitter=0.2, periodic=periodic)
    n_quads = 35
    assert m.n_cells == n_quads * (2 if tri else 1)
    if periodic:
        assert m.n_faces == n_quads * (3 if tri else 2)
        assert np.all(m.face_cells[:, 1] >= 0)
    area = _signed_area(m)
    assert area.min() > 0
    assert abs(area.sum() - 6.0) < 1e-12
    # the right-hand normal of every face points out of its left cell
    a = m.node_xy[m.face_nodes[:, 0]]
    b = m.node_xy[m.face_nodes[:, 1]]
    n = np.stack([b[:, 1] - a[:, 1], a[:, 0] - b[:, 0]], 1)
    cen = lambda c: np.array([m.node_xy[m.cell_nodes[i, :(3 if m.cell_nodes[i, 3] < 0 else 4)]].mean(0) for i in c])
    cl = cen(m.face_cells[:, 0])
    mid = 0.5 * (a + b)
    assert np.all(np.einsum("fk,fk->f", n, cl - mid) < 0)
    if periodic:
        cr = cen(m.face_cells[:, 1]) + m.face_shift
        assert np.all(np.einsum("fk,fk->f", n, cr - mid) > 0)
    # periodic closure: every cell's edge vectors sum to zero
    clo = np.zeros((m.n_cells, 2))
    np.add.at(clo, m.face_cells[:, 0], n)
    inner = m.face_cells[:, 1] >= 0
    np.add.at(clo, m.face_cells[inner, 1], -n[inner])
    if periodic:
        assert np.abs(clo).max() < 1e-14


def test_gmsh_reader(tmp_path):
    p = tmp_path / "sq.msh"
    p.write_text("""$MeshFormat
2.2 0 8
$EndMeshFormat
$PhysicalNames
2
1 1 "bc-3"
2 2 "fluid"
$EndPhysicalNames
$Nodes
5
1 0 0 0
2 1 0 0
3 1 1 0
4 0 1 0
5 0.5 0.5 0
$EndNodes
$Elements
8
1 1 2 1 1 1 2
2 1 2 1 1 2 3
3 1 2 1 1 3 4
4 1 2 1 1 4 1
5 2 2 2 1 1 2 5
6 2 2 2 1 2 3 5
7 2 2 2 1 3 5 4
8 2 2 2 1 4 5 1
$EndElements
""")
    m = M.read_gmsh2(str(p))
    assert m.n_cells == 4 and m.n_faces == 8
    assert np.sum(m.face_bc == M.BC_WALL_EULER) == 4
    assert _signed_area(m).min() > 0


def test_settings_layout_matches_oracle():
    import pyoracle

    assert C.sizeof(S.Settings) == C.sizeof(pyoracle.OrcSettings)
    for (a, ta), (b, tb) in zip(S.Settings._fields_, pyoracle.OrcSettings._fields_):
        assert getattr(S.Settings, a).offset == getattr(pyoracle.OrcSettings, b).offset


def test_settings_from_reference_keys():
    s = S.make_settings(S.preset("riemann"))
    assert s.riemann == 2 and s.weight_scheme_geom == 2 and s.weight_scheme_dir == 0
    assert s.use_local_coord == 0 and s.anisotropic_lengths == 1 and s.limiter == 1
    assert abs(s.weight_len_scale - 0.5) < 1e-15 and abs(s.wbap_smooth_indicator_scale - 0.1) < 1e-15
    v = S.make_settings(S.preset("vortex"))
    assert v.riemann == 1 and v.weight_scheme_geom == 3 and v.weight_scheme_dir == 1 and v.use_local_coord == 1


def test_c_abi_library_exports_header_symbols():
    from dnds_b200 import _lib, build

    build.build()
    header = open(os.path.join(ROOT, "include", "dndsg.h")).read()
    declared = set(re.findall(r"\b(dndsg_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations found"
    assert declared == set(_lib.EXPORTS)
    L = C.CDLL(build.LIB)
    for name in declared:
        assert hasattr(L, name), name
    # the binding resolves every prototype
    _lib.lib()


def test_no_oracle_in_product():
    """The product package must not import or link the oracle."""
    pkg = os.path.join(ROOT, "dnds_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith((".py", ".cu", ".cuh", ".h", ".hpp", ".cpp")):
                txt = open(os.path.join(dirpath, fn)).read()
                assert "pyoracle" not in txt and "dnds_oracle" not in txt, fn
