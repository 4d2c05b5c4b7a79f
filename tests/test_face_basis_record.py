"""The face basis record, on the host: per face and side the basis values at the face centre, the
centre's frame coordinates and the frame offset to the outer Gauss points (18 values per face; the
device headers' setup_face and FaceBasisSide, compiled as plain C++ from tests/face_basis_check.cpp).
The values it gives at the 3 Gauss points must equal the direct evaluation of the basis there (the
30-value table it replaces): FP64 to rounding, and within FP32 resolution when the record is stored in
FP32.  Meshes: jittered periodic triangles (faces that pair a cell with a translated neighbour),
jittered quads with the local principal-axes frame, the Riemann mesh with boundary faces (whose right
side is all zeros) and a coarse NACA 0012 C-mesh with stretched wall cells."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from dnds_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    so = tmp_path_factory.mktemp("fb") / "face_basis_check.so"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "dnds_b200", "csrc"),
                        os.path.join(ROOT, "tests", "face_basis_check.cpp"), "-o", str(so)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(str(so))
    L.face_basis_check.restype = C.c_int
    L.face_basis_check.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 6 + [C.c_int, C.c_void_p, C.c_void_p]
    return L


def _check(lib, m, local):
    arrs = [np.ascontiguousarray(m.node_xy, np.float64), np.ascontiguousarray(m.cell_nodes, np.int32),
            np.ascontiguousarray(m.face_nodes, np.int32), np.ascontiguousarray(m.face_cells, np.int32),
            np.ascontiguousarray(m.face_bc, np.int32), np.ascontiguousarray(m.face_shift, np.float64)]
    e64, e32 = C.c_double(), C.c_double()
    rc = lib.face_basis_check(m.n_cells, m.n_faces, *[a.ctypes.data for a in arrs], int(local),
                              C.addressof(e64), C.addressof(e32))
    assert rc == 0
    return e64.value, e32.value


@pytest.mark.parametrize("name,local", [("vortex_tri", 0), ("vortex_quad", 1), ("riemann_tri", 0), ("naca_cmesh", 1)])
def test_record_gives_the_basis_at_every_gauss_point(lib, name, local):
    m = {"vortex_tri": lambda: M.vortex_mesh(12, True, jitter=0.2, seed=5),
         "vortex_quad": lambda: M.vortex_mesh(12, False, jitter=0.2, seed=6),
         "riemann_tri": lambda: M.riemann_mesh(12),
         "naca_cmesh": lambda: M.naca0012_cmesh(32, 16, 16, first=1e-3, far=10.0)}[name]()
    if name == "vortex_tri":
        assert np.abs(m.face_shift).max() > 0  # periodic faces are covered
    if name == "riemann_tri":
        assert (m.face_cells[:, 1] < 0).any()  # boundary faces are covered
    e64, e32 = _check(lib, m, local)
    # the basis values are O(1) in the cell's frame: FP64 to rounding (measured 4e-15 to 5e-14, the
    # largest on the stretched C-mesh cells), FP32 to a few of its ulps (measured about 1e-7)
    assert e64 < 2e-13, e64
    assert e32 < 5e-7, e32
