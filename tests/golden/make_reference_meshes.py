"""Stores two of the reference's own Gmsh meshes as test fixtures (the GPU box has no copy of the
reference): data/mesh/Uniform128.msh (128 x 128 quads on the unit square, walls "bc-3" =
Wall_Euler) and data/mesh/NACA0012_WIDE_H3_NS.msh (14,280 quads around a NACA 0012, "bc-4" =
Wall_NoSlip, "bc-2" = Farfield).  Each fixture holds the parsed file content -- nodes, cells,
boundary lines and physical-group names, as dnds_b200.mesh.parse_gmsh2 reads them -- so the tests
build the mesh with the same code path as read_gmsh2.

Run from the repository root with the reference checked out at ../reference or REFERENCE_ROOT:
    python tests/golden/make_reference_meshes.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from dnds_b200 import mesh as M  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
MESHES = {"gmsh_uniform128": "Uniform128.msh", "gmsh_naca0012_wide_h3_ns": "NACA0012_WIDE_H3_NS.msh"}


def reference_mesh_dir():
    ref = os.environ.get("REFERENCE_ROOT", "/root/reference")
    return os.path.join(ref, "data", "mesh")


def fixture_arrays(g):
    return dict(nodes=g["nodes"], cells=g["cells"].astype(np.int32), bnd=g["bnd"].astype(np.int32),
                names=np.array(json.dumps({str(k): v for k, v in g["names"].items()})))


def load_fixture(name):
    """The parsed Gmsh content of a stored fixture, as parse_gmsh2 returns it."""
    d = np.load(os.path.join(OUT, f"{name}.npz"))
    return {"nodes": d["nodes"], "cells": d["cells"].astype(np.int64), "bnd": d["bnd"].astype(np.int64),
            "names": {int(k): v for k, v in json.loads(str(d["names"])).items()}}


if __name__ == "__main__":
    for name, fn in MESHES.items():
        g = M.parse_gmsh2(os.path.join(reference_mesh_dir(), fn))
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **fixture_arrays(g))
        m = M.gmsh_mesh(g, fn)
        print(name, m.n_nodes, "nodes", m.n_cells, "cells", m.n_faces, "faces")
