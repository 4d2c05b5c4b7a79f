"""Tecplot binary output of solver results, the file the reference writes for post-processing.

`write_plt` restates `CompactFacedMeshSerialRW::PrintSerialPartPltBinaryDataArray`
(DNDS_Mesh.hpp:1639-1817): a "#!TDV112" binary file with one finite-element quadrilateral zone,
X / Y / Z at the nodes (Z = 0 in 2-D), the data arrays and "iPart" cell-centred, every value in
double precision, triangles written as quadrilaterals with the last node repeated, zero-based
connectivity.  `print_data` restates `EulerSolver::PrintData` (DNDS_FV_EulerSolver.hpp:1436-1492): per
cell the density, velocity, pressure, temperature p / (rho Rgas), Mach number, the limiter indicator
over WBAP_SmoothIndicatorScale, the density entry of the latest ODE right-hand side and, for the SA
variable, U5 / rho; the names are the reference's list cut to its length nVars + 4 (so, in 2-D, the
reference labels pressure "W", temperature "P" and so on; the labels are kept so that the
reference's post-processing reads these files the same way).

`read_plt` parses such a file back (used by the tests, and handy for A/B comparisons).
"""
from __future__ import annotations

import struct

import numpy as np

_NAMES = ["R", "U", "V", "W", "P", "T", "M", "ifUseLimiter", "RHSr"]


def _s(text: str) -> bytes:
    return struct.pack(f"<{len(text) + 1}i", *[ord(ch) for ch in text], 0)


def write_plt(path: str, node_xy: np.ndarray, cell_nodes: np.ndarray, names, data, t: float = 0.0,
              title: str = "TitleHahaha", n_parts: int = 1, part=None) -> None:
    """Writes the zone: node_xy [n_nodes][2 or 3], cell_nodes [n_cells][4] (-1 in the last column for a
    triangle), names [k], data [k][n_cells], part [n_cells] (the owning rank; 0 when None)."""
    xyz = np.zeros((len(node_xy), 3))
    xyz[:, : node_xy.shape[1]] = node_xy
    cn = np.asarray(cell_nodes, dtype=np.int64)
    quad = cn.copy()
    tri = quad[:, 3] < 0
    quad[tri, 3] = quad[tri, 2]
    data = np.asarray(data, dtype=np.float64).reshape(len(names), len(cn))
    part = np.zeros(len(cn)) if part is None else np.asarray(part, dtype=np.float64)
    k = len(names)
    out = [b"#!TDV112", struct.pack("<ii", 1, 0), _s(title), struct.pack("<i", k + 3 + 1)]
    out += [_s("X"), _s("Y"), _s("Z")] + [_s(nm) for nm in names] + [_s("iPart")]
    out += [struct.pack("<f", 299.0), _s("zone_0"), struct.pack("<ii", -1, -1), struct.pack("<d", t),
            struct.pack("<iii", -1, 3, 1)]
    out += [struct.pack("<3i", 0, 0, 0), struct.pack(f"<{k}i", *([1] * k)), struct.pack("<i", 1)]
    out += [struct.pack("<ii", 0, 0), struct.pack("<ii", len(xyz), len(cn)), struct.pack("<4i", 0, 0, 0, 0)]
    out += [struct.pack("<f", 357.0), struct.pack("<f", 299.0), struct.pack(f"<{k + 4}i", *([2] * (k + 4)))]
    out += [struct.pack("<iii", 0, 0, -1)]
    for d in range(3):
        out.append(struct.pack("<dd", xyz[:, d].min(), xyz[:, d].max()))
    for j in range(k):
        out.append(struct.pack("<dd", data[j].min(), data[j].max()))
    out.append(struct.pack("<dd", 0.0, float(n_parts)))
    out += [np.ascontiguousarray(xyz[:, d], dtype="<f8").tobytes() for d in range(3)]
    out += [np.ascontiguousarray(data[j], dtype="<f8").tobytes() for j in range(k)]
    out.append(np.ascontiguousarray(part, dtype="<f8").tobytes())
    out.append(np.ascontiguousarray(quad, dtype="<i4").tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(out))


def read_plt(path: str) -> dict:
    """Parses a file written by write_plt: title, names, t, node coordinates [n][3], data
    {name: [n_cells]}, connectivity [n_cells][4]."""
    b = open(path, "rb").read()
    assert b[:8] == b"#!TDV112", "not a Tecplot v112 binary file"
    pos = 8

    def i32(n=1):
        nonlocal pos
        v = struct.unpack_from(f"<{n}i", b, pos)
        pos += 4 * n
        return v if n > 1 else v[0]

    def f32():
        nonlocal pos
        v = struct.unpack_from("<f", b, pos)[0]
        pos += 4
        return v

    def f64(n=1):
        nonlocal pos
        v = struct.unpack_from(f"<{n}d", b, pos)
        pos += 8 * n
        return v if n > 1 else v[0]

    def string():
        chars = []
        while True:
            c = i32()
            if c == 0:
                return "".join(chars)
            chars.append(chr(c))

    i32(2)
    title = string()
    nv = i32()
    names = [string() for _ in range(nv)]
    assert f32() == 299.0
    string()  # zone name
    i32(2)
    t = f64()
    i32()
    zone_type, located = i32(), i32()
    assert zone_type == 3 and located == 1
    i32(nv)  # locations
    i32(2)
    n_nodes, n_cells = i32(), i32()
    i32(4)
    assert f32() == 357.0 and f32() == 299.0
    i32(nv)  # formats
    i32(3)
    f64(2 * nv)  # min / max
    xyz = np.stack([np.frombuffer(b, "<f8", n_nodes, pos + 8 * n_nodes * d) for d in range(3)], 1)
    pos += 24 * n_nodes
    data = {}
    for nm in names[3:]:
        data[nm] = np.frombuffer(b, "<f8", n_cells, pos).copy()
        pos += 8 * n_cells
    conn = np.frombuffer(b, "<i4", 4 * n_cells, pos).reshape(n_cells, 4).copy()
    pos += 16 * n_cells
    assert pos == len(b)
    return {"title": title, "names": names, "t": t, "xyz": xyz, "data": data, "conn": conn}


def print_data(path: str, mesh, u: np.ndarray, cfg: dict, rhs=None, limiter=None, t: float = 0.0) -> None:
    """EulerSolver::PrintData from the cell means u [n_cells][nvars] (host), the latest ODE
    right-hand side rhs [n_cells][nvars] (None: zeros) and the limiter indicator [n_cells] (None:
    zeros)."""
    gas = cfg.get("eulerSetting", {}).get("idealGasProperty", {})
    gamma, rgas = float(gas.get("gamma", 1.4)), float(gas.get("Rgas", 1.0))
    scale = float(cfg.get("vfvSetting", {}).get("WBAP_SmoothIndicatorScale", 1e-100))
    u = np.asarray(u, dtype=np.float64)
    n, nvars = u.shape
    rho = u[:, 0]
    vel = u[:, 1:3] / rho[:, None]
    vsqr = (vel ** 2).sum(1)
    p = (gamma - 1) * (u[:, 3] - 0.5 * rho * vsqr)
    a2 = gamma * p / rho
    out = [rho, vel[:, 0], vel[:, 1], p, p / rho / rgas, np.sqrt(vsqr / a2),
           (np.zeros(n) if limiter is None else np.asarray(limiter)) / (scale + 1e-200),
           np.zeros(n) if rhs is None else np.asarray(rhs)[:, 0]]
    out += [u[:, i] / rho for i in range(4, nvars)]
    names = (_NAMES + [f"V{i - 3}" for i in range(4, nvars)])[: nvars + 4]
    write_plt(path, mesh.node_xy, mesh.cell_nodes, names, np.stack(out), t=t)
