"""Unstructured 2-D meshes for the DNDS hot path.

A mesh is a set of flat arrays, the same ones the C-ABI takes
(``dndsg_mesh_desc`` in include/dndsg.h):

* ``node_xy``    float64 [n_nodes, 2]
* ``cell_nodes`` int32   [n_cells, 4], counter-clockwise, -1 in slot 3 for a triangle
* ``face_nodes`` int32   [n_faces, 2], ordered so that the right-hand normal of
  node0->node1 points out of the left cell
* ``face_cells`` int32   [n_faces, 2], (left, right); right = -1 on a boundary
* ``face_bc``    int32   [n_faces], DNDS ``BoundaryType`` (DNDS_Mesh.hpp:21-35):
  -1 inner, 1 Wall, 2 Farfield, 3 Wall_Euler, 4 Wall_NoSlip,
  -4 Special_IVFar, -5 Special_2DRiemannFar
* ``face_shift`` float64 [n_faces, 2], the translation that brings the right
  cell next to the face (non-zero only on periodic faces)

The reference builds this topology from Gmsh files
(``CompactFacedMeshSerialRW``, DNDS_Mesh.hpp:634-1906).  The reference has no
periodic boundary; periodic faces are interior faces whose right cell is seen
through ``face_shift``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BC_INNER = -1
BC_WALL = 1
BC_FARFIELD = 2
BC_WALL_EULER = 3
BC_WALL_NOSLIP = 4
BC_DMR_FAR = -2
BC_RT_FAR = -3
BC_IV_FAR = -4
BC_2DRIEMANN_FAR = -5

# Gmsh physical-group names -> BoundaryType (DNDS_Mesh.hpp:801-829)
GMSH_BC_NAMES = {
    "bc-1": BC_WALL,
    "bc-2": BC_FARFIELD,
    "bc-3": BC_WALL_EULER,
    "bc-4": BC_WALL_NOSLIP,
    "bc-DMRFar": BC_DMR_FAR,
    "bc-RTFar": BC_RT_FAR,
    "bc-IVFar": BC_IV_FAR,
    "bc-2DRiemannFar": BC_2DRIEMANN_FAR,
}


@dataclass
class Mesh:
    node_xy: np.ndarray
    cell_nodes: np.ndarray
    face_nodes: np.ndarray
    face_cells: np.ndarray
    face_bc: np.ndarray
    face_shift: np.ndarray
    name: str = "mesh"
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.node_xy.shape[0])

    @property
    def n_cells(self) -> int:
        return int(self.cell_nodes.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_nodes.shape[0])

    def validate(self) -> None:
        """Host-side checks the kernels rely on (they do no bounds checks of their own)."""
        n, f = self.n_cells, self.n_faces
        assert self.node_xy.dtype == np.float64 and self.node_xy.shape == (self.n_nodes, 2)
        assert self.cell_nodes.dtype == np.int32 and self.cell_nodes.shape == (n, 4)
        assert self.face_nodes.dtype == np.int32 and self.face_nodes.shape == (f, 2)
        assert self.face_cells.dtype == np.int32 and self.face_cells.shape == (f, 2)
        assert self.face_bc.dtype == np.int32 and self.face_bc.shape == (f,)
        assert self.face_shift.dtype == np.float64 and self.face_shift.shape == (f, 2)
        cn = self.cell_nodes
        assert cn[:, :3].min() >= 0 and cn.max() < self.n_nodes
        assert self.face_nodes.min() >= 0 and self.face_nodes.max() < self.n_nodes
        L, R = self.face_cells[:, 0], self.face_cells[:, 1]
        assert L.min() >= 0 and L.max() < n and R.max() < n and R.min() >= -1
        assert np.all((R >= 0) == (self.face_bc == BC_INNER)), "inner faces need a right cell"
        deg = np.bincount(L, minlength=n) + np.bincount(R[R >= 0], minlength=n)
        nn = np.where(cn[:, 3] < 0, 3, 4)
        assert np.array_equal(deg, nn), "every cell needs one face per edge"


def _as_mesh(node_xy, cell_nodes, faces, name, meta) -> Mesh:
    fn, fc, fb, fs = faces
    m = Mesh(
        node_xy=np.ascontiguousarray(node_xy, dtype=np.float64),
        cell_nodes=np.ascontiguousarray(cell_nodes, dtype=np.int32),
        face_nodes=np.ascontiguousarray(fn, dtype=np.int32),
        face_cells=np.ascontiguousarray(fc, dtype=np.int32),
        face_bc=np.ascontiguousarray(fb, dtype=np.int32),
        face_shift=np.ascontiguousarray(fs, dtype=np.float64),
        name=name,
        meta=meta,
    )
    m.validate()
    return m


def structured_grid(
    nx: int,
    ny: int,
    lx: float = 10.0,
    ly: float = 10.0,
    x0: float = 0.0,
    y0: float = 0.0,
    triangles: bool = False,
    jitter: float = 0.0,
    seed: int = 1234,
    periodic: bool = True,
    bc: int = BC_FARFIELD,
    name: str | None = None,
) -> Mesh:
    """An nx x ny grid of quads (or 2 triangles per quad) stored as an unstructured mesh.

    ``jitter`` moves every interior node by U(-jitter*h, jitter*h) in x and in y
    (h = grid spacing per direction), drawn from numpy's PCG64 seeded with
    ``seed``; boundary nodes stay put, so periodic faces pair exactly.
    Triangles alternate their diagonal with the parity of (i + j).
    ``periodic`` pairs opposite sides; otherwise every side gets ``bc``.
    """
    hx, hy = lx / nx, ly / ny
    I, J = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")  # [ny+1, nx+1]
    X = x0 + I * hx
    Y = y0 + J * hy
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        d = rng.uniform(-jitter, jitter, size=(ny + 1, nx + 1, 2))
        inner = (I > 0) & (I < nx) & (J > 0) & (J < ny)
        X = X + np.where(inner, d[..., 0] * hx, 0.0)
        Y = Y + np.where(inner, d[..., 1] * hy, 0.0)
    node_xy = np.stack([X.ravel(), Y.ravel()], axis=1)

    def nid(i, j):
        return (j * (nx + 1) + i).astype(np.int64)

    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    ii = ii.ravel()
    jj = jj.ravel()
    q = jj * nx + ii  # quad id, row-major
    n00, n10, n11, n01 = nid(ii, jj), nid(ii + 1, jj), nid(ii + 1, jj + 1), nid(ii, jj + 1)
    nq = nx * ny

    fnodes, fcells, fbc, fshift = [], [], [], []

    def add(nodes, cells, bcs, shifts):
        fnodes.append(nodes)
        fcells.append(cells)
        fbc.append(bcs)
        fshift.append(shifts)

    if not triangles:
        cell_nodes = np.stack([n00, n10, n11, n01], axis=1)
        cid = q
        # bottom edge of quad (i,j): left = this quad (above), right = quad (i, j-1)
        below = jj > 0
        rb = np.where(below, (jj - 1) * nx + ii, (ny - 1) * nx + ii)
        # left edge of quad (i,j): left = this quad, right = quad (i-1, j)
        lft = ii > 0
        rl = np.where(lft, jj * nx + ii - 1, jj * nx + nx - 1)
        cb_b = cid
        cl_l = cid
        cell_of_top = lambda i, j: j * nx + i  # noqa: E731
        cell_of_right = lambda i, j: j * nx + i  # noqa: E731
    else:
        even = ((ii + jj) % 2) == 0
        t0 = 2 * q
        t1 = 2 * q + 1
        tri0 = np.where(even[:, None], np.stack([n00, n10, n11], 1), np.stack([n00, n10, n01], 1))
        tri1 = np.where(even[:, None], np.stack([n00, n11, n01], 1), np.stack([n10, n11, n01], 1))
        cell_nodes = np.full((2 * nq, 4), -1, dtype=np.int64)
        cell_nodes[0::2, :3] = tri0
        cell_nodes[1::2, :3] = tri1
        cb_b = t0  # the bottom edge always belongs to triangle 0
        cl_l = np.where(even, t1, t0)  # left edge: even -> T1, odd -> T0

        def cell_of_top(i, j):  # top edge of quad (i,j) belongs to triangle 1
            return 2 * (j * nx + i) + 1

        def cell_of_right(i, j):  # right edge: even -> T0, odd -> T1
            return 2 * (j * nx + i) + np.where(((i + j) % 2) == 0, 0, 1)

        rb = None
        rl = None

    # --- bottom faces
    jb = jj - 1
    wrap_b = jj == 0
    if periodic:
        rbc = np.where(wrap_b, cell_of_top(ii, np.full_like(jj, ny - 1)), cell_of_top(ii, np.maximum(jb, 0)))
        sh = np.stack([np.zeros(nq), np.where(wrap_b, -ly, 0.0)], 1)
        add(np.stack([n00, n10], 1), np.stack([cb_b, rbc], 1), np.full(nq, BC_INNER), sh)
    else:
        rbc = np.where(wrap_b, -1, cell_of_top(ii, np.maximum(jb, 0)))
        add(np.stack([n00, n10], 1), np.stack([cb_b, rbc], 1), np.where(wrap_b, bc, BC_INNER), np.zeros((nq, 2)))
    # --- left faces
    il = ii - 1
    wrap_l = ii == 0
    if periodic:
        rlc = np.where(wrap_l, cell_of_right(np.full_like(ii, nx - 1), jj), cell_of_right(np.maximum(il, 0), jj))
        sh = np.stack([np.where(wrap_l, -lx, 0.0), np.zeros(nq)], 1)
        add(np.stack([n01, n00], 1), np.stack([cl_l, rlc], 1), np.full(nq, BC_INNER), sh)
    else:
        rlc = np.where(wrap_l, -1, cell_of_right(np.maximum(il, 0), jj))
        add(np.stack([n01, n00], 1), np.stack([cl_l, rlc], 1), np.where(wrap_l, bc, BC_INNER), np.zeros((nq, 2)))
    # --- diagonals
    if triangles:
        even = ((ii + jj) % 2) == 0
        dn = np.where(even[:, None], np.stack([n00, n11], 1), np.stack([n01, n10], 1))
        add(dn, np.stack([2 * q + 1, 2 * q], 1), np.full(nq, BC_INNER), np.zeros((nq, 2)))
    if not periodic:
        # top row and right column boundary faces
        it = np.arange(nx)
        add(
            np.stack([nid(it + 1, np.full(nx, ny)), nid(it, np.full(nx, ny))], 1),
            np.stack([cell_of_top(it, np.full(nx, ny - 1)), np.full(nx, -1)], 1),
            np.full(nx, bc),
            np.zeros((nx, 2)),
        )
        jt = np.arange(ny)
        add(
            np.stack([nid(np.full(ny, nx), jt), nid(np.full(ny, nx), jt + 1)], 1),
            np.stack([cell_of_right(np.full(ny, nx - 1), jt), np.full(ny, -1)], 1),
            np.full(ny, bc),
            np.zeros((ny, 2)),
        )
    # interleave the per-quad faces so that faces of nearby cells are nearby in memory
    nper = 3 if triangles else 2
    fn = np.stack([a for a in fnodes[:nper]], 1).reshape(-1, 2)
    fc = np.stack([a for a in fcells[:nper]], 1).reshape(-1, 2)
    fb = np.stack([a for a in fbc[:nper]], 1).reshape(-1)
    fs = np.stack([a for a in fshift[:nper]], 1).reshape(-1, 2)
    if len(fnodes) > nper:
        fn = np.concatenate([fn] + fnodes[nper:], 0)
        fc = np.concatenate([fc] + fcells[nper:], 0)
        fb = np.concatenate([fb] + fbc[nper:], 0)
        fs = np.concatenate([fs] + fshift[nper:], 0)
    # a periodic face's right cell is the cell on the opposite side: its shift
    # moves that cell next to the face (bottom: R lies at the top -> -ly)
    meta = dict(nx=nx, ny=ny, lx=lx, ly=ly, x0=x0, y0=y0, triangles=triangles, jitter=jitter, seed=seed,
                periodic=periodic)
    nm = name or f"{'tri' if triangles else 'quad'}{nx}x{ny}{'_per' if periodic else ''}"
    return _as_mesh(node_xy, cell_nodes, (fn, fc, fb, fs), nm, meta)


def vortex_mesh(n: int, triangles: bool, jitter: float = 0.0, seed: int = 1234) -> Mesh:
    """Periodic [0,10]^2 isentropic-vortex mesh (n x n quads, optionally split)."""
    return structured_grid(n, n, 10.0, 10.0, triangles=triangles, jitter=jitter, seed=seed, periodic=True)


def riemann_mesh(n: int, jitter: float = 0.15, seed: int = 4321) -> Mesh:
    """[0,1]^2 four-quadrant Riemann mesh, triangles, Special_2DRiemannFar on all sides."""
    return structured_grid(n, n, 1.0, 1.0, triangles=True, jitter=jitter, seed=seed, periodic=False,
                           bc=BC_2DRIEMANN_FAR)


def faces_from_cells(node_xy, cell_nodes, boundary_bc):
    """Faces of a conforming mesh of counter-clockwise cells.  An edge a->b of a cell
    has its right-hand normal out of that cell, so the first cell met owns the face as
    its left cell and the cell that runs the edge b->a becomes the right cell.
    boundary_bc(a, b) gives the BoundaryType of an edge with one cell."""
    cell_nodes = np.asarray(cell_nodes)
    key_face = {}
    fn, fc = [], []
    for c in range(cell_nodes.shape[0]):
        nodes = [int(v) for v in cell_nodes[c] if v >= 0]
        for k in range(len(nodes)):
            a, b = nodes[k], nodes[(k + 1) % len(nodes)]
            key = (a, b) if a < b else (b, a)
            f = key_face.get(key)
            if f is None:
                key_face[key] = len(fn)
                fn.append((a, b))
                fc.append([c, -1])
            else:
                assert fc[f][1] < 0 and fn[f] == (b, a), "non-conforming or mis-oriented cells"
                fc[f][1] = c
    fb = [BC_INNER if r >= 0 else int(boundary_bc(a, b)) for (a, b), (_, r) in zip(fn, fc)]
    return np.array(fn), np.array(fc), np.array(fb), np.zeros((len(fn), 2))


def _geometric_ratio(d0: float, n: int, total: float) -> float:
    """The ratio q > 1 with d0 (q^n - 1) / (q - 1) = total (bisection; needs n d0 < total)."""
    assert n * d0 < total
    lo, hi = 1.0 + 1e-12, 2.0
    while d0 * (hi ** n - 1) / (hi - 1) < total:
        hi *= 2
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if d0 * (mid ** n - 1) / (mid - 1) < total:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def naca0012_cmesh(n_airfoil: int = 256, n_wake: int = 128, nj: int = 128, first: float = 1e-6,
                   far: float = 20.0, wall_bc: int = BC_WALL_NOSLIP, far_bc: int = BC_FARFIELD) -> Mesh:
    """C-mesh of quadrilaterals around the NACA 0012 (4-digit thickness formula, closed trailing
    edge, chord 1 from (0,0) to (1,0)): n_airfoil cells along the surface (cosine-clustered at both
    edges), n_wake cells on each wake branch out to x = 1 + far, nj cells from the wall to the outer
    boundary at distance `far`, the first one `first` (times the line length over `far`) thick and
    the rest growing geometrically at the ratio that reaches `far` in nj cells.  The wake cut is a
    line of interior faces.  Cells run (n_wake + n_airfoil + n_wake) x nj; faces on the airfoil get
    wall_bc, the outer C and the two outflow lines far_bc."""
    assert n_airfoil % 2 == 0
    ni = 2 * n_wake + n_airfoil

    def yt(x):
        return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)

    h = n_airfoil // 2
    xs = 0.5 * (1 - np.cos(np.pi * np.arange(h + 1) / h))          # LE (0) -> TE (1)
    lower = np.stack([xs[::-1], -yt(xs[::-1])], 1)                   # TE -> LE
    upper = np.stack([xs[1:], yt(xs[1:])], 1)                        # after LE -> TE
    surf = np.concatenate([lower, upper])                            # n_airfoil + 1 points
    # wake: geometric from the trailing-edge spacing to x = 1 + far
    d0 = xs[-1] - xs[-2]
    r = _geometric_ratio(d0, n_wake, far)
    xw = 1.0 + d0 * (r ** np.arange(n_wake + 1) - 1) / (r - 1)
    xw[-1] = 1.0 + far
    wl = np.stack([xw[::-1], np.zeros(n_wake + 1)], 1)[:-1]          # far -> TE (TE excluded)
    wu = np.stack([xw, np.zeros(n_wake + 1)], 1)[1:]                 # after TE -> far
    inner = np.concatenate([wl, surf, wu])                           # ni + 1 points
    # outer C: straight lines below/above the wake, half circle of radius far about (1, 0).
    # Surface point x maps to the circle point straight above/below it (phi = asin((1 - x)/far)),
    # fanning out towards the leading edge ((pi/2) s^8, s = 0 at the trailing edge, 1 at the
    # leading edge); grid lines are straight from the surface to the outer boundary.
    sfrac = np.arange(h + 1) / h                                      # TE (0) -> LE (1)
    phi = np.maximum(np.arcsin(np.minimum(1.0, (1 - xs[::-1]) / far)), 0.5 * np.pi * sfrac ** 8)
    lo_out = np.stack([1 - far * np.sin(phi), -far * np.cos(phi)], 1)            # TE -> LE
    up_out = np.stack([1 - far * np.sin(phi[::-1]), far * np.cos(phi[::-1])], 1)[1:]  # after LE -> TE
    outer = np.concatenate([np.stack([xw[::-1][:-1], -far * np.ones(n_wake)], 1), lo_out, up_out,
                            np.stack([xw[1:], far * np.ones(n_wake)], 1)])
    # distances: first cell `first`, geometric ratio q reaching `far` in nj cells
    q = _geometric_ratio(first, nj, far)
    dist = first * (q ** np.arange(nj + 1) - 1) / (q - 1)
    frac = dist / dist[-1]
    P = inner[:, None, :] + frac[None, :, None] * (outer - inner)[:, None, :]  # [ni+1, nj+1, 2]
    # node numbering; upper-wake wall nodes are the lower-wake ones (the cut)
    nid = np.arange((ni + 1) * (nj + 1)).reshape(ni + 1, nj + 1)
    for i in range(n_wake + 1):
        nid[ni - i, 0] = nid[i, 0]
    used = np.unique(nid)
    remap = -np.ones(nid.size, dtype=np.int64)
    remap[used] = np.arange(used.size)
    nid = remap[nid]
    xy = np.zeros((used.size, 2))
    xy[nid.ravel()] = P.reshape(-1, 2)
    ii, jj = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")
    cells = np.stack([nid[ii, jj], nid[ii + 1, jj], nid[ii + 1, jj + 1], nid[ii, jj + 1]], -1).reshape(-1, 4)
    wall_nodes = set(int(v) for v in nid[n_wake:n_wake + n_airfoil + 1, 0])

    def bc(a, b):
        return wall_bc if (a in wall_nodes and b in wall_nodes) else far_bc

    faces = faces_from_cells(xy, cells, bc)
    meta = dict(kind="naca0012_cmesh", n_airfoil=n_airfoil, n_wake=n_wake, nj=nj, first=first, far=far,
                normal_ratio=float(q), wake_ratio=float(r))
    return _as_mesh(xy, cells, faces, f"naca0012_c{ni}x{nj}", meta)


def hilbert_order(points: np.ndarray, bits: int = 16) -> np.ndarray:
    """The indices that sort points [n, 2] along a Hilbert curve through their bounding square, quantised
    to a 2^bits x 2^bits grid (the iterative index of the curve: per bit level, the quadrant's
    contribution s^2 ((3 rx) xor ry), then the quadrant's rotation).  Consecutive points of the order
    are close in space."""
    pts = np.asarray(points, dtype=np.float64)
    lo = pts.min(0)
    span = max(float(np.ptp(pts[:, 0])), float(np.ptp(pts[:, 1])), 1e-300)
    n = 1 << bits
    q = np.clip(((pts - lo) / span * (n - 1)).astype(np.int64), 0, n - 1)
    x, y = q[:, 0].copy(), q[:, 1].copy()
    d = np.zeros(len(pts), dtype=np.int64)
    s = n >> 1
    while s > 0:
        rx = ((x & s) > 0).astype(np.int64)
        ry = ((y & s) > 0).astype(np.int64)
        d += s * s * ((3 * rx) ^ ry)
        flip = (ry == 0) & (rx == 1)
        x = np.where(flip, n - 1 - x, x)
        y = np.where(flip, n - 1 - y, y)
        swap = ry == 0
        x, y = np.where(swap, y, x), np.where(swap, x, y)
        s >>= 1
    return np.argsort(d, kind="stable")


def renumber(m: Mesh, order: np.ndarray | None = None) -> tuple[Mesh, np.ndarray]:
    """A METIS-free renumbering for locality: the mesh with its cells in `order` (new cell k is old cell
    order[k]; default the Hilbert order of the cell centroids) and its faces sorted by the lower new
    index of their cells, so that the cells and faces a kernel gathers together sit close in memory.
    Every cell keeps its nodes (hence its element-local face order) and every face its nodes, cells
    (renumbered), boundary type and periodic shift, so the discretisation is unchanged: results on the
    new mesh are those of the old one, permuted.  Returns (mesh, order); a state of the old mesh maps
    to the new one as u[order]."""
    n = m.n_cells
    cn = m.cell_nodes
    valid = cn >= 0
    cent = (m.node_xy[np.maximum(cn, 0)] * valid[:, :, None]).sum(1) / valid.sum(1)[:, None]
    order = hilbert_order(cent) if order is None else np.asarray(order, dtype=np.int64)
    if order.shape != (n,) or not np.array_equal(np.sort(order), np.arange(n)):
        raise ValueError("order is not a permutation of the cells")
    new_of_old = np.empty(n, dtype=np.int64)
    new_of_old[order] = np.arange(n)
    L = new_of_old[m.face_cells[:, 0]]
    R = np.where(m.face_cells[:, 1] >= 0, new_of_old[np.maximum(m.face_cells[:, 1], 0)], -1)
    lo = np.where(R >= 0, np.minimum(L, R), L)
    fperm = np.lexsort((np.maximum(L, R), lo))
    faces = (m.face_nodes[fperm], np.stack([L, R], 1)[fperm], m.face_bc[fperm], m.face_shift[fperm])
    meta = {"renumbered_from": m.name}
    return _as_mesh(m.node_xy, cn[order], faces, f"{m.name}_renumbered", meta), order


def line_scan_order(m: Mesh) -> np.ndarray:
    """LU-SGS scan order for a C-mesh from naca0012_cmesh: the wall-normal grid lines, even ones
    first, then odd ones, each from the wall outwards.  Like the natural cell order (which also runs
    along the wall-normal lines fastest) it sweeps the strongly coupled stretched cells of a line in
    sequence, but lines of one parity share no face (the wake cut pairs line i with line
    2 n_wake + n_airfoil - 1 - i, of the other parity), so a level-scheduled sweep has nj + 1 levels
    (the odd lines run one level behind the even ones) instead of the natural order's ni + nj - 1."""
    assert m.meta.get("kind") == "naca0012_cmesh", "line_scan_order needs a naca0012_cmesh"
    nj = m.meta["nj"]
    ni = m.n_cells // nj
    idx = np.arange(ni * nj).reshape(ni, nj)
    return np.concatenate([idx[0::2].ravel(), idx[1::2].ravel()]).astype(np.int64)


def parse_gmsh2(path: str) -> dict:
    """The raw content of a Gmsh 2.2 ASCII file (SerialGmshReader2d, DNDS_Mesh.hpp:87-236), for 2-D
    meshes: nodes [n][2] indexed by Gmsh node id (row 0 unused), cells [n][4] Gmsh node ids (Tri3 with
    slot 3 = -1, Quad4), boundary lines [n][3] (node, node, physical group) and the physical-group
    names."""
    with open(path) as fh:
        lines = [ln.strip() for ln in fh]
    k = 0
    names = {}
    nodes = None
    cells = []
    bnd = []
    while k < len(lines):
        ln = lines[k]
        if ln == "$PhysicalNames":
            cnt = int(lines[k + 1])
            for t in range(cnt):
                parts = lines[k + 2 + t].split()
                names[int(parts[1])] = parts[2].strip('"')
            k += cnt + 3
        elif ln == "$Nodes":
            cnt = int(lines[k + 1])
            arr = np.array([lines[k + 2 + t].split() for t in range(cnt)], dtype=np.float64)
            ids = arr[:, 0].astype(np.int64)
            nodes = np.zeros((int(ids.max()) + 1, 2))
            nodes[ids] = arr[:, 1:3]
            k += cnt + 3
        elif ln == "$Elements":
            cnt = int(lines[k + 1])
            for t in range(cnt):
                p = [int(v) for v in lines[k + 2 + t].split()]
                et, ntag = p[1], p[2]
                phys = p[3] if ntag > 0 else -1
                conn = p[3 + ntag:]
                if et == 1:
                    bnd.append((conn[0], conn[1], phys))
                elif et == 2:
                    cells.append(conn[:3] + [-1])
                elif et == 3:
                    cells.append(conn[:4])
                else:
                    raise ValueError(f"{path}: element type {et} is not a 2-D Line2 / Tri3 / Quad4 element")
            k += cnt + 3
        else:
            k += 1
    if nodes is None:
        raise ValueError(f"{path}: no $Nodes section")
    return {"nodes": nodes, "cells": np.array(cells, dtype=np.int64).reshape(-1, 4),
            "bnd": np.array(bnd, dtype=np.int64).reshape(-1, 3),
            "names": names}


def gmsh_mesh(g: dict, name: str = "gmsh") -> Mesh:
    """The mesh of parsed Gmsh content (parse_gmsh2): cells made counter-clockwise, faces extracted from
    the cell edges in cell order and local edge order (the reference's vol2face construction,
    DNDS_Mesh.hpp:260-320), boundary faces typed from their physical-group names as in
    DNDS_Mesh.hpp:801-829 (bc-1 Wall, bc-2 Farfield, bc-3 Wall_Euler, bc-4 Wall_NoSlip, bc-DMRFar,
    bc-RTFar, bc-IVFar, bc-2DRiemannFar).  A boundary face without a line element, or on a line of
    another name, is an error (the reference asserts)."""
    nodes, cells, bnd, names = g["nodes"], g["cells"], g["bnd"], g["names"]
    used = np.unique(np.concatenate([cells[cells >= 0].ravel(), bnd[:, :2].ravel()]))
    remap = -np.ones(nodes.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    node_xy = nodes[used]
    cn = np.where(cells >= 0, remap[np.maximum(cells, 0)], -1)
    # orient counter-clockwise
    for i in range(cn.shape[0]):
        nn = 3 if cn[i, 3] < 0 else 4
        p = node_xy[cn[i, :nn]]
        a = 0.5 * np.sum(p[:, 0] * np.roll(p[:, 1], -1) - np.roll(p[:, 0], -1) * p[:, 1])
        if a < 0:
            cn[i, :nn] = cn[i, :nn][::-1]
    bmap = {}
    for a, b, phys in bnd:
        key = (min(remap[a], remap[b]), max(remap[a], remap[b]))
        nm = names.get(int(phys), "")
        if nm not in GMSH_BC_NAMES:
            raise ValueError(f"boundary physical group {phys} named {nm!r} is not a DNDS boundary name")
        bmap[key] = GMSH_BC_NAMES[nm]
    edges = {}
    fn, fc, fb = [], [], []
    for i in range(cn.shape[0]):
        nn = 3 if cn[i, 3] < 0 else 4
        for e in range(nn):
            a, b = int(cn[i, e]), int(cn[i, (e + 1) % nn])
            key = (min(a, b), max(a, b))
            if key in edges:
                fc[edges[key]][1] = i
            else:
                edges[key] = len(fn)
                fn.append([a, b])
                fc.append([i, -1])
    for f, (a, b) in enumerate(fn):
        key = (min(a, b), max(a, b))
        if fc[f][1] >= 0:
            fb.append(BC_INNER)
        elif key in bmap:
            fb.append(bmap[key])
        else:
            raise ValueError(f"boundary face ({a}, {b}) has no boundary line element")
    nf = len(fn)
    return _as_mesh(node_xy, cn, (np.array(fn), np.array(fc), np.array(fb), np.zeros((nf, 2))), name, {})


def read_gmsh2(path: str) -> Mesh:
    """Gmsh 2.2 ASCII reader for 2-D meshes (SerialGmshReader2d, DNDS_Mesh.hpp:87-236, and the face
    and boundary set-up of DNDS_Mesh.hpp:260-320, 801-829): parse_gmsh2, then gmsh_mesh."""
    return gmsh_mesh(parse_gmsh2(path), path)
