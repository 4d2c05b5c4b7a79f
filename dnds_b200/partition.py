"""Partitioned runs: the reference's MPI domain decomposition (one rank per partition, a one-cell
ghost layer pulled after every reconstruction sweep and stage, ``ArrayDOFV::StartPersistentPullClean``
in ``DNDS_FV_EulerSolver.hpp:713-837``) with one solver context per partition.

``partition_mesh`` cuts the cells into ``nparts`` contiguous blocks of the cell order (the
generators number cells row by row, so these are slabs) and builds, per part, a mesh of its owned
cells followed by one layer of ghost cells (every cell across a face of an owned cell).  A ghost's
faces to cells outside the part become far-field faces, so every local cell is closed and the usual
setup applies; ghost values are recomputed locally but overwritten by the exchange before anything
owned reads them, so the owned cells evolve exactly as in the whole mesh.

``PartitionedRun`` steps all parts by SSP-RK3 stage through the C ABI (``dndsg_rk_*``), exchanging
ghost coefficients after each sweep (and limiter) and ghost means after each stage update, and
reducing dt over the parts.  In one process the parts share a GPU and the exchange is a device copy;
``exchange`` is the only step a multi-GPU run replaces (NCCL send / receive of the same packed
buffers between ranks).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import mesh as M


@dataclass
class Part:
    mesh: M.Mesh
    cells: np.ndarray    # global ids of the local cells: owned first, then ghosts
    n_owned: int
    # exchange lists: recv[q] = local ghost indices owned by part q; send[q] = local owned indices that
    # part q holds as ghosts (both in increasing global id, so that they pair up)
    recv: dict
    send: dict


def _neighbours(mesh: M.Mesh):
    L, R = mesh.face_cells[:, 0], mesh.face_cells[:, 1]
    inner = R >= 0
    a = np.concatenate([L[inner], R[inner]])
    b = np.concatenate([R[inner], L[inner]])
    order = np.argsort(a, kind="stable")
    a, b = a[order], b[order]
    start = np.searchsorted(a, np.arange(mesh.n_cells + 1))
    return start, b


def block_owner(n_cells: int, nparts: int) -> np.ndarray:
    """The part of every cell: nparts contiguous blocks of the cell order (int32)."""
    return ((np.arange(n_cells, dtype=np.int64) * nparts) // n_cells).astype(np.int32)


def partition_mesh(mesh: M.Mesh, nparts: int) -> list[Part]:
    n = mesh.n_cells
    owner = block_owner(n, nparts).astype(np.int64)
    start, nb = _neighbours(mesh)
    parts = []
    for p in range(nparts):
        owned = np.nonzero(owner == p)[0]
        ring = np.unique(np.concatenate([nb[start[i]:start[i + 1]] for i in owned])) if len(owned) else np.zeros(0, int)
        ghosts = ring[owner[ring] != p]
        cells = np.concatenate([owned, ghosts])
        g2l = np.full(n, -1, dtype=np.int64)
        g2l[cells] = np.arange(len(cells))
        # nodes of the local cells
        cn = mesh.cell_nodes[cells]
        used = np.unique(cn[cn >= 0])
        n2l = np.full(mesh.n_nodes, -1, dtype=np.int64)
        n2l[used] = np.arange(len(used))
        xy = [mesh.node_xy[used]]
        n_nodes = len(used)
        cell_nodes = np.where(cn >= 0, n2l[np.maximum(cn, 0)], -1)
        # faces touching a local cell, in global order
        L, R = mesh.face_cells[:, 0], mesh.face_cells[:, 1]
        lL, lR = g2l[L], np.where(R >= 0, g2l[np.maximum(R, 0)], -1)
        keep = np.nonzero((lL >= 0) | (lR >= 0))[0]
        fn, fc, fb, fs = [], [], [], []
        for f in keep:
            a, b = mesh.face_nodes[f]
            if lL[f] >= 0 and (R[f] < 0 or lR[f] >= 0):  # a boundary face or an inner face of two local cells
                fn.append((n2l[a], n2l[b]))
                fc.append((lL[f], lR[f] if R[f] >= 0 else -1))
                fb.append(mesh.face_bc[f])
                fs.append(mesh.face_shift[f])
            elif lL[f] >= 0:  # the right cell lies outside: a far-field face of the left (ghost) cell
                fn.append((n2l[a], n2l[b]))
                fc.append((lL[f], -1))
                fb.append(M.BC_FARFIELD)
                fs.append((0.0, 0.0))
            else:  # the left cell lies outside: reversed, and in the right cell's own frame on a periodic face
                s = mesh.face_shift[f]
                if s[0] != 0.0 or s[1] != 0.0:
                    xy.append(np.stack([mesh.node_xy[b] - s, mesh.node_xy[a] - s]))
                    na, nb_ = n_nodes, n_nodes + 1
                    n_nodes += 2
                else:
                    na, nb_ = n2l[b], n2l[a]
                fn.append((na, nb_))
                fc.append((lR[f], -1))
                fb.append(M.BC_FARFIELD)
                fs.append((0.0, 0.0))
        sub = M._as_mesh(np.concatenate(xy), cell_nodes, (np.array(fn), np.array(fc), np.array(fb), np.array(fs)),
                         f"{mesh.name}_part{p}of{nparts}", {"owned": len(owned)})
        recv = {}
        for q in np.unique(owner[ghosts]):
            gq = ghosts[owner[ghosts] == q]
            recv[int(q)] = g2l[gq].astype(np.int32)
        parts.append(Part(sub, cells, len(owned), recv, {}))
    for p, part in enumerate(parts):  # send lists: what part q holds of p, in the same (global id) order
        for q, other in enumerate(parts):
            if q == p or p not in other.recv:
                continue
            g = other.cells[other.recv[p]]
            g2l = {int(c): k for k, c in enumerate(part.cells[: part.n_owned])}
            part.send[q] = np.array([g2l[int(c)] for c in g], dtype=np.int32)
    return parts


class PartitionedRun:
    """All parts of a mesh on one GPU, stepped together; ``u`` gathers the owned means."""

    def __init__(self, mesh: M.Mesh, cfg: dict, nparts: int, precision: int = 0, device: int = 0):
        import torch

        from .solver import Solver

        self.mesh, self.parts = mesh, partition_mesh(mesh, nparts)
        self.solvers = [Solver(p.mesh, cfg, device=device, precision=precision) for p in self.parts]
        self.dev = torch.device(f"cuda:{device}")
        self.urec_dtype = torch.float32 if precision == 1 else torch.float64
        self.limiter = bool(cfg.get("useLimiter", False))
        for p, s in zip(self.parts, self.solvers):
            mask = np.zeros(p.mesh.n_cells, dtype=np.uint8)
            mask[: p.n_owned] = 1
            s._check(s.L.dndsg_set_owned(s.h, mask.ctypes.data_as(C.c_void_p)))
        # device index lists of every exchange
        self._lists = {}
        for pi, p in enumerate(self.parts):
            for q, idx in p.recv.items():
                self._lists[(pi, q)] = (torch.tensor(idx, device=self.dev),
                                        torch.tensor(self.parts[q].send[pi], device=self.dev))

    def set_u(self, u: np.ndarray):
        for p, s in zip(self.parts, self.solvers):
            s.set_u(np.ascontiguousarray(u[p.cells]))

    def get_u(self) -> np.ndarray:
        out = np.empty((self.mesh.n_cells, 4))
        for p, s in zip(self.parts, self.solvers):
            out[p.cells[: p.n_owned]] = s.get_u()[: p.n_owned]
        return out

    def exchange(self, what: int):
        """Ghost values from their owners: pack on the owner, unpack on the holder.  The pack and
        the unpack are ordered only by their stream: every part must run on one stream (the
        solvers here use the legacy default stream), which is checked."""
        import torch

        streams = {s.stream.value if s.stream else None for s in self.solvers}
        if len(streams) != 1:
            raise ValueError("PartitionedRun.exchange needs every part on one stream")

        w = 4 if what == 0 else 20
        for (pi, q), (recv, send) in self._lists.items():
            src, dst = self.solvers[q], self.solvers[pi]
            dt = torch.float64 if what == 0 else self.urec_dtype
            buf = torch.empty((len(recv), w), dtype=dt, device=self.dev)
            src._check(src.L.dndsg_halo_pack(src.h, what, C.c_void_p(send.data_ptr()), len(send),
                                             C.c_void_p(buf.data_ptr()), src.stream))
            dst._check(dst.L.dndsg_halo_unpack(dst.h, what, C.c_void_p(recv.data_ptr()), len(recv),
                                               C.c_void_p(buf.data_ptr()), dst.stream))

    def ssprk3_step(self, cfl: float, t_end: float = 1e300) -> float:
        dmins = []
        for s in self.solvers:
            d = C.c_double()
            s._check(s.L.dndsg_rk_dt(s.h, float(cfl), C.byref(d), s.stream))
            dmins.append(d.value)
        dt = max(0.0, min(min(dmins), t_end - self.solvers[0].time))
        for s in self.solvers:
            s._check(s.L.dndsg_rk_set_dt(s.h, dt, s.stream))
        for k in range(3):
            for s in self.solvers:
                s._check(s.L.dndsg_rk_vr(s.h, s.stream))
            self.exchange(1)
            if self.limiter:
                for s in self.solvers:
                    s._check(s.L.dndsg_rk_limit(s.h, s.stream))
                self.exchange(1)
            for s in self.solvers:
                s._check(s.L.dndsg_rk_stage(s.h, k, s.stream))
            self.exchange(0)
        for s in self.solvers:
            s._check(s.L.dndsg_rk_finish(s.h, s.stream))
        return dt

    def close(self):
        for s in self.solvers:
            s.close()


def halo_exchange(send: dict, recv: dict, group=None):
    """Point-to-point exchange of packed halo buffers between ranks: ``send[q]`` goes to rank q and
    ``recv[q]`` (preallocated, same length as what q sends) is filled from rank q.  One batch of
    paired send / receive operations, so that no ordering of the ranks can deadlock (NCCL for device
    buffers, gloo for host buffers)."""
    import torch.distributed as dist

    ops = []
    for q in sorted(set(send) | set(recv)):
        if q in send:
            ops.append(dist.P2POp(dist.isend, send[q], q, group))
        if q in recv:
            ops.append(dist.P2POp(dist.irecv, recv[q], q, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


class DistributedRun:
    """One part per rank (``torch.distributed`` initialised, rank r on GPU LOCAL_RANK): every rank
    partitions the mesh the same way and holds part ``rank``; ghosts travel by ``halo_exchange`` of
    the buffers that ``dndsg_halo_pack`` fills, dt is reduced by an all-reduce (MIN)."""

    def __init__(self, mesh: M.Mesh, cfg: dict, precision: int = 0, device: int = 0):
        import torch
        import torch.distributed as dist

        from .solver import Solver

        self.rank, world = dist.get_rank(), dist.get_world_size()
        self.mesh, self.parts = mesh, partition_mesh(mesh, world)
        self.part = self.parts[self.rank]
        self.s = Solver(self.part.mesh, cfg, device=device, precision=precision)
        self.dev = torch.device(f"cuda:{device}")
        self.urec_dtype = torch.float32 if precision == 1 else torch.float64
        self.limiter = bool(cfg.get("useLimiter", False))
        mask = np.zeros(self.part.mesh.n_cells, dtype=np.uint8)
        mask[: self.part.n_owned] = 1
        self.s._check(self.s.L.dndsg_set_owned(self.s.h, mask.ctypes.data_as(C.c_void_p)))
        self.send_idx = {q: torch.tensor(v, device=self.dev) for q, v in self.part.send.items()}
        self.recv_idx = {q: torch.tensor(v, device=self.dev) for q, v in self.part.recv.items()}

    def set_u(self, u: np.ndarray):
        self.s.set_u(np.ascontiguousarray(u[self.part.cells]))

    def owned_u(self) -> np.ndarray:
        return self.s.get_u()[: self.part.n_owned]

    def exchange(self, what: int):
        import torch

        s, w = self.s, 4 if what == 0 else 20
        dt = torch.float64 if what == 0 else self.urec_dtype
        send, recv = {}, {}
        for q, idx in self.send_idx.items():
            send[q] = torch.empty((len(idx), w), dtype=dt, device=self.dev)
            s._check(s.L.dndsg_halo_pack(s.h, what, C.c_void_p(idx.data_ptr()), len(idx),
                                         C.c_void_p(send[q].data_ptr()), s.stream))
        for q, idx in self.recv_idx.items():
            recv[q] = torch.empty((len(idx), w), dtype=dt, device=self.dev)
        torch.cuda.synchronize(self.dev)
        halo_exchange(send, recv)
        for q, idx in self.recv_idx.items():
            s._check(s.L.dndsg_halo_unpack(s.h, what, C.c_void_p(idx.data_ptr()), len(idx),
                                           C.c_void_p(recv[q].data_ptr()), s.stream))

    def ssprk3_step(self, cfl: float, t_end: float = 1e300) -> float:
        import torch
        import torch.distributed as dist

        s = self.s
        d = C.c_double()
        s._check(s.L.dndsg_rk_dt(s.h, float(cfl), C.byref(d), s.stream))
        dmin = torch.tensor([d.value], dtype=torch.float64, device=self.dev)
        dist.all_reduce(dmin, op=dist.ReduceOp.MIN)
        dt = max(0.0, min(float(dmin.item()), t_end - s.time))
        s._check(s.L.dndsg_rk_set_dt(s.h, dt, s.stream))
        for k in range(3):
            s._check(s.L.dndsg_rk_vr(s.h, s.stream))
            self.exchange(1)
            if self.limiter:
                s._check(s.L.dndsg_rk_limit(s.h, s.stream))
                self.exchange(1)
            s._check(s.L.dndsg_rk_stage(s.h, k, s.stream))
            self.exchange(0)
        s._check(s.L.dndsg_rk_finish(s.h, s.stream))
        return dt
