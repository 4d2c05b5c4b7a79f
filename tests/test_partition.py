"""Partitioned runs (the reference's MPI domain decomposition with a one-cell ghost layer): the
partitioner's ownership, ghost and exchange lists, and on the GPU several parts of one mesh,
exchanging ghost values through the C ABI's halo pack / unpack, reproduce the whole-mesh SSP-RK3
steps on every owned cell."""
import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import partition as P
from dnds_b200 import settings as S


@pytest.mark.parametrize("mesh", [M.vortex_mesh(12, True, jitter=0.2), M.riemann_mesh(16),
                                  M.naca0012_cmesh(32, 16, 16, first=2e-3, far=10.0, wall_bc=M.BC_WALL_EULER)],
                         ids=["periodic", "riemann", "naca"])
def test_partition_owns_every_cell_once_and_pairs_the_ghosts(mesh):
    parts = P.partition_mesh(mesh, 4)
    owned = np.concatenate([p.cells[: p.n_owned] for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(mesh.n_cells))
    L, R = mesh.face_cells[:, 0], mesh.face_cells[:, 1]
    for pi, p in enumerate(parts):
        p.mesh.validate()  # every local cell closed: one face per edge
        # an owned cell keeps its neighbours, in global ids
        loc = p.cells
        pl, pr = p.mesh.face_cells[:, 0], p.mesh.face_cells[:, 1]
        for c in range(p.n_owned):
            g = loc[c]
            nb_glob = sorted(np.concatenate([R[(L == g) & (R >= 0)], L[R == g]]))
            nb_loc = sorted(loc[np.concatenate([pr[(pl == c) & (pr >= 0)], pl[pr == c]])])
            assert nb_glob == nb_loc
        # the ghosts are exactly the cells across an owned cell's faces, each received from its owner
        ghosts = loc[p.n_owned:]
        recv = np.concatenate([loc[idx] for idx in p.recv.values()]) if p.recv else np.zeros(0, int)
        assert np.array_equal(np.sort(recv), np.sort(ghosts))
        for q, idx in p.recv.items():
            assert np.array_equal(loc[idx], parts[q].cells[parts[q].send[pi]])


@pytest.mark.gpu
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_vortex_matches_whole_mesh(nparts):
    from dnds_b200.solver import Solver

    m, cfg = M.vortex_mesh(32, True, jitter=0.2), S.preset("vortex")
    u0 = G.isentropic_vortex(m)
    whole = Solver(m, cfg, precision=0)
    whole.set_u(u0)
    run = P.PartitionedRun(m, cfg, nparts, precision=0)
    run.set_u(u0)
    for _ in range(3):
        whole.ssprk3_step(0.5)
        run.ssprk3_step(0.5)
    ref = whole.get_u()
    assert np.abs(run.get_u() - ref).max() < 1e-13 * np.abs(ref).max()
    assert abs(run.solvers[0].time - whole.time) < 1e-15


@pytest.mark.gpu
def test_partitioned_riemann_with_limiter_matches_whole_mesh():
    """The limiter reads the neighbours' coefficients: the ghosts are refreshed after the sweep and
    again after the limiter.  HLLC, 2-D Riemann far field, FP32 bulk."""
    from dnds_b200.solver import Solver

    m, cfg = M.riemann_mesh(32), S.preset("riemann")
    u0 = G.quadrant_states(m, S.RIEMANN_2D_STATES)
    whole = Solver(m, cfg, precision=1)
    whole.set_u(u0)
    run = P.PartitionedRun(m, cfg, 4, precision=1)
    run.set_u(u0)
    for _ in range(3):
        whole.ssprk3_step(0.4, 0.3)
        run.ssprk3_step(0.4, 0.3)
    ref = whole.get_u()
    assert np.abs(run.get_u() - ref).max() < 1e-12 * np.abs(ref).max()


def _exchange_worker(rank, world, port, out):
    import datetime
    import os

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    parts = P.partition_mesh(M.vortex_mesh(12, True, jitter=0.2), world)
    part = parts[rank]
    # what travels: the global ids of the cells (two columns, as a packed [n][w] halo buffer)
    send = {q: torch.tensor(np.repeat(part.cells[idx][:, None], 2, 1), dtype=torch.float64)
            for q, idx in part.send.items()}
    recv = {q: torch.empty((len(idx), 2), dtype=torch.float64) for q, idx in part.recv.items()}
    P.halo_exchange(send, recv)
    ok = all(np.array_equal(recv[q].numpy()[:, 0], part.cells[idx]) for q, idx in part.recv.items())
    out[rank] = (ok, sorted(part.recv))
    dist.barrier()
    dist.destroy_process_group()


def test_halo_exchange_between_gloo_ranks():
    """The rank-to-rank protocol of a distributed run: 3 gloo ranks, each holding one part of the
    periodic vortex mesh, swap packed halo buffers in one batch of paired sends and receives; every
    ghost receives its owner's values (here its global id), and the periodic wrap pairs the first
    and the last part."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_exchange_worker, args=(3, port, out), nprocs=3, join=True)
    for r in range(3):
        ok, peers = out[r]
        assert ok and peers == sorted({0, 1, 2} - {r})


@pytest.mark.gpu
def test_distributed_run_on_one_rank_matches_whole_mesh():
    """The distributed driver with one NCCL rank (no ghosts; the dt all-reduce and the stage-level
    calls) against the whole-mesh step."""
    import datetime
    import os
    import socket

    import torch.distributed as dist

    from dnds_b200.solver import Solver

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        m, cfg = M.vortex_mesh(16, True, jitter=0.2), S.preset("vortex")
        u0 = G.isentropic_vortex(m)
        run = P.DistributedRun(m, cfg, precision=0)
        run.set_u(u0)
        whole = Solver(m, cfg, precision=0)
        whole.set_u(u0)
        for _ in range(2):
            run.ssprk3_step(0.5)
            whole.ssprk3_step(0.5)
        assert np.abs(run.owned_u() - whole.get_u()).max() < 1e-14
    finally:
        dist.destroy_process_group()
