"""Host-side logic of the multi-GPU bench (independent replicas, one per rank),
exercised with 2 gloo ranks on the CPU: the job is timed by the slowest rank
and the throughput is summed over ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    local_ms = [10.0, 25.0][rank]
    ms = bench.max_over_ranks(local_ms)
    out[rank] = (ms, bench.replica_throughput(1000, 4, ms, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_aggregation():
    import torch.multiprocessing as mp

    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    for r in (0, 1):
        ms, v = out[r]
        assert ms == 25.0
        assert v == pytest.approx(1000 * 3 * 4 / 0.025 * 2)


def test_single_process_identity():
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(10, 2, 1000.0, 1) == pytest.approx(60.0)


def test_shim_header_compiles(tmp_path):
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "use_shim.cpp"
    src.write_text('#include "dndsg_shim.hpp"\n'
                   "int main(){ dndsg_mesh_desc m{}; dndsg_settings s{}; (void)m; (void)s;\n"
                   "  if (false) { dndsg::Context c(m, s); dndsg::VRFiniteVolume2DGPU vr(c); dndsg::EulerEvaluatorGPU ev(c);\n"
                   "    std::vector<double> r; vr.ReconstructionJacobiStep(); ev.EvaluateRHS(r, 0.0);\n"
                   "    ev.SetLUSGSOrder(1); ev.LUSGSMatrixInit(1e100, 1.0); ev.UpdateLUSGSForward(1.0, nullptr, nullptr);\n"
                   "    ev.UpdateLUSGSBackward(1.0, nullptr, nullptr); dndsg::ImplicitSteadyGPU st(c);\n"
                   "    st.Step(100.0, 1e-8, 10, 1e100, 1, false, &r); ev.LUSGSMatrixVec(1.0, nullptr, nullptr);\n"
                   "    dndsg::ImplicitDualTimeStepGPU ode(c, 1, 2); ode.Step(0.1, 0.0, 100.0, 10, 1e-3, 1, false, 2, 10, 2);\n"
                   "    dndsg::GMRES_LeftPreconditionedGPU g(c, 10); g.solve(1.0, nullptr, nullptr, 2);\n"
                   "    dndsg::ExplicitSSPRK3GPU rk(c); rk.Step(0.5); rk.Steps(0.5, 10, 2.0); } return 0; }\n")
    from dnds_b200 import build

    build.build()
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "include"), str(src), "-o", str(tmp_path / "a.out"),
                        build.LIB, f"-Wl,-rpath,{os.path.dirname(build.LIB)}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
