"""The C++ route of the boundary: include/dndsg_shim.hpp, the header-only shim
with the reference's class and method names (EulerEvaluator, VRFiniteVolume2D,
the ODE drivers) over the C ABI.

CPU: every shim class and method compiles and links against libdndsg.so.
GPU: tests/shim_driver.cpp, a C++ program written against the shim, runs
ReconstructionJacobiStep -> EvaluateDt -> EvaluateRHS -> two
ExplicitSSPRK3GPU::Step calls on the jittered periodic vortex mesh of the
golden fixture and matches the oracle's outputs (FP64: 1e-11 for single
evaluations, 1e-12 after two steps, as the Python-route parity tests).
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _compile(src, exe):
    from dnds_b200 import build

    build.build()
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        build.LIB, f"-Wl,-rpath,{os.path.dirname(build.LIB)}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_shim_header_compiles(tmp_path):
    src = tmp_path / "use_shim.cpp"
    src.write_text('#include "dndsg_shim.hpp"\n'
                   "int main(){ dndsg_mesh_desc m{}; dndsg_settings s{}; (void)m; (void)s;\n"
                   "  if (false) { dndsg::Context c(m, s); dndsg::VRFiniteVolume2DGPU vr(c); dndsg::EulerEvaluatorGPU ev(c);\n"
                   "    std::vector<double> r; vr.ReconstructionJacobiStep(); ev.EvaluateRHS(r, 0.0);\n"
                   "    ev.SetLUSGSOrder(1); ev.SetLUSGSParts(nullptr, 1); ev.LUSGSMatrixInit(1e100, 1.0); ev.UpdateLUSGSForward(1.0, nullptr, nullptr);\n"
                   "    ev.UpdateLUSGSBackward(1.0, nullptr, nullptr); dndsg::ImplicitSteadyGPU st(c);\n"
                   "    st.Step(100.0, 1e-8, 10, 1e100, 1, false, &r); ev.LUSGSMatrixVec(1.0, nullptr, nullptr);\n"
                   "    dndsg::ImplicitDualTimeStepGPU ode(c, 1, 2); ode.Step(0.1, 0.0, 100.0, 10, 1e-3, 1, false, 2, 10, 2);\n"
                   "    dndsg::GMRES_LeftPreconditionedGPU g(c, 10); g.solve(1.0, nullptr, nullptr, 2);\n"
                   "    dndsg::ExplicitSSPRK3GPU rk(c); rk.Step(0.5); rk.Steps(0.5, 10, 2.0);\n"
                   "    vr.ReconstructionWBAPLimitFacialV2(true); dndsg_steady_settings ss{}; st.Run(ss, &r, &r); } return 0; }\n")
    _compile(src, tmp_path / "a.out")


def test_shim_driver_compiles(tmp_path):
    _compile(os.path.join(ROOT, "tests", "shim_driver.cpp"), tmp_path / "shim_driver")


def _write_input(path, m, settings, u0, cfl, t_rhs):
    with open(path, "wb") as f:
        np.array([m.n_nodes, m.n_cells, m.n_faces], dtype=np.int64).tofile(f)
        np.ascontiguousarray(m.node_xy, dtype=np.float64).tofile(f)
        for a in (m.cell_nodes, m.face_nodes, m.face_cells, m.face_bc):
            np.ascontiguousarray(a, dtype=np.int32).tofile(f)
        np.ascontiguousarray(m.face_shift, dtype=np.float64).tofile(f)
        f.write(bytes(settings))
        np.ascontiguousarray(u0, dtype=np.float64).tofile(f)
        np.array([cfl, t_rhs], dtype=np.float64).tofile(f)


@pytest.mark.gpu
def test_shim_program_matches_golden(tmp_path):
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S

    m = M.vortex_mesh(8, True, jitter=0.2, seed=1234)  # the mesh of vortex_tri8_jitter.npz
    ref = np.load(os.path.join(GOLDEN, "vortex_tri8_jitter.npz"))
    st = S.make_settings(S.preset("vortex", useLimiter=False))
    st.sor_instead = 0
    st.precision = 0
    exe = tmp_path / "shim_driver"
    _compile(os.path.join(ROOT, "tests", "shim_driver.cpp"), exe)
    _write_input(tmp_path / "in.bin", m, st, ref["u0"], 0.5, 0.1)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    n = m.n_cells
    assert out.size == 1 + n + 4 * n + 4 * n + 1
    dtmin, dt, rhs, u2, t2 = out[0], out[1:1 + n], out[1 + n:1 + 5 * n], out[1 + 5 * n:1 + 9 * n], out[-1]

    def rel(a, b):
        return np.abs(a - b).max() / np.abs(b).max()

    assert abs(dtmin - float(ref["dtmin"])) < 1e-13 * float(ref["dtmin"])
    assert rel(dt, ref["dt"]) < 1e-13
    assert rel(rhs.reshape(n, 4), ref["rhs"]) < 1e-11
    assert rel(u2.reshape(n, 4), ref["u_rk2"]) < 1e-12
    assert abs(t2 - float(ref["t_rk2"])) < 1e-14
