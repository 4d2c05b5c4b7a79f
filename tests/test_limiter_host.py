"""The limiter's building blocks on the host (tests/limiter_host_check.cpp compiles dndsg_limiter.cuh as
plain C++; on the host the FP32 quotients and square roots are the IEEE ones, so this checks the FP32
algebra, and the GPU parity tests check the hardware approximations on top).

char_rows: the left and right characteristic matrices at a face's mean state (DNDS_FV_EulerSolver.hpp:
749-795, Gas::EulerGasLeft/RightEigenVector) are inverses, R L = I, in FP64 and in the FP32 branch that
works with reciprocals of rho, a^2 and gamma - 1; the FP32 rows agree with the FP64 ones.
wbap_biway: the FP32 version (the ratio capped at 1e9 so that its fourth power stays finite) agrees
with the FP64 one relative to |u1|, over ratios from 1e-9 to past the cap."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    so = tmp_path_factory.mktemp("lim") / "limiter_host_check.so"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "dnds_b200", "csrc"),
                        os.path.join(ROOT, "tests", "limiter_host_check.cpp"), "-o", str(so)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(str(so))
    L.char_rows_check.restype = None
    L.char_rows_check.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.biway_check.restype = C.c_double
    L.biway_check.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double]
    return L


def _states(rng, n, gamma):
    """n pairs of conservative states: density 0.1-2, velocities N(0, 1.5), pressure 0.05-2."""
    rho = rng.uniform(0.1, 2.0, (n, 2))
    u, v = rng.normal(0, 1.5, (n, 2)), rng.normal(0, 1.5, (n, 2))
    p = rng.uniform(0.05, 2.0, (n, 2))
    E = p / (gamma - 1) + 0.5 * rho * (u * u + v * v)
    return np.ascontiguousarray(np.stack([rho[:, 0], rho[:, 0] * u[:, 0], rho[:, 0] * v[:, 0], E[:, 0],
                                          rho[:, 1], rho[:, 1] * u[:, 1], rho[:, 1] * v[:, 1], E[:, 1]], 1))


@pytest.mark.parametrize("gamma", [1.4, 5.0 / 3.0])
def test_characteristic_matrices_are_inverses(lib, gamma):
    rng = np.random.default_rng(3)
    n = 20000
    S = _states(rng, n, gamma)
    th = rng.uniform(0, 2 * np.pi, n)
    N = np.ascontiguousarray(np.stack([np.cos(th), np.sin(th)], 1))
    e64, e32, d32 = C.c_double(), C.c_double(), C.c_double()
    lib.char_rows_check(n, S.ctypes.data, N.ctypes.data, gamma, C.addressof(e64), C.addressof(e32),
                        C.addressof(d32))
    # measured (gamma 1.4): 1.5e-14, 9.2e-6 and 3.3e-6
    assert e64.value < 1e-12, e64.value
    assert e32.value < 5e-5, e32.value
    assert d32.value < 2e-5, d32.value


@pytest.mark.parametrize("n_std", [1.0, 10.0])
def test_biway_fp32_matches_fp64(lib, n_std):
    rng = np.random.default_rng(4)
    n = 20000
    u1 = np.ascontiguousarray(rng.normal(0, 1, n) * 10 ** rng.uniform(-6, 3, n))
    u2 = np.ascontiguousarray(rng.normal(0, 1, n) * 10 ** rng.uniform(-8, 3, n))
    assert (np.abs(u1) / (np.abs(u2) + 1e-12)).max() > 1e9  # ratios past the FP32 cap are covered
    # measured about 2.3e-7 of |u1|
    assert lib.biway_check(n, u1.ctypes.data, u2.ctypes.data, n_std) < 2e-6
