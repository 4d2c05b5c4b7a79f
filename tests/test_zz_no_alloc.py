"""The allocation-free RHS entry point (dndsg_eval_rhs_noalloc) against the
regular one (dndsg_eval_rhs), through the C ABI on the GPU.

It serves callers that cannot allocate device memory when they need a
residual (real-time loops that cannot take cudaMalloc's implicit device
synchronisation, hosts that forbid allocations after start-up).  This file
is collected last so that a run stopping at the first failure has already run
every other test; it passes alone in a fresh process as well.
"""
import numpy as np
import pytest

from dnds_b200 import geometry as G
from dnds_b200 import mesh as M
from dnds_b200 import settings as S

pytestmark = pytest.mark.gpu


def _case(preset):
    """A mesh inside the scratch limit and its initial state: the periodic vortex (Roe) or the
    2-D Riemann problem (HLLC, time-dependent far field)."""
    if preset == "vortex":
        m = M.vortex_mesh(64, True, jitter=0.2, seed=1234)  # 12,288 faces
        return m, G.isentropic_vortex(m)
    m = M.riemann_mesh(64)  # 12,416 faces
    return m, G.quadrant_states(m, S.RIEMANN_2D_STATES)


@pytest.mark.parametrize("preset", ["vortex", "riemann"])
@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 1e-13)])
def test_noalloc_rhs_matches_eval_rhs_twice(preset, precision, tol):
    import torch

    from dnds_b200.solver import BUF_U, BUF_UREC, Solver

    m, u0 = _case(preset)
    s = Solver(m, S.preset(preset), precision=precision)
    s.set_u(u0)
    s.ReconstructionJacobiStep(3)
    s.EvaluateDt(0.4)
    t = 0.01
    ref = s.EvaluateRHS(t)
    u_ptr, _ = s.device_buffer(BUF_U)
    r_ptr, _ = s.device_buffer(BUF_UREC)
    out = torch.full((m.n_cells, 4), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        s.EvaluateRHS_noalloc(u_ptr, r_ptr, out.data_ptr(), t)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    s.close()


def test_noalloc_rejects_meshes_beyond_the_limit():
    import torch

    from dnds_b200.solver import BUF_U, BUF_UREC, DndsgError, Solver

    m = M.vortex_mesh(300, True)  # 270,000 faces > 262,144
    s = Solver(m, S.preset("vortex"), precision=0)
    u_ptr, _ = s.device_buffer(BUF_U)
    r_ptr, _ = s.device_buffer(BUF_UREC)
    out = torch.empty((m.n_cells, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(DndsgError, match="scratch limit"):
        s.EvaluateRHS_noalloc(u_ptr, r_ptr, out.data_ptr(), 0.0)
    s.close()


@pytest.mark.parametrize("which", ["u", "urec", "rhs"])
def test_noalloc_rejects_pointers_not_16_byte_aligned(which):
    """An 8-byte-aligned double pointer (an offset into a larger array) is refused on the host,
    before any launch: the kernels move these arrays in 16-byte vectors."""
    import torch

    from dnds_b200.solver import BUF_U, BUF_UREC, DndsgError, Solver

    m = M.vortex_mesh(16, True, jitter=0.2, seed=1234)
    s = Solver(m, S.preset("vortex"), precision=0)
    s.set_u(G.isentropic_vortex(m))
    u_ptr, _ = s.device_buffer(BUF_U)
    r_ptr, _ = s.device_buffer(BUF_UREC)
    big = torch.zeros((m.n_cells + 1) * 4, dtype=torch.float64, device="cuda")
    ptrs = {"u": u_ptr, "urec": r_ptr, "rhs": big.data_ptr()}
    ptrs[which] += 8
    with pytest.raises(DndsgError, match="16-byte aligned"):
        s.EvaluateRHS_noalloc(ptrs["u"], ptrs["urec"], ptrs["rhs"], 0.0)
    torch.cuda.synchronize()
    assert bool(torch.all(big == 0))  # nothing was launched
    s.close()
