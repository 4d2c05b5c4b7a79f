"""Host-side mirror of DNDS's solver/evaluator call surface over the C ABI.

``Solver`` owns one ``dndsg_ctx``: the mesh, the FP64 VR setup and the
resident state on one GPU.  Its methods carry the reference's member-function
names and argument meanings:

* ``ReconstructionJacobiStep``      VRFiniteVolume2D, DNDS_FV_VR.hpp:1474-1713
* ``ReconstructionWBAPLimitFacialV3`` VRFiniteVolume2D, DNDS_FV_VR.hpp:2053-2329
* ``EvaluateDt``                    EulerEvaluator, DNDS_FV_EulerEvaluator.cpp:14-183
* ``EvaluateRHS``                   EulerEvaluator, DNDS_FV_EulerEvaluator.cpp:198-640
* ``EvaluateResidual``              EulerEvaluator, DNDS_FV_EulerEvaluator.cpp:1557-1592
* ``ssprk3_step``                   ExplicitSSPRK3LocalDt::Step with the EulerSolver stage body

Where the reference aborts (``DNDS_assert``), these raise ``DndsgError``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh
from .settings import make_settings

BUF_U, BUF_UREC, BUF_RHS, BUF_DT, BUF_SA_U, BUF_SA_UREC = 0, 1, 2, 3, 4, 5


class DndsgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dndsg error {code}: {msg}")
        self.code = code


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Solver:
    def __init__(self, mesh: Mesh, cfg: dict, device: int = 0, precision: int | None = None, stream=None):
        self.L = _lib.lib()
        s = make_settings(cfg)
        if precision is not None:
            s.precision = int(precision)
        s.sor_instead = 0
        self.settings = s
        self.mesh = mesh
        self.stream = C.c_void_p(stream) if stream else None
        self._keep = [mesh.node_xy, mesh.cell_nodes, mesh.face_nodes, mesh.face_cells, mesh.face_bc, mesh.face_shift]
        md = _lib.MeshDesc(mesh.n_nodes, mesh.n_cells, mesh.n_faces, *[_p(a) for a in self._keep])
        h = C.c_void_p()
        rc = self.L.dndsg_create(C.byref(md), C.byref(s), device, C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.dndsg_last_error(h).decode() if h else "no context"
            if h:
                self.L.dndsg_destroy(h)
            self.h = None
            raise DndsgError(rc, msg)
        self.N = mesh.n_cells
        self.F = mesh.n_faces
        self.nv = int(s.nvars)

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "h", None):
            self.L.dndsg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise DndsgError(rc, self.L.dndsg_last_error(self.h).decode())

    # ------------------------------------------------------------------ state
    def set_u(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.N, self.nv)
        self._check(self.L.dndsg_set_u(self.h, _p(u), self.stream))

    def get_u(self, out: np.ndarray | None = None) -> np.ndarray:
        u = np.empty((self.N, self.nv)) if out is None else out
        assert u.dtype == np.float64 and u.flags.c_contiguous and u.size == self.N * self.nv
        self._check(self.L.dndsg_get_u(self.h, _p(u), self.stream))
        return u

    def set_urec(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(self.N, 5, self.nv)
        self._check(self.L.dndsg_set_urec(self.h, _p(r), self.stream))

    def get_urec(self) -> np.ndarray:
        r = np.empty((self.N, 5, self.nv))
        self._check(self.L.dndsg_get_urec(self.h, _p(r), self.stream))
        return r

    def get_dt(self) -> np.ndarray:
        d = np.empty(self.N)
        self._check(self.L.dndsg_get_dt(self.h, _p(d), self.stream))
        return d

    @property
    def time(self) -> float:
        t = C.c_double()
        self._check(self.L.dndsg_get_time(self.h, C.byref(t), self.stream))
        return t.value

    @time.setter
    def time(self, t: float):
        self._check(self.L.dndsg_set_time(self.h, float(t), self.stream))

    def device_buffer(self, which: int):
        p = C.c_void_p()
        n = C.c_int64()
        self._check(self.L.dndsg_device_buffer(self.h, which, C.byref(p), C.byref(n)))
        return p.value, n.value

    # ------------------------------------------------------------------ reference-named operations
    def ReconstructionJacobiStep(self, nsweeps: int = 1, with_increment: bool = False):
        inc = C.c_double()
        self._check(self.L.dndsg_vr_jacobi_step(self.h, nsweeps, C.byref(inc) if with_increment else None,
                                                self.stream))
        return inc.value if with_increment else None

    def ReconstructionWBAPLimitFacialV3(self, if_all: bool = False, indicator: bool = False):
        ind = np.empty(self.N) if indicator else None
        self._check(self.L.dndsg_limiter_wbap(self.h, int(if_all), _p(ind) if indicator else None, self.stream))
        return ind

    def ReconstructionWBAPLimitFacialV2(self, if_all: bool = False, indicator: bool = False):
        """3WBAP limiting (DNDS_FV_VR.hpp:1749-2047) of the resident coefficients in place."""
        ind = np.empty(self.N) if indicator else None
        self._check(self.L.dndsg_limiter_wbap_v2(self.h, int(if_all), _p(ind) if indicator else None, self.stream))
        return ind

    def EvaluateDt(self, cfl: float, max_dt: float = 1e100, use_local_dt: bool = False) -> float:
        dmin = C.c_double()
        self._check(self.L.dndsg_eval_dt(self.h, cfl, max_dt, int(use_local_dt), C.byref(dmin), self.stream))
        return dmin.value

    def EvaluateRHS(self, t: float = 0.0, copy: bool = True):
        rhs = np.empty((self.N, self.nv)) if copy else None
        self._check(self.L.dndsg_eval_rhs(self.h, float(t), _p(rhs) if copy else None, self.stream))
        return rhs

    def EvaluateRHS_noalloc(self, u_ptr: int, urec_ptr: int, rhs_ptr: int, t: float = 0.0):
        """EvaluateRHS from caller-owned device arrays without any device allocation
        (dndsg_eval_rhs_noalloc): for callers that cannot allocate device memory
        when they need a residual.  Meshes are limited to DNDSG_NOALLOC_MAX_FACES
        faces; concurrent calls on the GPU share one scratch array and race."""
        self._check(self.L.dndsg_eval_rhs_noalloc(self.h, C.c_void_p(u_ptr), C.c_void_p(urec_ptr),
                                                  C.c_void_p(rhs_ptr), float(t), self.stream))

    def EvaluateResidual(self, p: int = 1, vol_wise: bool = False) -> np.ndarray:
        out = np.empty(self.nv)
        self._check(self.L.dndsg_residual(self.h, int(p), int(vol_wise), _p(out), self.stream))
        return out

    def ssprk3_step(self, cfl: float, t_end: float = 1e300):
        self._check(self.L.dndsg_ssprk3_step(self.h, cfl, t_end, self.stream))

    def ssprk3_steps(self, cfl: float, n: int, t_end: float = 1e300):
        """n SSP-RK3 steps, pairs of them replayed from a CUDA graph (dndsg_ssprk3_steps)."""
        self._check(self.L.dndsg_ssprk3_steps(self.h, cfl, t_end, int(n), self.stream))

    # ------------------------------------------------------------------ implicit steady path
    def lusgs_colours(self):
        """(colour of every cell, number of colours) of the LU-SGS colouring."""
        col = np.empty(self.N, dtype=np.int32)
        n = C.c_int()
        self._check(self.L.dndsg_lusgs_colours(self.h, _p(col), C.byref(n)))
        return col, n.value

    def lusgs_set_order(self, mode: int = 0, scan2cell=None) -> int:
        """LU-SGS schedule: 0 colour batches; 1 the sequential sweep in scan2cell (None: natural
        cell order), level-scheduled.  Returns the forward plus backward batches per iteration."""
        nb = C.c_int()
        o = None if scan2cell is None else np.ascontiguousarray(scan2cell, dtype=np.int64)
        self._check(self.L.dndsg_lusgs_set_order(self.h, int(mode), _p(o) if o is not None else None, C.byref(nb)))
        return nb.value

    def lusgs_set_parts(self, part=None, n_parts: int = 1) -> int:
        """Partitioned scan-order sweeps, as the reference on n_parts ranks: part [N] in [0, n_parts)
        (None: one part).  Switches to the scan-order schedule (the order last given to
        lusgs_set_order, natural if none).  Returns the most levels of one part, forward plus backward."""
        nb = C.c_int()
        self._parts = None if part is None else np.ascontiguousarray(part, dtype=np.int32)
        self._check(self.L.dndsg_lusgs_set_parts(self.h, _p(self._parts) if self._parts is not None else None,
                                                 int(n_parts), C.byref(nb)))
        return nb.value

    def LUSGSMatrixInit(self, dt: float = 1e100, alpha_diag: float = 1.0):
        """LUSGSMatrixInit (DNDS_FV_EulerEvaluator.cpp:995-1047) from the last EvaluateDt."""
        self._check(self.L.dndsg_lusgs_matrix_init(self.h, float(dt), float(alpha_diag), self.stream))

    def UpdateLUSGSForward(self, alpha_diag: float, rhs_ptr: int, inc_ptr: int):
        """In place on the device array inc [N][4] (DNDS_FV_EulerEvaluator.cpp:1149-1276)."""
        self._check(self.L.dndsg_lusgs_forward(self.h, float(alpha_diag), C.c_void_p(rhs_ptr), C.c_void_p(inc_ptr),
                                               self.stream))

    def UpdateLUSGSBackward(self, alpha_diag: float, rhs_ptr: int, inc_ptr: int):
        """In place on the device array inc [N][4] (DNDS_FV_EulerEvaluator.cpp:1285-1357)."""
        self._check(self.L.dndsg_lusgs_backward(self.h, float(alpha_diag), C.c_void_p(rhs_ptr), C.c_void_p(inc_ptr),
                                                self.stream))

    def bdf_begin(self):
        self._check(self.L.dndsg_bdf_begin(self.h, self.stream))

    def implicit_iteration(self, cfl: float, dt: float = 1e100, alpha_diag: float = 1.0, n_rec: int = 1,
                           vol_wise: bool = False, t: float = 0.0):
        """One first-order BDF pseudo-time iteration; returns (L1 norm of the increment, wall flux)."""
        res = np.empty(self.nv)
        wf = np.empty(self.nv)
        self._check(self.L.dndsg_implicit_iteration(self.h, float(cfl), float(dt), float(alpha_diag), int(n_rec),
                                                    int(vol_wise), float(t), _p(res), _p(wf), self.stream))
        return res, wf

    def dual_reset(self):
        """A fresh dual-time integrator: the BDF history is forgotten."""
        self._check(self.L.dndsg_dual_reset(self.h))

    def dual_step(self, dt: float, t: float = 0.0, scheme: str = "sdirk4", bdf_order: int = 2, cfl: float = 100.0,
                  max_iter: int = 10, threshold: float = 1e-100, n_rec: int = 1, vol_wise: bool = False,
                  gmres_code: int = 0, n_gmres_space: int = 10, n_gmres_iter: int = 2):
        """One physical step of the reference's implicit driver: ImplicitSDIRK4DualTimeStep
        (scheme "sdirk4", odeCode 0) or ImplicitBDFDualTimeStep of order bdf_order (scheme "bdf",
        odeCode 1), DNDS_ODE.hpp:269-497; fsolve by LU-SGS (gmres_code 0), GMRES over LU-SGS (1), or
        LU-SGS then GMRES (2).  Returns (internal iterations per stage, last fstop ratios)."""
        from ._lib import DualSettings

        d = DualSettings(scheme={"sdirk4": 0, "bdf": 1}[scheme], bdf_order=int(bdf_order), cfl=float(cfl),
                         max_iter=int(max_iter), threshold=float(threshold), n_rec=int(n_rec),
                         vol_wise=int(vol_wise), gmres_code=int(gmres_code), n_gmres_space=int(n_gmres_space),
                         n_gmres_iter=int(n_gmres_iter))
        its = np.zeros(3, dtype=np.int32)
        res = np.zeros(self.nv)
        self._check(self.L.dndsg_dual_step(self.h, C.byref(d), float(dt), float(t), _p(its), _p(res), self.stream))
        return its, res

    def LUSGSMatrixVec(self, alpha_diag: float, x_ptr: int, ax_ptr: int):
        """LUSGSMatrixVec (DNDS_FV_EulerEvaluator.cpp:1062-1143) on device arrays [N][4], with the
        diagonal of the last LUSGSMatrixInit."""
        self._check(self.L.dndsg_lusgs_matvec(self.h, float(alpha_diag), C.c_void_p(x_ptr), C.c_void_p(ax_ptr),
                                              self.stream))

    def gmres_lusgs(self, alpha_diag: float, n_space: int, n_restart: int, b_ptr: int, x_ptr: int):
        """GMRES_LeftPreconditioned over LUSGSMatrixVec with the LU-SGS sweeps as preconditioner, on
        device arrays [N][4]; x holds the initial guess and receives the result."""
        self._check(self.L.dndsg_gmres_lusgs(self.h, float(alpha_diag), int(n_space), int(n_restart),
                                             C.c_void_p(b_ptr), C.c_void_p(x_ptr), self.stream))

    def steady_run(self, cfl: float = 100.0, threshold: float = 1e-8, max_iter: int = 10000, dt: float = 1e100,
                   cfl_ramp_start: int = 10**9, cfl_ramp_length: int = 0, cfl_ramp_end: float | None = None,
                   gmres_code: int = 0, n_gmres_space: int = 10, n_gmres_iter: int = 2, n_rec: int = 1,
                   vol_wise: bool = False, history: bool = False):
        """The steady internal loop of EulerSolver with ifSteadyQuit in one C call (dndsg_steady_solve):
        first-order BDF pseudo time with the CFL ramp of fstop and fsolve per gmresCode, until the
        density increment ratio drops below threshold.  Returns (iterations, fstop ratios, wall flux,
        density ratio per iteration or None)."""
        from ._lib import SteadySettings

        st = SteadySettings(cfl=float(cfl), cfl_ramp_end=float(cfl if cfl_ramp_end is None else cfl_ramp_end),
                            cfl_ramp_start=int(cfl_ramp_start), cfl_ramp_length=int(cfl_ramp_length),
                            max_iter=int(max_iter), threshold=float(threshold), dt=float(dt), n_rec=int(n_rec),
                            vol_wise=int(vol_wise), gmres_code=int(gmres_code), n_gmres_space=int(n_gmres_space),
                            n_gmres_iter=int(n_gmres_iter))
        it = C.c_int()
        rel = np.zeros(self.nv)
        wf = np.zeros(self.nv)
        hist = np.zeros(max_iter) if history else None
        self._check(self.L.dndsg_steady_solve(self.h, C.byref(st), C.byref(it), _p(rel), _p(wf),
                                              _p(hist) if history else None, self.stream))
        return it.value, rel, wf, (hist[: it.value] if history else None)

    def steady_solve(self, cfl: float, threshold: float = 1e-8, max_iter: int = 10000, dt: float = 1e100,
                     n_rec: int = 1, vol_wise: bool = False, history: list | None = None):
        """Pseudo-time iterations until the density component of the increment norm, relative to its
        largest value so far, drops below threshold (fstop, DNDS_FV_EulerSolver.hpp:984-994).
        Returns (iterations, relative residual, wall flux of the last iteration)."""
        self.bdf_begin()
        base = None
        rel = np.ones(self.nv)
        wf = np.zeros(self.nv)
        it = 0
        for it in range(1, max_iter + 1):
            res, wf = self.implicit_iteration(cfl, dt, 1.0, n_rec, vol_wise)
            base = res.copy() if base is None else np.maximum(base, res)
            rel = res / np.where(base > 0, base, 1.0)
            if history is not None:
                history.append(res.copy())
            if rel[0] < threshold:
                break
        return it, rel, wf

    # ------------------------------------------------------------------ learned warm start
    def set_warm_start_features(self, mode: int):
        """The warm start's input design: 0 Jacobi extrapolation, 1 the previous-step coefficients and
        the neighbour mean differences (dndsg_set_warm_start_features)."""
        self._check(self.L.dndsg_set_warm_start_features(self.h, int(mode)))

    def mlp_features(self, X_ptr: int, scales_ptr: int):
        """Features [N][64] and scales [N][4] of the current state into device arrays."""
        self._check(self.L.dndsg_mlp_features(self.h, C.c_void_p(X_ptr), C.c_void_p(scales_ptr), self.stream))

    def vr_to_tolerance(self, tol: float, max_sweeps: int = 200, mlp=None, harvest_x: int = 0,
                        harvest_t: int = 0):
        """Jacobi sweeps until the rms coefficient increment <= tol; returns (sweeps, cells on the learned start)."""
        sw = C.c_int()
        acc = C.c_int64()
        self._check(self.L.dndsg_vr_to_tolerance(self.h, mlp.h if mlp is not None else None, float(tol),
                                                  int(max_sweeps), C.byref(sw), C.byref(acc),
                                                  C.c_void_p(harvest_x or None), C.c_void_p(harvest_t or None),
                                                  self.stream))
        return sw.value, acc.value

    def ssprk3_step_tol(self, cfl: float, tol: float, max_sweeps: int = 200, mlp=None, t_end: float = 1e300,
                        harvest_x: int = 0, harvest_t: int = 0) -> int:
        """One SSP-RK3 step with every stage's reconstruction iterated to tol; returns the sweeps taken."""
        sw = C.c_int()
        self._check(self.L.dndsg_ssprk3_step_tol(self.h, mlp.h if mlp is not None else None, float(cfl),
                                                  float(t_end), float(tol), int(max_sweeps), C.byref(sw),
                                                  C.c_void_p(harvest_x or None), C.c_void_p(harvest_t or None),
                                                  self.stream))
        return sw.value

    def face_values(self, t: float = 0.0) -> np.ndarray:
        out = np.empty((self.F, 3, 2, 4))
        self._check(self.L.dndsg_face_values(self.h, float(t), _p(out), self.stream))
        return out

    def status(self):
        f = C.c_uint32()
        n = C.c_uint64()
        self._check(self.L.dndsg_get_status(self.h, C.byref(f), C.byref(n), self.stream))
        return f.value, n.value

    def run_to(self, t_end: float, cfl: float, max_steps: int = 10**9) -> int:
        """SSP-RK3 steps until the device clock reaches t_end (last step clipped); returns the steps
        taken.  Steps go in batches of at most half the remaining steps at the last batch's mean dt
        (at most 64), so the host reads the clock rarely and no zero-length step is run or counted."""
        steps = 0
        t = self.time
        dts = 0.0
        while steps < max_steps and t < t_end - 1e-12 * max(1.0, abs(t_end)):
            k = int(min(64, max(1, 0.5 * (t_end - t) / dts))) if dts > 0 else 1
            k = min(k, max_steps - steps)
            for _ in range(k):
                self.ssprk3_step(cfl, t_end)
            t_new = self.time
            dts = (t_new - t) / k
            steps += k
            t = t_new
        return steps
