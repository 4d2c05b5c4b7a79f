"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libdnds_oracle.so")
_lib = None


class OrcMesh(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("n_cells", C.c_int64),
        ("n_faces", C.c_int64),
        ("node_xy", C.c_void_p),
        ("cell_nodes", C.c_void_p),
        ("face_nodes", C.c_void_p),
        ("face_cells", C.c_void_p),
        ("face_bc", C.c_void_p),
        ("face_shift", C.c_void_p),
    ]


class OrcSettings(C.Structure):
    _fields_ = [
        ("nvars", C.c_int32),
        ("rec_order", C.c_int32),
        ("riemann", C.c_int32),
        ("sor_instead", C.c_int32),
        ("jacobi_relax", C.c_double),
        ("tang_weight", C.c_double),
        ("tang_weight_mod_min", C.c_double),
        ("tang_weight_mod_power", C.c_double),
        ("tang_weight_mod_loc", C.c_int32),
        ("tang_weight_direction", C.c_int32),
        ("base_center_type", C.c_int32),
        ("use_local_coord", C.c_int32),
        ("anisotropic_lengths", C.c_int32),
        ("weight_scheme_geom", C.c_int32),
        ("weight_scheme_dir", C.c_int32),
        ("limiter", C.c_int32),
        ("weight_len_scale", C.c_double),
        ("wall_weight", C.c_double),
        ("far_weight", C.c_double),
        ("wbap_smooth_indicator_scale", C.c_double),
        ("wbap_n_std", C.c_double),
        ("gamma", C.c_double),
        ("far_field", C.c_double * 6),
        ("n_threads", C.c_int32),
        ("pad0", C.c_int32),
        ("mu_gas", C.c_double),
        ("cp_gas", C.c_double),
        ("pr_gas", C.c_double),
        ("t_ref", C.c_double),
        ("c_sutherland", C.c_double),
    ]


def build() -> str:
    """Compile the oracle (make in oracle/); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int, C.c_double
        L.orc_create.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcSettings), C.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_last_error.argtypes = [vp]
        L.orc_last_error.restype = C.c_char_p
        for nm in ["orc_set_u", "orc_get_u", "orc_set_urec", "orc_get_urec", "orc_init_isentropic_vortex"]:
            getattr(L, nm).argtypes = [vp] + ([vp] if nm != "orc_init_isentropic_vortex" else [])
        L.orc_get_geometry.argtypes = [vp, vp, vp, vp]
        L.orc_exact_isentropic_vortex.argtypes = [vp, dbl, vp]
        L.orc_init_quadrants.argtypes = [vp, dbl, dbl, vp]
        L.orc_vr_step.argtypes = [vp, i32]
        L.orc_vr_last_increment.argtypes = [vp]
        L.orc_vr_last_increment.restype = dbl
        L.orc_limiter_wbap.argtypes = [vp, i32, vp]
        L.orc_limiter_wbap_v2.argtypes = [vp, i32, vp]
        L.orc_eval_dt.argtypes = [vp, dbl, dbl, i32, vp, vp]
        L.orc_eval_rhs.argtypes = [vp, dbl, vp, vp]
        L.orc_face_values.argtypes = [vp, dbl, vp]
        L.orc_ssprk3_step.argtypes = [vp, dbl, dbl]
        L.orc_residual.argtypes = [vp, vp, i32, i32, vp]
        L.orc_get_vr_blocks.argtypes = [vp, vp, vp, vp]
        L.orc_get_face_dibj.argtypes = [vp, vp]
        L.orc_lusgs_matrix_init.argtypes = [vp, vp, dbl, dbl]
        L.orc_lusgs_forward.argtypes = [vp, dbl, vp, vp, vp]
        L.orc_lusgs_backward.argtypes = [vp, dbl, vp, vp, vp]
        L.orc_implicit_iteration.argtypes = [vp, dbl, dbl, dbl, vp, vp, dbl, i32, vp]
        L.orc_lusgs_matvec.argtypes = [vp, dbl, vp, vp]
        L.orc_set_lusgs_parts.argtypes = [vp, vp]
        L.orc_gmres_lusgs.argtypes = [vp, dbl, i32, i32, vp, vp, vp]
        L.orc_dual_reset.argtypes = [vp]
        L.orc_dual_step.argtypes = [vp, C.POINTER(OrcDual), dbl, dbl, vp, vp, vp]
        L.orc_riemann_flux.argtypes = [i32, vp, vp, dbl, dbl, vp]
        L.orc_riemann_flux.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def riemann_flux(kind: int, ul, ur, gamma=1.4, dlambda=0.0) -> np.ndarray:
    ul = np.ascontiguousarray(ul, dtype=np.float64)
    ur = np.ascontiguousarray(ur, dtype=np.float64)
    f = np.zeros(4)
    lib().orc_riemann_flux(kind, _p(ul), _p(ur), gamma, dlambda, _p(f))
    return f


class OrcDual(C.Structure):
    """orc_dual_settings (dnds_oracle.h), field for field."""
    _fields_ = [("scheme", C.c_int), ("bdf_order", C.c_int), ("cfl", C.c_double), ("max_iter", C.c_int),
                ("threshold", C.c_double), ("n_rec", C.c_int), ("vol_wise", C.c_int), ("gmres_code", C.c_int),
                ("n_gmres_space", C.c_int), ("n_gmres_iter", C.c_int)]


def dual_settings(scheme="sdirk4", bdf_order=2, cfl=100.0, max_iter=10, threshold=1e-100, n_rec=1, vol_wise=False,
                  gmres_code=0, n_gmres_space=10, n_gmres_iter=2):
    """The dual-time settings with the reference's config names in mind: odeCode (scheme "sdirk4" = 0,
    "bdf" = 1), nTimeStepInternal, rhsThresholdInternal, nInternalRecStep, useVolWiseResidual,
    gmresCode, nGmresSpace, nGmresIter."""
    return dict(scheme={"sdirk4": 0, "bdf": 1}[scheme], bdf_order=bdf_order, cfl=cfl, max_iter=max_iter,
                threshold=threshold, n_rec=n_rec, vol_wise=int(vol_wise), gmres_code=gmres_code,
                n_gmres_space=n_gmres_space, n_gmres_iter=n_gmres_iter)


class Oracle:
    """FP64 restatement of DNDS's VR + Euler evaluator on one mesh."""

    def __init__(self, mesh, cfg: dict, n_threads: int = 0):
        from dnds_b200.settings import make_settings

        ps = make_settings(cfg)
        s = OrcSettings()
        for name, _ in OrcSettings._fields_:
            if name == "pad0":
                continue
            if name == "far_field":
                for k in range(6):
                    s.far_field[k] = ps.far_field[k]
            elif name == "sor_instead":
                s.sor_instead = int(cfg.get("vfvSetting", {}).get("SOR_Instead", False))
            else:
                setattr(s, name, getattr(ps, name))
        s.n_threads = n_threads
        self.mesh = mesh
        self._keep = [mesh.node_xy, mesh.cell_nodes, mesh.face_nodes, mesh.face_cells, mesh.face_bc, mesh.face_shift]
        m = OrcMesh(mesh.n_nodes, mesh.n_cells, mesh.n_faces, *[_p(a) for a in self._keep])
        h = C.c_void_p()
        rc = lib().orc_create(C.byref(m), C.byref(s), C.byref(h))
        self.h = h
        if rc != 0:
            msg = lib().orc_last_error(h).decode()
            lib().orc_destroy(h)
            self.h = None
            raise RuntimeError(f"oracle setup failed ({rc}): {msg}")
        self.N = mesh.n_cells
        self.F = mesh.n_faces
        self.nv = s.nvars

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    # state
    def set_u(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.N, self.nv)
        lib().orc_set_u(self.h, _p(u))

    def get_u(self):
        u = np.empty((self.N, self.nv))
        lib().orc_get_u(self.h, _p(u))
        return u

    def set_urec(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(self.N, 5, self.nv)
        lib().orc_set_urec(self.h, _p(r))

    def get_urec(self):
        r = np.empty((self.N, 5, self.nv))
        lib().orc_get_urec(self.h, _p(r))
        return r

    def geometry(self):
        vol = np.empty(self.N)
        bary = np.empty((self.N, 2))
        area = np.empty(self.F)
        lib().orc_get_geometry(self.h, _p(vol), _p(bary), _p(area))
        return vol, bary, area

    def init_vortex(self):
        lib().orc_init_isentropic_vortex(self.h)

    def exact_vortex(self, t):
        out = np.empty((self.N, self.nv))
        lib().orc_exact_isentropic_vortex(self.h, t, _p(out))
        return out

    def init_quadrants(self, xs, ys, states):
        q = np.ascontiguousarray(np.array(states, dtype=np.float64).reshape(4, 4))
        lib().orc_init_quadrants(self.h, xs, ys, _p(q))

    def vr_step(self, n=1):
        lib().orc_vr_step(self.h, n)
        return lib().orc_vr_last_increment(self.h)

    def limiter(self, if_all=False):
        ind = np.empty(self.N)
        lib().orc_limiter_wbap(self.h, int(if_all), _p(ind))
        return ind

    def limiter_v2(self, if_all=False):
        """ReconstructionWBAPLimitFacialV2 (3WBAP) in place; returns the smoothness indicator."""
        ind = np.empty(self.N)
        lib().orc_limiter_wbap_v2(self.h, int(if_all), _p(ind))
        return ind

    def eval_dt(self, cfl, max_dt=1e100, use_local_dt=False):
        dt = np.empty(self.N)
        dmin = C.c_double()
        lib().orc_eval_dt(self.h, cfl, max_dt, int(use_local_dt), _p(dt), C.byref(dmin))
        return dt, dmin.value

    def eval_rhs(self, t=0.0):
        rhs = np.empty((self.N, self.nv))
        wf = np.empty(self.nv)
        lib().orc_eval_rhs(self.h, t, _p(rhs), _p(wf))
        return rhs, wf

    def face_values(self, t=0.0):
        out = np.empty((self.F, 3, 2, self.nv))
        lib().orc_face_values(self.h, t, _p(out))
        return out

    def ssprk3_step(self, dt, t):
        lib().orc_ssprk3_step(self.h, dt, t)

    # ---------------------------------------------------------------- implicit path
    @staticmethod
    def _order(scan2cell):
        if scan2cell is None:
            return None, None
        o = np.ascontiguousarray(scan2cell, dtype=np.int64)
        return o, _p(o)

    def set_lusgs_parts(self, part=None):
        """Partitioned LU-SGS sweeps (the reference on several MPI ranks); None: one part."""
        self._parts = None if part is None else np.ascontiguousarray(part, dtype=np.int32)
        lib().orc_set_lusgs_parts(self.h, _p(self._parts) if self._parts is not None else None)

    def lusgs_matrix_init(self, dt, alpha=1.0, dtau=None):
        d = None if dtau is None else np.ascontiguousarray(dtau, dtype=np.float64)
        lib().orc_lusgs_matrix_init(self.h, _p(d) if d is not None else None, dt, alpha)

    def lusgs_forward(self, rhs, inc, alpha=1.0, scan2cell=None):
        """In place on inc (float64 [N][nv])."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        o, op = self._order(scan2cell)
        if lib().orc_lusgs_forward(self.h, alpha, _p(rhs), _p(inc), op):
            raise RuntimeError("lusgs_matrix_init first")

    def lusgs_backward(self, rhs, inc, alpha=1.0, scan2cell=None):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        o, op = self._order(scan2cell)
        if lib().orc_lusgs_backward(self.h, alpha, _p(rhs), _p(inc), op):
            raise RuntimeError("lusgs_matrix_init first")

    def implicit_iteration(self, cfl, x_last, dt=1e100, alpha=1.0, scan2cell=None, t=0.0, n_rec=1):
        """One first-order BDF pseudo-time iteration; returns the increment [N][nv]."""
        xl = np.ascontiguousarray(x_last, dtype=np.float64)
        inc = np.empty((self.N, self.nv))
        o, op = self._order(scan2cell)
        lib().orc_implicit_iteration(self.h, cfl, dt, alpha, _p(xl), op, t, n_rec, _p(inc))
        return inc

    def lusgs_matvec(self, x, alpha=1.0):
        """LUSGSMatrixVec with the diagonal of the last lusgs_matrix_init."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        ax = np.empty_like(x)
        if lib().orc_lusgs_matvec(self.h, alpha, _p(x), _p(ax)):
            raise RuntimeError("orc_lusgs_matvec: lusgs_matrix_init first")
        return ax

    def gmres_lusgs(self, b, x0=None, alpha=1.0, n_space=10, n_restart=2, scan2cell=None):
        """GMRES over LUSGSMatrixVec, LU-SGS preconditioned, from x0 (zero by default)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
        o, op = self._order(scan2cell)
        if lib().orc_gmres_lusgs(self.h, alpha, n_space, n_restart, _p(b), _p(x), op):
            raise RuntimeError("orc_gmres_lusgs: lusgs_matrix_init first")
        return x

    def dual_reset(self):
        lib().orc_dual_reset(self.h)

    def dual_step(self, dt, t=0.0, scan2cell=None, **settings):
        """One physical dual-time step (see dual_settings); returns (iterations per stage, last fstop
        ratios)."""
        d = OrcDual(**dual_settings(**settings))
        its = np.zeros(3, dtype=np.int32)
        res = np.zeros(self.nv)
        o, op = self._order(scan2cell)
        if lib().orc_dual_step(self.h, C.byref(d), dt, t, op, _p(its), _p(res)):
            raise RuntimeError("orc_dual_step: bad settings or a BDF history of another dt")
        return its, res

    def residual(self, rhs, p=1, vol_wise=False):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        out = np.empty(self.nv)
        lib().orc_residual(self.h, _p(rhs), p, int(vol_wise), _p(out))
        return out

    def vr_blocks(self):
        a = np.empty((self.N, 5, 5))
        b = np.empty((self.N, 4, 5, 5))
        v = np.empty((self.N, 4, 5))
        lib().orc_get_vr_blocks(self.h, _p(a), _p(b), _p(v))
        return a, b, v

    def face_dibj(self):
        out = np.empty((self.F, 3, 2, 6, 6))
        lib().orc_get_face_dibj(self.h, _p(out))
        return out

    def run_vortex(self, t_end, cfl=0.5, max_steps=10**9):
        """SSP-RK3 with global dt (EvaluateDt, UseLocaldt=false), last step clipped to t_end."""
        t = 0.0
        steps = 0
        while t < t_end - 1e-14 and steps < max_steps:
            _, dtmin = self.eval_dt(cfl)
            dt = min(dtmin, t_end - t)
            self.ssprk3_step(dt, t)
            t += dt
            steps += 1
        return t, steps
