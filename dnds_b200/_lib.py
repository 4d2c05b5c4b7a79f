"""ctypes binding of libdndsg.so (include/dndsg.h).  No fallback: if the
library is missing or a call fails, an exception says so."""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB

_lib = None

# every symbol include/dndsg.h declares
EXPORTS = [
    "dndsg_create", "dndsg_destroy", "dndsg_last_error", "dndsg_n_cells", "dndsg_n_faces",
    "dndsg_set_u", "dndsg_get_u", "dndsg_set_urec", "dndsg_get_urec", "dndsg_get_dt",
    "dndsg_device_buffer", "dndsg_get_time", "dndsg_set_time", "dndsg_vr_jacobi_step",
    "dndsg_limiter_wbap", "dndsg_limiter_wbap_v2", "dndsg_eval_dt", "dndsg_eval_rhs", "dndsg_ssprk3_step", "dndsg_ssprk3_steps",
    "dndsg_residual", "dndsg_face_values", "dndsg_get_status", "dndsg_eval_rhs_noalloc",
    "dndsg_mlp_create", "dndsg_mlp_destroy", "dndsg_mlp_last_error", "dndsg_mlp_set_params",
    "dndsg_mlp_get_params", "dndsg_mlp_forward", "dndsg_mlp_gradient", "dndsg_mlp_train_step",
    "dndsg_mlp_features", "dndsg_vr_to_tolerance", "dndsg_ssprk3_step_tol", "dndsg_mlp_set_features",
    "dndsg_set_warm_start_features",
    "dndsg_lusgs_colours", "dndsg_lusgs_set_order", "dndsg_lusgs_set_parts", "dndsg_lusgs_matrix_init", "dndsg_lusgs_forward", "dndsg_lusgs_backward",
    "dndsg_bdf_begin", "dndsg_implicit_iteration", "dndsg_dual_reset", "dndsg_dual_step", "dndsg_lusgs_matvec", "dndsg_gmres_lusgs",
    "dndsg_set_owned", "dndsg_rk_dt", "dndsg_rk_set_dt", "dndsg_rk_vr", "dndsg_rk_limit", "dndsg_rk_stage",
    "dndsg_rk_finish", "dndsg_halo_pack", "dndsg_halo_unpack", "dndsg_steady_solve",
]
_NO_STATUS = ("dndsg_destroy", "dndsg_last_error", "dndsg_n_cells", "dndsg_n_faces", "dndsg_mlp_destroy",
              "dndsg_mlp_last_error")

MLP_IN, MLP_OUT, MLP_NPARAM = 64, 20, 14560


class DualSettings(C.Structure):
    """dndsg_dual_settings (include/dndsg.h), field for field."""
    _fields_ = [("scheme", C.c_int), ("bdf_order", C.c_int), ("cfl", C.c_double), ("max_iter", C.c_int),
                ("threshold", C.c_double), ("n_rec", C.c_int), ("vol_wise", C.c_int), ("gmres_code", C.c_int),
                ("n_gmres_space", C.c_int), ("n_gmres_iter", C.c_int)]


class SteadySettings(C.Structure):
    """dndsg_steady_settings (include/dndsg.h), field for field."""
    _fields_ = [("cfl", C.c_double), ("cfl_ramp_end", C.c_double), ("cfl_ramp_start", C.c_int),
                ("cfl_ramp_length", C.c_int), ("max_iter", C.c_int), ("threshold", C.c_double), ("dt", C.c_double),
                ("n_rec", C.c_int), ("vol_wise", C.c_int), ("gmres_code", C.c_int), ("n_gmres_space", C.c_int),
                ("n_gmres_iter", C.c_int)]


class MeshDesc(C.Structure):
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


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise RuntimeError(f"{LIB} is not built; run `python -m dnds_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB)
    vp, i32, dbl, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    from .settings import Settings

    L.dndsg_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Settings), i32, C.POINTER(vp)]
    L.dndsg_destroy.argtypes = [vp]
    L.dndsg_destroy.restype = None
    L.dndsg_last_error.argtypes = [vp]
    L.dndsg_last_error.restype = C.c_char_p
    L.dndsg_n_cells.argtypes = [vp]
    L.dndsg_n_cells.restype = i64
    L.dndsg_n_faces.argtypes = [vp]
    L.dndsg_n_faces.restype = i64
    for nm in ["dndsg_set_u", "dndsg_get_u", "dndsg_set_urec", "dndsg_get_urec", "dndsg_get_dt"]:
        getattr(L, nm).argtypes = [vp, vp, vp]
    L.dndsg_device_buffer.argtypes = [vp, i32, C.POINTER(vp), C.POINTER(i64)]
    L.dndsg_get_time.argtypes = [vp, C.POINTER(dbl), vp]
    L.dndsg_set_time.argtypes = [vp, dbl, vp]
    L.dndsg_vr_jacobi_step.argtypes = [vp, i32, C.POINTER(dbl), vp]
    L.dndsg_limiter_wbap.argtypes = [vp, i32, vp, vp]
    L.dndsg_limiter_wbap_v2.argtypes = [vp, i32, vp, vp]
    L.dndsg_eval_dt.argtypes = [vp, dbl, dbl, i32, C.POINTER(dbl), vp]
    L.dndsg_eval_rhs.argtypes = [vp, dbl, vp, vp]
    L.dndsg_ssprk3_step.argtypes = [vp, dbl, dbl, vp]
    L.dndsg_ssprk3_steps.argtypes = [vp, dbl, dbl, C.c_int64, vp]
    L.dndsg_residual.argtypes = [vp, i32, i32, vp, vp]
    L.dndsg_face_values.argtypes = [vp, dbl, vp, vp]
    L.dndsg_get_status.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), vp]
    L.dndsg_eval_rhs_noalloc.argtypes = [vp, vp, vp, vp, dbl, vp]
    L.dndsg_mlp_create.argtypes = [i32, C.c_uint64, C.POINTER(vp)]
    L.dndsg_mlp_destroy.argtypes = [vp]
    L.dndsg_mlp_destroy.restype = None
    L.dndsg_mlp_last_error.argtypes = [vp]
    L.dndsg_mlp_last_error.restype = C.c_char_p
    L.dndsg_mlp_set_params.argtypes = [vp, vp]
    L.dndsg_mlp_get_params.argtypes = [vp, vp]
    L.dndsg_mlp_forward.argtypes = [vp, vp, i64, vp, vp]
    L.dndsg_mlp_gradient.argtypes = [vp, vp, vp, i64, C.POINTER(dbl), vp, vp]
    L.dndsg_mlp_train_step.argtypes = [vp, vp, vp, i64, C.c_float, C.POINTER(dbl), vp]
    L.dndsg_mlp_features.argtypes = [vp, vp, vp, vp]
    L.dndsg_mlp_set_features.argtypes = [vp, i32]
    L.dndsg_set_warm_start_features.argtypes = [vp, i32]
    L.dndsg_vr_to_tolerance.argtypes = [vp, vp, dbl, i32, C.POINTER(i32), C.POINTER(i64), vp, vp, vp]
    L.dndsg_ssprk3_step_tol.argtypes = [vp, vp, dbl, dbl, dbl, i32, C.POINTER(i32), vp, vp, vp]
    L.dndsg_lusgs_colours.argtypes = [vp, vp, C.POINTER(i32)]
    L.dndsg_lusgs_set_order.argtypes = [vp, i32, vp, C.POINTER(i32)]
    L.dndsg_lusgs_set_parts.argtypes = [vp, vp, i32, C.POINTER(i32)]
    L.dndsg_lusgs_matrix_init.argtypes = [vp, dbl, dbl, vp]
    L.dndsg_lusgs_forward.argtypes = [vp, dbl, vp, vp, vp]
    L.dndsg_lusgs_backward.argtypes = [vp, dbl, vp, vp, vp]
    L.dndsg_bdf_begin.argtypes = [vp, vp]
    L.dndsg_implicit_iteration.argtypes = [vp, dbl, dbl, dbl, i32, i32, dbl, vp, vp, vp]
    L.dndsg_dual_reset.argtypes = [vp]
    L.dndsg_dual_step.argtypes = [vp, C.POINTER(DualSettings), dbl, dbl, vp, vp, vp]
    L.dndsg_lusgs_matvec.argtypes = [vp, dbl, vp, vp, vp]
    L.dndsg_gmres_lusgs.argtypes = [vp, dbl, i32, i32, vp, vp, vp]
    L.dndsg_set_owned.argtypes = [vp, vp]
    L.dndsg_rk_dt.argtypes = [vp, dbl, C.POINTER(dbl), vp]
    L.dndsg_rk_set_dt.argtypes = [vp, dbl, vp]
    L.dndsg_rk_vr.argtypes = [vp, vp]
    L.dndsg_rk_limit.argtypes = [vp, vp]
    L.dndsg_rk_stage.argtypes = [vp, i32, vp]
    L.dndsg_rk_finish.argtypes = [vp, vp]
    L.dndsg_halo_pack.argtypes = [vp, i32, vp, i64, vp, vp]
    L.dndsg_halo_unpack.argtypes = [vp, i32, vp, i64, vp, vp]
    L.dndsg_steady_solve.argtypes = [vp, C.POINTER(SteadySettings), C.POINTER(i32), vp, vp, vp, vp]
    for nm in EXPORTS:
        if nm not in _NO_STATUS:
            getattr(L, nm).restype = i32
    _lib = L
    return L
