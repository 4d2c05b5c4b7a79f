"""Solver settings: the subset of DNDS JSON keys the hot path reads.

Keys and defaults follow ``VRFiniteVolume2D::Setting`` (DNDS_FV_VR.hpp:170-230),
``EulerEvaluator::Setting`` (DNDS_FV_EulerEvaluator.hpp:138-194) and the
parser ``EulerSolver::ConfigureFromJson`` (DNDS_FV_EulerSolver.hpp:133-427).
``Settings`` is laid out exactly like ``dndsg_settings`` in include/dndsg.h.
"""
from __future__ import annotations

import ctypes as C

RIEMANN = {"Roe": 1, "HLLC": 2}
WEIGHT_GEOM = {"None": 0, "D": 1, "S": 2, "SDHQM": 3}
WEIGHT_DIR = {"None": 0, "optHQM": 1}
TANG_DIR = {"Norm": 0, "Bary": 1}
CENTER = {"Bary": 0, "Param": 1}

PRECISION_FP64 = 0
PRECISION_FP32 = 1


class Settings(C.Structure):
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
        ("precision", C.c_int32),
        ("mu_gas", C.c_double),
        ("cp_gas", C.c_double),
        ("pr_gas", C.c_double),
        ("t_ref", C.c_double),
        ("c_sutherland", C.c_double),
    ]


def make_settings(cfg: dict) -> Settings:
    """Build a ``Settings`` from a DNDS-style config dict (``vfvSetting`` / ``eulerSetting`` keys)."""
    vfv = cfg.get("vfvSetting", {})
    eul = cfg.get("eulerSetting", {})
    s = Settings()
    s.nvars = int(cfg.get("nvars", 4))
    s.rec_order = int(cfg.get("recOrder", 2))
    s.riemann = RIEMANN[eul.get("riemannSolverType", "Roe")]
    s.sor_instead = 1 if vfv.get("SOR_Instead", False) else 0
    s.jacobi_relax = float(vfv.get("JacobiRelax", 1.0))
    s.tang_weight = float(vfv.get("tangWeight", 1.0))
    s.tang_weight_mod_min = float(vfv.get("tangWeightModMin", 1.0))
    s.tang_weight_mod_power = float(vfv.get("tangWeightModPower", 1.0))
    s.tang_weight_mod_loc = int(vfv.get("tangWeightModLoc", 0))
    s.tang_weight_direction = TANG_DIR[vfv.get("tangWeightDirection", "Bary")]
    s.base_center_type = CENTER[vfv.get("baseCenterType", "Bary")]
    s.use_local_coord = 1 if vfv.get("useLocalCoord", False) else 0
    s.anisotropic_lengths = 1 if vfv.get("anisotropicLengths", False) else 0
    s.weight_scheme_geom = WEIGHT_GEOM[vfv.get("weightSchemeGeom", "None")]
    s.weight_scheme_dir = WEIGHT_DIR[vfv.get("weightSchemeDir", "None")]
    # limiterProcedure (DNDS_FV_EulerSolver.hpp:108): 0 = ReconstructionWBAPLimitFacialV2 (3WBAP, the
    # reference's default), 1 = ReconstructionWBAPLimitFacialV3 (CWBAP); settings.limiter 2 and 1
    s.limiter = (1 if int(cfg.get("limiterProcedure", 0)) == 1 else 2) if cfg.get("useLimiter", False) else 0
    s.weight_len_scale = float(vfv.get("weightLenScale", 1.0))
    s.wall_weight = float(vfv.get("wallWeight", 1.0))
    s.far_weight = float(vfv.get("farWeight", 0.0))
    s.wbap_smooth_indicator_scale = float(vfv.get("WBAP_SmoothIndicatorScale", 1e-10))
    s.wbap_n_std = float(vfv.get("WBAP_nStd", 10.0))
    gas = eul.get("idealGasProperty", {})
    s.gamma = float(gas.get("gamma", 1.4))
    ff = list(eul.get("farFieldStaticValue", [1.0, 0.0, 0.0, 2.5]))
    for k in range(6):
        s.far_field[k] = float(ff[k]) if k < len(ff) else 0.0
    s.n_threads = int(cfg.get("nThreads", 0))
    s.precision = int(cfg.get("precision", PRECISION_FP64))
    # idealGasProperty defaults of EulerEvaluator::Setting (DNDS_FV_EulerEvaluator.hpp:150-160); without
    # muGas the model is inviscid
    rgas = float(gas.get("Rgas", 1.0))
    s.mu_gas = float(gas.get("muGas", 0.0))
    s.cp_gas = float(gas.get("CpGas", rgas * s.gamma / (s.gamma - 1)))
    s.pr_gas = float(gas.get("prGas", 0.72))
    s.t_ref = float(gas.get("TRef", 273.15))
    s.c_sutherland = float(gas.get("CSutherland", 110.4))
    return s


# vfvSetting of data/euler_config_IV.json:59-91 (recOrder 2 as the vortex cases ask);
# SOR_Instead is off: the GPU sweep is a true Jacobi sweep.
ISENTROPIC_VORTEX = {
    "recOrder": 2,
    "useLimiter": False,
    "vfvSetting": {
        "SOR_Instead": False,
        "JacobiRelax": 1.0,
        "anisotropicLengths": True,
        "tangWeight": 0.0,
        "tangWeightModMin": 1.0,
        "tangWeightDirection": "Norm",
        "useLocalCoord": True,
        "wallWeight": 0.5,
        "farWeight": 0.0,
        "weightSchemeGeom": "SDHQM",
        "weightSchemeDir": "optHQM",
        "baseCenterType": "Bary",
    },
    "eulerSetting": {
        "riemannSolverType": "Roe",
        "idealGasProperty": {"gamma": 1.4},
        "farFieldStaticValue": [1.0, 1.0, 1.0, 3.5],
    },
}

# vfvSetting of data/euler_config_2DRiemann.json:60-91, HLLC flux, CWBAP limiter (limiterProcedure 1, :27)
RIEMANN_2D = {
    "recOrder": 2,
    "useLimiter": True,
    "limiterProcedure": 1,
    "vfvSetting": {
        "SOR_Instead": False,
        "JacobiRelax": 1.0,
        "anisotropicLengths": True,
        "tangWeight": 1.0,
        "tangWeightModMin": 1.0,
        "tangWeightDirection": "Norm",
        "useLocalCoord": False,
        "wallWeight": 0.5,
        "farWeight": 0.0,
        "weightLenScale": 0.5,
        "weightSchemeGeom": "S",
        "weightSchemeDir": "None",
        "baseCenterType": "Bary",
        "WBAP_SmoothIndicatorScale": 1e-1,
    },
    "eulerSetting": {
        "riemannSolverType": "HLLC",
        "idealGasProperty": {"gamma": 1.4},
        "farFieldStaticValue": [1.0, 0.0, 0.0, 2.5],
    },
}

# four-quadrant states (rho, u, v, p): NE, NW, SW, SE, split at (0.8, 0.8)
RIEMANN_2D_STATES = [
    (1.5, 0.0, 0.0, 1.5),
    (0.5323, 1.206, 0.0, 0.3),
    (0.138, 1.206, 1.206, 0.029),
    (0.5323, 0.0, 1.206, 0.3),
]


def free_stream(mach: float, alpha_deg: float, gamma: float = 1.4):
    """Conservative free stream (rho, rho u, rho v, E) with rho = 1 and |V| = 1 at the given Mach
    number and angle of attack."""
    import math

    a = math.radians(alpha_deg)
    p = 1.0 / (gamma * mach * mach)
    return [1.0, math.cos(a), math.sin(a), p / (gamma - 1) + 0.5]


# vfvSetting of data/eulerSA_config_BenchSA.json:61-77 (Jacobi sweep instead of SOR), Roe flux,
# free stream at M 0.15, alpha 10 degrees; the steady inviscid case of the implicit path
NACA0012 = {
    "recOrder": 2,
    "vfvSetting": {
        "SOR_Instead": False,
        "JacobiRelax": 1.0,
        "anisotropicLengths": False,
        "tangWeight": 0.1,
        "wallWeight": 1.5,
        "farWeight": 1.0,
        "weightSchemeGeom": "None",
        "baseCenterType": "Bary",
    },
    "eulerSetting": {
        "riemannSolverType": "Roe",
        "idealGasProperty": {"gamma": 1.4},
        "farFieldStaticValue": free_stream(0.15, 10.0),
    },
}


def laminar_gas(mach: float, reynolds: float, gamma: float = 1.4) -> dict:
    """idealGasProperty for a laminar case with rho = 1, |V| = 1, chord 1 and Rgas = 1: the reference
    temperature is the free-stream one (T = p / rho), Sutherland's constant scaled from 110.4 K at
    288.15 K, and muGas = 1 / Re, so that the free-stream viscosity is 1 / Re."""
    t_inf = 1.0 / (gamma * mach * mach)
    return {"gamma": gamma, "Rgas": 1.0, "muGas": 1.0 / reynolds, "prGas": 0.72, "TRef": t_inf,
            "CSutherland": 110.4 / 288.15 * t_inf}


# the laminar NACA 0012 at M 0.5, Re 5000, alpha 0 (no-slip wall): the Navier-Stokes case of the
# implicit path, with the NACA0012 vfvSetting
NACA0012_LAMINAR = {
    "recOrder": 2,
    "vfvSetting": dict(NACA0012["vfvSetting"]),
    "eulerSetting": {
        "riemannSolverType": "Roe",
        "idealGasProperty": laminar_gas(0.5, 5000.0),
        "farFieldStaticValue": free_stream(0.5, 0.0),
    },
}


def naca0012_sa(mach: float = 0.15, alpha: float = 10.0, reynolds: float = 6e6, nut_ratio: float = 3.0) -> dict:
    """RANS-SA over the NACA 0012 (5 variables: rho, rho u, rho v, E, rho nu~ / muGas) with the
    NACA0012 vfvSetting; the free-stream SA variable is nut_ratio times the laminar viscosity."""
    gas = laminar_gas(mach, reynolds)
    return {
        "nvars": 5,
        "recOrder": 2,
        "vfvSetting": dict(NACA0012["vfvSetting"]),
        "eulerSetting": {
            "riemannSolverType": "Roe",
            "idealGasProperty": gas,
            "farFieldStaticValue": free_stream(mach, alpha) + [nut_ratio],
        },
    }


def preset(name: str, **overrides) -> dict:
    import copy

    base = {"vortex": ISENTROPIC_VORTEX, "riemann": RIEMANN_2D, "naca0012": NACA0012,
            "naca0012_laminar": NACA0012_LAMINAR, "naca0012_sa": naca0012_sa()}[name]
    cfg = copy.deepcopy(base)
    for k, v in overrides.items():
        if isinstance(v, dict) and isinstance(cfg.get(k), dict):
            cfg[k].update(v)
        else:
            cfg[k] = v
    return cfg
