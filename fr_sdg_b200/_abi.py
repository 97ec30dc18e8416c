"""ctypes mirror of include/frsdg.h and the loader of libfrsdg.so.

The library is the product: there is no Python or CPU fallback.  Loading fails
with an ImportError naming the missing file when libfrsdg.so has not been built
(`python -m fr_sdg_b200.build`).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfrsdg.so"

POST_STEP_STATIC_MAX_DOFS = 4194304  # FRSDG_POST_STEP_STATIC_MAX_DOFS in include/frsdg.h
# frsdg_rk_stage_fused flags
STAGE_MIXED, STAGE_LIMIT, STAGE_POST_STEP = 1, 2, 4

# status codes
OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_NODEVICE = 0, -1, -2, -3, -4, -5
# policies
GAS_IDEAL, GAS_VDW = 0, 1
RUSANOV, HLLC = 0, 1
COORD_CARTESIAN, COORD_RADIAL = 0, 1
GEOM_CARTESIAN, GEOM_DELAVAL, GEOM_WALL_PROFILE, GEOM_SINE_WARP = 0, 1, 2, 3
PROFILE_FLAT, PROFILE_WEDGE_BUMP, PROFILE_WEDGE_BC, PROFILE_GAUSS_BUMP = 0, 1, 2, 3
LEFT, RIGHT, TOP, BOTTOM = 0, 1, 2, 3
(BC_OUTFLOW, BC_WALL, BC_PERIODIC, BC_DIRICHLET, BC_SLIP_WALL, BC_VORTEX,
 BC_SUBSONIC_INFLOW, BC_PRESSURE_OUTLET) = range(8)


class frsdg_bc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad_", C.c_int32),
                ("state", C.c_double * 4), ("params", C.c_double * 6)]


class frsdg_config(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("poly_deg", C.c_int32), ("n_elems", C.c_int32 * 2),
        ("box_length", C.c_double * 2), ("radau_corr", C.c_double),
        ("gas_law", C.c_int32), ("riemann", C.c_int32),
        ("gamma", C.c_double), ("R_spec", C.c_double), ("vdw_a", C.c_double), ("vdw_b", C.c_double),
        ("coord_sys", C.c_int32), ("geometry", C.c_int32), ("geom_profile", C.c_int32), ("pad0_", C.c_int32),
        ("geom_params", C.c_double * 4),
        ("bc", frsdg_bc * 4),
        ("apply_filter", C.c_int32), ("filt_cut_off", C.c_int32), ("filt_strength", C.c_int32),
        ("apply_weno", C.c_int32),
        ("filt_alpha", C.c_double), ("weno_gamma", C.c_double),
        ("shock_theta", C.c_double), ("shock_threshold", C.c_double),
        ("cond_sys", C.c_int32), ("jvp_exact_bc", C.c_int32),
        ("csd_eps", C.c_double),
        ("pp_limit", C.c_int32), ("mixed_tc", C.c_int32), ("pp_eps", C.c_double),
    ]


# every entry point declared in include/frsdg.h: name -> (restype, argtypes)
_P = C.c_void_p
_D = C.c_double
SIGNATURES = {
    "frsdg_abi_version": (C.c_int, []),
    "frsdg_last_error": (C.c_char_p, []),
    "frsdg_config_default": (C.c_int, [C.POINTER(frsdg_config)]),
    "frsdg_create": (C.c_int, [C.POINTER(frsdg_config), C.POINTER(_P)]),
    "frsdg_destroy": (C.c_int, [_P]),
    "frsdg_n_dofs": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "frsdg_residual": (C.c_int, [_P, _D, _P, _P, _P]),
    "frsdg_rhs": (C.c_int, [_P, _D, _P, _P, _P]),
    "frsdg_ifunction": (C.c_int, [_P, _D, _P, _P, _P, _P]),
    "frsdg_jvp_prepare": (C.c_int, [_P, _D, _D, _P]),
    "frsdg_jvp": (C.c_int, [_P, _P, _P, _P]),
    "frsdg_rk_stage": (C.c_int, [_P, _D, _P, _P, _D, _P, _D, _D, _P, _P, _D, _P]),
    "frsdg_jac_blocks": (C.c_int, [_P, _D, _D, _P, _P, _P]),
    "frsdg_residual_f32": (C.c_int, [_P, _D, _P, _P, _P]),
    "frsdg_set_row_window": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "frsdg_rk_stage_mixed": (C.c_int, [_P, _D, _P, _P, _D, _P, _D, _D, _P, _P, _D, _P]),
    "frsdg_rk_stage_fused": (C.c_int, [_P, _D, _P, _P, _D, _P, _D, _D, _P, _P, _D, C.c_int32, _P]),
    "frsdg_pc_setup": (C.c_int, [_P, _D, _D, _P, _P]),
    "frsdg_pc_apply": (C.c_int, [_P, _P, _P, _P]),
    "frsdg_jac_blocks5": (C.c_int, [_P, _D, _D, _P, _P, _P]),
    "frsdg_pc_setup_gs": (C.c_int, [_P, _D, _D, _P, _P]),
    "frsdg_post_step": (C.c_int, [_P, _P, _P]),
    "frsdg_post_step_to": (C.c_int, [_P, _P, _P, _P]),
    "frsdg_post_step_static": (C.c_int, [C.POINTER(frsdg_config), _P, _P]),
    "frsdg_prim_to_cons": (C.c_int, [_P, _P, _P, _P]),
    "frsdg_pp_limit": (C.c_int, [_P, _P, _P, _P]),
    "frsdg_rhs_host": (C.c_int, [_P, _D, _P, _P, _P]),
    "frsdg_status": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "frsdg_check_state": (C.c_int, [_P, _P, _P]),
    "frsdg_batch_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P), C.POINTER(_D), C.POINTER(_D),
                                     C.POINTER(_D), C.c_int32, C.POINTER(_P)]),
    "frsdg_batch_step": (C.c_int, [_P, _P]),
    "frsdg_batch_run": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int64), _P]),
    "frsdg_batch_times": (C.c_int, [_P, C.POINTER(_D), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "frsdg_batch_groups": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "frsdg_batch_tuning": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "frsdg_batch_destroy": (C.c_int, [_P]),
    "frsdg_device_math": (C.c_int, [C.c_int32, _P, _P, C.c_int64, _P]),
    "frsdg_tc_lines": (C.c_int, [C.c_int32, _P, _P, _P, C.c_int64, _P]),
    "frsdg_gmres_work_doubles": (C.c_int64, [C.c_int64]),
    "frsdg_gmres_arnoldi": (C.c_int, [_P, C.c_int64, C.c_int32, _P, C.c_int64, _P, C.c_int32, _P, _P, _P, _P, _P,
                                      _P]),
    "frsdg_gmres_solve": (C.c_int, [_P, C.c_int32, _P, C.c_int32, _P, _P]),
    "frsdg_petsc_vec_record_bytes": (C.c_int, [C.c_int64, C.c_int32, C.POINTER(C.c_int64)]),
    "frsdg_petsc_vec_pack": (C.c_int, [_P, C.c_int64, C.c_int32, _P, _P]),
    "frsdg_reference_element": (C.c_int, [C.c_int32, _D, _P, _P, _P, _P, _P]),
    "frsdg_filter_matrix": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _D, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libfrsdg.so once; raise ImportError when it is missing."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("FRSDG_LIB", LIB_PATH))
        if not path.exists():
            raise ImportError(f"{path} is missing: build it with `python -m fr_sdg_b200.build`")
        handle = C.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class FrsdgError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().frsdg_last_error().decode(errors="replace")
        super().__init__(f"{where} failed ({code}): {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != OK:
        raise FrsdgError(code, where)
