"""ctypes binding of liblesb200.so (include/les_abi.h, include/les_synth.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblesb200.so"
CHECKED_LIB_PATH = Path(__file__).resolve().parent / "liblesb200_checked.so"
if os.environ.get("LES_B200_CHECKED") == "1":  # the bounds-checked build (tests)
    LIB_PATH = CHECKED_LIB_PATH

LES_OK, LES_ERR_BAD_ARG, LES_ERR_DIMS, LES_ERR_CUDA, LES_ERR_TIMEOUT, LES_ERR_NAN, \
    LES_ERR_NOMEM, LES_ERR_STATE, LES_ERR_IO = range(9)
LES_INFLOW_POWER_LAW, LES_INFLOW_EXTERNAL = 0, 1
# les_ctx_set_reduction_mode bits: sums taken in the reference's serial FP32 order
LES_RED_CANONICAL, LES_RED_F_RHSAV, LES_RED_F_SOR, LES_RED_F_PAV, LES_RED_FAITHFUL = 0, 1, 2, 4, 7
(LES_DD_BEGIN, LES_DD_MOMENTUM, LES_DD_RHSAV, LES_DD_SOR_ITER, LES_DD_SOR_TEST, LES_DD_PAV_SUM,
 LES_DD_PAV_END) = range(7)
FIELD_IDS = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold", "hold",
             "rhs", "sm", "amask1", "bmask1", "cmask1", "dmask1"]
HALO_IDS = ["p", "uvw", "uvwsum", "fgh", "fgh_old", "rhs", "sm"]

fp = C.POINTER(C.c_float)


class LesParams(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int),
                ("dt", C.c_float), ("ro", C.c_float), ("vn", C.c_float),
                ("alpha", C.c_float), ("beta", C.c_float), ("cs0", C.c_float),
                ("nmaxp", C.c_int), ("pjuge", C.c_float), ("omega", C.c_float),
                ("inflow_mode", C.c_int), ("ical", C.c_int)]


HOST_FIELD_NAMES = ["u", "v", "w", "p", "usum", "vsum", "wsum", "f", "g", "h", "fold", "gold",
                    "hold", "rhs", "sm", "amask1", "dmask1", "bmask1", "cmask1", "cn1", "cn2l",
                    "cn2s", "cn3l", "cn3s", "cn4l", "cn4s", "dx1", "dy1", "dzn", "dzs", "dxs",
                    "dys", "z2", "delx1", "wind_profile"]


class LesHostFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in HOST_FIELD_NAMES]


class LesMetrics(C.Structure):
    _fields_ = [("n", C.c_int), ("sor_iters", C.c_int), ("sor", C.c_float), ("rhsav", C.c_float),
                ("pav", C.c_float), ("uout", C.c_float), ("p_centre", C.c_float),
                ("u_centre", C.c_float), ("v_centre", C.c_float), ("w_centre", C.c_float)]


AVEFLOW_CELL = ["aveu", "avev", "avew", "avep", "avel", "aveuu", "avevv", "aveww", "avesm", "avesmsm",
                "uwfx"]
AVEFLOW_COL = ["avesu", "avesv", "avesw", "avesuu", "avesvv", "avesww", "uwfxs"]


class LesAveflowFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in AVEFLOW_CELL + AVEFLOW_COL]


class LesRefineMetrics(C.Structure):
    _fields_ = [("rhsav", C.c_double), ("pav", C.c_double), ("rel_initial", C.c_double),
                ("rel_final", C.c_double), ("outer", C.c_int)]


class LesSynthCfg(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int),
                ("dx", C.c_float), ("dy", C.c_float), ("dz0", C.c_float), ("dz_growth", C.c_float),
                ("plan_area", C.c_float), ("foot_min", C.c_int), ("foot_max", C.c_int),
                ("h_mean", C.c_float), ("h_sigma_ln", C.c_float), ("h_min", C.c_float),
                ("h_max", C.c_float), ("ustar", C.c_float), ("z0", C.c_float),
                ("kappa", C.c_float), ("noise", C.c_float), ("seed", C.c_uint64)]


class LesError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"les status {status}: {msg}")
        self.status = status


_lib = None

_P = C.c_void_p
_I = C.POINTER(C.c_int)
_F = C.POINTER(C.c_float)

_SIGS = {
    "les_last_error_string": (C.c_char_p, []),
    "les_version": (C.c_char_p, []),
    "les_params_default": (C.c_int, [C.POINTER(LesParams), C.c_int, C.c_int, C.c_int]),
    "les_ctx_create": (C.c_int, [C.POINTER(LesParams), C.POINTER(C.c_void_p)]),
    "les_ctx_destroy": (C.c_int, [_P]),
    "les_ctx_upload": (C.c_int, [_P, C.POINTER(LesHostFields)]),
    "les_ctx_download": (C.c_int, [_P, C.POINTER(LesHostFields)]),
    "les_ctx_warmup": (C.c_int, [_P, C.c_int]),
    "les_step": (C.c_int, [_P, C.c_int, C.c_int]),
    "les_set_wind_profile": (C.c_int, [_P, _P]),
    "les_ctx_sync": (C.c_int, [_P]),
    "les_last_metrics": (C.c_int, [_P, C.POINTER(LesMetrics)]),
    "les_ctx_stream": (C.c_void_p, [_P]),
    "les_ctx_field_sums": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "les_ctx_launch_count": (C.c_uint64, [_P]),
    "les_ctx_set_timing": (C.c_int, [_P, C.c_int]),
    "les_ctx_set_sor_path": (C.c_int, [_P, C.c_int]),
    "les_ctx_set_reduction_mode": (C.c_int, [_P, C.c_int]),
    "les_bounds_violations": (C.c_int, [C.POINTER(C.c_ulonglong), _I]),
    "les_ctx_sor_iters_per_launch": (C.c_float, [_P]),
    "les_ctx_sor_tile": (C.c_int, [_P, _I, _I]),
    "les_ctx_sor_shape": (C.c_int, [_P, _I, _I, _I, _I]),
    "les_ctx_sor_rows": (C.c_int, [_P, _I]),
    "les_ctx_phase_times": (C.c_int, [_P, C.c_int, _F, C.c_int]),
    "les_ctx_field": (C.c_int, [_P, C.c_int, C.POINTER(C.c_void_p), _I, _I, _I, _I]),
    "les_ctx_halo_floats": (C.c_size_t, [_P, C.c_int]),
    "les_ctx_halo_read": (C.c_int, [_P, C.c_int, _P]),
    "les_ctx_halo_write": (C.c_int, [_P, C.c_int, _P]),
    "les_halo_buffer_floats": (C.c_size_t, [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int]),
    "les_halo_pack": (C.c_int, [_P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _P]),
    "les_halo_unpack": (C.c_int, [_P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _P]),
    "les_halo_pack_inner": (C.c_int, [_P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _P]),
    "les_halo_unpack_inner": (C.c_int, [_P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _P]),
    **{f"les_halo_{op}_{v}": (C.c_int, [_P, _P, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, _P])
       for op in ("pack", "unpack", "pack_inner", "unpack_inner") for v in (1, 2, 4, 16)},
    "les_grid_metrics": (C.c_int, [C.c_int, C.c_int, C.c_int] + [_P] * 9),
    "les_poisson_coeffs": (C.c_int, [C.c_int, C.c_int, C.c_int] + [_P] * 10),
    "les_building_masks": (C.c_int, [C.c_int, C.c_int, C.c_int] + [_P] * 7),
    "les_synth_default": (None, [C.POINTER(LesSynthCfg), C.c_int, C.c_int, C.c_int, C.c_uint64]),
    "les_synth_grid": (C.c_int, [C.POINTER(LesSynthCfg)] + [_P] * 9),
    "les_synth_terrain": (C.c_float, [C.POINTER(LesSynthCfg), _P]),
    "les_synth_inflow": (C.c_int, [C.POINTER(LesSynthCfg), _P, _P, _P]),
    "les_press_rhs_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int] + [_P] * 10 + [C.c_float, _P, _P]),
    "les_aveflow": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_char_p, C.c_char_p]),
    "les_aveflow_upload": (C.c_int, [_P, C.POINTER(LesAveflowFields)]),
    "les_aveflow_download": (C.c_int, [_P, C.POINTER(LesAveflowFields)]),
    "les_write_restart": (C.c_int, [_P, C.c_char_p, C.c_char_p, _P]),
    "les_read_restart": (C.c_int, [_P, C.c_char_p, C.c_char_p, _I, _F, _P]),
    "les_ensemble_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "les_ensemble_step": (C.c_int, [_P, C.c_int, C.c_int]),
    "les_ensemble_sync": (C.c_int, [_P]),
    "les_ensemble_stream": (C.c_void_p, [_P]),
    "les_ensemble_tune_info": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
    "les_ensemble_launch_count": (C.c_uint64, [_P]),
    "les_ensemble_destroy": (C.c_int, [_P]),
    "les_press_refine_fp64": (C.c_int, [_P, C.c_int, C.c_int, C.c_double]),
    "les_netcdf_open": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "les_netcdf_write": (C.c_int, [_P, _P, C.c_int]),
    "les_netcdf_write_host": (C.c_int, [_P, C.c_int] + [_P] * 7),
    "les_netcdf_close": (C.c_int, [_P]),
    "les_last_refine_metrics": (C.c_int, [_P, C.POINTER(LesRefineMetrics)]),
    "les_ctx_set_drag": (C.c_int, [_P, _P]),
    "les_adj_create": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "les_adj_destroy": (C.c_int, [_P]),
    "les_adj_save": (C.c_int, [_P, C.c_int]),
    "les_adj_load": (C.c_int, [_P, C.c_int]),
    "les_adj_zero": (C.c_int, [_P]),
    "les_adj_tke": (C.c_int, [_P, C.c_int, _P, C.POINTER(C.c_double)]),
    "les_adj_seed_tke": (C.c_int, [_P, C.c_int, _P, C.c_double]),
    "les_adj_step_b": (C.c_int, [_P, C.c_int, C.c_int]),
    "les_adj_read": (C.c_int, [_P, _P, _P, C.POINTER(LesHostFields)]),
    "les_adj_write": (C.c_int, [_P, C.POINTER(LesHostFields)]),
    "les_dd_area_part": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_ulonglong), C.POINTER(C.c_longlong), _I]),
    "les_dd_set_owned": (C.c_int, [_P, C.c_int, C.c_int, C.c_ulonglong, C.c_longlong, C.c_int]),
    "les_dd_block_floats": (C.c_longlong, [_P, C.c_uint, C.c_int]),
    "les_dd_pack": (C.c_int, [_P, C.c_uint, C.c_int, C.c_int, _P]),
    "les_dd_unpack": (C.c_int, [_P, C.c_uint, C.c_int, C.c_int, _P]),
    "les_dd_sums": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "les_dd_phase": (C.c_int, [_P, C.c_int, C.c_int]),
    "les_dd_local_sum": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
}

# Per-routine entries: every argument is a pointer (Fortran by-reference).
ROUTINES = {
    "les_velnw_": 15, "les_bondv1_": 11, "les_bondv1_ext_wind_profile_": 12, "les_velfg_": 44,
    "les_feedbf_": 21, "les_les_": 20, "les_boundsm_": 4, "les_adam_": 11, "les_press_": 25,
    "les_bondfg_": 6, "les_boundp1_": 4, "les_boundp2_": 4,
    "les_press_rhsav_": 15, "les_press_sor_sweep_": 14, "les_press_residual_": 13, "les_press_pav_adj_": 8,
    "les_aveflow_": 32, "les_press_b_": 24,
    "les_velnw_b_": 15, "les_feedbf_b_": 21, "les_adam_b_": 11, "les_les_b_": 28,
}


def lib():
    """The loaded library; raises if it was never built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} not built: run __graft_entry__.build() or python -m les_halo_b200.build")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        for name, nargs in ROUTINES.items():
            fn = getattr(L, name, None)
            if fn is not None:
                fn.restype = C.c_int
                fn.argtypes = [_P] * nargs
        _lib = L
    return _lib


def check(status: int):
    if status != LES_OK:
        raise LesError(status, lib().les_last_error_string().decode())
