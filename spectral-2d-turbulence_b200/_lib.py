"""ctypes binding of libs2d.so (the C ABI declared in include/s2d.h).

The library is the product: there is no fallback.  Importing this module
without a built ``libs2d.so`` raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libs2d.so")

S2D_OK = 0
S2D_NO_DATA = 1
S2D_ERR_ARG = -1
S2D_ERR_UNSUPPORTED_N = -2
S2D_ERR_CUDA = -3
S2D_ERR_DESTROYED = -4
S2D_ERR_NAN = -5
S2D_ERR_UNREGISTERED = -6
S2D_ERR_NO_DEVICE = -7

S2D_MAX_SPLATS = 8
S2D_STEP_DYE = 1
S2D_STEP_REDUCE = 2
S2D_STEP_RELATCH = 4
S2D_FFT_FP32 = 0
S2D_FFT_TC_F16 = 1
S2D_FFT_TC_BF16 = 2
S2D_DYE_NONE = 0
S2D_DYE_BANDS = 1
S2D_SCENARIO_SHEAR_LAYER = 0
S2D_SCENARIO_TAYLOR_GREEN = 1
S2D_SCENARIO_DIPOLE = 2
S2D_SCENARIO_MERGER = 3
S2D_SCENARIO_POLYGON = 4
S2D_SCENARIO_MAX_BLOBS = 256
RENDER_MODES = ["dye", "vorticity", "dye over vorticity", "speed"]     # render.js:4

BUFFER_IDS = {
    "state0": 0, "state1": 1, "state2": 2, "packA": 3, "packB": 4, "physZ": 5,
    "rhs": 6, "force": 7, "vel": 8, "dt": 9,
}


class s2d_params(C.Structure):
    _fields_ = [("beta", C.c_float), ("drag", C.c_float), ("viscosity", C.c_float),
                ("hyper_p", C.c_int32), ("force_amp", C.c_float), ("force_k", C.c_float),
                ("force_width", C.c_float), ("cfl", C.c_float), ("dt_min", C.c_float),
                ("dt_max", C.c_float), ("dye_fade", C.c_float)]


class s2d_splat(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("dx", C.c_float), ("dy", C.c_float),
                ("color", C.c_float * 3), ("radius", C.c_float), ("amp", C.c_float),
                ("dye_amp", C.c_float)]


S2D_TUNE_MAX = 8


class s2d_tune_report(C.Structure):
    _fields_ = [("phys_variants", C.c_int32), ("spec_variants", C.c_int32), ("phys_choice", C.c_int32),
                ("spec_choice", C.c_int32), ("phys_us", C.c_float * S2D_TUNE_MAX),
                ("spec_us", C.c_float * S2D_TUNE_MAX)]


class s2d_info(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("nbins", C.c_int32), ("phase", C.c_int32),
                ("dye_parity", C.c_int32), ("step_index", C.c_uint32), ("primed", C.c_int32),
                ("fft_precision", C.c_int32), ("nu_h", C.c_float), ("sim_time", C.c_double)]


class s2d_instance_desc(C.Structure):
    _fields_ = [("n", C.c_int32), ("beta", C.c_float), ("drag", C.c_float), ("nu_h", C.c_float),
                ("hyper_p", C.c_int32), ("dt", C.c_float), ("force_amp", C.c_float),
                ("force_k", C.c_float), ("force_width", C.c_float), ("seed", C.c_uint32)]


_vp = C.c_void_p
_i = C.c_int
_u = C.c_uint32
_f = C.c_float
_d = C.c_double
_sz = C.c_size_t

# name -> (restype, argtypes); every symbol declared in include/s2d.h
PROTOTYPES = {
    "s2d_version": (_i, []),
    "s2d_status_string": (C.c_char_p, [_i]),
    "s2d_last_error": (C.c_char_p, []),
    "s2d_radix_schedule": (_i, [_i, C.POINTER(_i), C.POINTER(_i)]),
    "s2d_supported_grids": (_i, [C.POINTER(_i), _i, C.POINTER(_i)]),
    "s2d_digit_reverse_table": (_i, [_i, C.POINTER(_u)]),
    "s2d_wavenumber_table": (_i, [_i, C.POINTER(_f)]),
    "s2d_dealias_mask_table": (_i, [_i, C.POINTER(C.c_uint8)]),
    "s2d_dye_fast_path_check": (_i, [_i, _i]),
    "s2d_create": (_i, [_i, _i, _i, _i, C.POINTER(_vp)]),
    "s2d_destroy": (_i, [_vp]),
    "s2d_get_info": (_i, [_vp, C.POINTER(s2d_info)]),
    "s2d_set_phase": (_i, [_vp, _i, _i]),
    "s2d_set_sim_time": (_i, [_vp, _d]),
    "s2d_get_stream": (_i, [_vp, C.POINTER(_vp)]),
    "s2d_synchronize": (_i, [_vp]),
    "s2d_configure": (_i, [_vp, C.POINTER(s2d_params)]),
    "s2d_set_splats": (_i, [_vp, C.POINTER(s2d_splat), _i]),
    "s2d_seed": (_i, [_vp, _d, _d, _u]),
    "s2d_seed_physical": (_i, [_vp, C.POINTER(_f)]),
    "s2d_reset": (_i, [_vp, C.POINTER(_f), _d, _d, _u, _i]),
    "s2d_paint_dye": (_i, [_vp, _i]),
    "s2d_seed_band": (_i, [_vp, _f, _f, _f, _u]),
    "s2d_scenario_field": (_i, [_vp, _i, _d, C.POINTER(_f)]),
    "s2d_reset_scenario": (_i, [_vp, _i, _d, _i]),
    "s2d_render": (_i, [_vp, _i, _f, _f, _f, _i, _i, _vp]),
    "s2d_autotune": (_i, [_vp, _i, C.POINTER(s2d_tune_report)]),
    "s2d_tune_variant_name": (_i, [_vp, _i, _i, C.c_char_p, _i]),
    "s2d_tune_select": (_i, [_vp, _i, _i]),
    "s2d_encode_prime": (_i, [_vp]),
    "s2d_encode_step": (_i, [_vp]),
    "s2d_encode_dye": (_i, [_vp]),
    "s2d_encode_dye_passes": (_i, [_vp]),
    "s2d_encode_reduce": (_i, [_vp]),
    "s2d_step": (_i, [_vp, _i, C.c_uint]),
    "s2d_step_graph": (_i, [_vp, _i, C.c_uint]),
    "s2d_encode_diagnostics": (_i, [_vp]),
    "s2d_copy_diagnostics": (_i, [_vp]),
    "s2d_poll_diagnostics": (_i, [_vp]),
    "s2d_read_diagnostics": (_i, [_vp, C.POINTER(_d), C.POINTER(_f), C.POINTER(_d), C.POINTER(_d),
                                  C.POINTER(_f), C.POINTER(_f)]),
    "s2d_read_diagnostics_fixed": (_i, [_vp, C.POINTER(_f), C.POINTER(_f), C.POINTER(_f)]),
    "s2d_get_buffer": (_i, [_vp, _i, _vp, _sz]),
    "s2d_set_buffer": (_i, [_vp, _i, _vp, _sz]),
    "s2d_fft2": (_i, [_vp, _i, _i]),
    "s2d_velocity_pack": (_i, [_vp, _i]),
    "s2d_nl_pack": (_i, [_vp]),
    "s2d_assemble": (_i, [_vp]),
    "s2d_rk3_stage": (_i, [_vp, _i]),
    "s2d_get_dye": (_i, [_vp, C.POINTER(C.c_uint16)]),
    "s2d_set_dye": (_i, [_vp, C.POINTER(C.c_uint16)]),
    "s2d_profile": (_i, [_vp, _i]),
    "s2d_profile_read": (_i, [_vp, C.POINTER(_d), C.POINTER(_i)]),
    "s2d_cfl_dt_static": (_i, [_vp, _i, _f, _f, _f, _vp, _vp]),
    "s2d_probe_wait_timeout": (_i, [_vp, C.c_ulonglong]),
    "s2d_ensemble_create": (_i, [C.POINTER(s2d_instance_desc), _i, _i, C.POINTER(_vp)]),
    "s2d_ensemble_destroy": (_i, [_vp]),
    "s2d_ensemble_get_stream": (_i, [_vp, C.POINTER(_vp)]),
    "s2d_ensemble_synchronize": (_i, [_vp]),
    "s2d_ensemble_seed_band": (_i, [_vp, _f, _f, _f]),
    "s2d_ensemble_set_state": (_i, [_vp, _i, C.POINTER(_f)]),
    "s2d_ensemble_get_state": (_i, [_vp, _i, C.POINTER(_f)]),
    "s2d_ensemble_step": (_i, [_vp, _i, _i]),
    "s2d_ensemble_autotune": (_i, [_vp, _i, C.POINTER(s2d_tune_report)]),
    "s2d_ensemble_tune_variant_name": (_i, [_vp, _i, _i, C.c_char_p, _i]),
    "s2d_ensemble_tune_select": (_i, [_vp, _i, _i]),
    "s2d_ensemble_energy": (_i, [_vp, C.POINTER(_d), C.POINTER(_d)]),
}


class S2DError(RuntimeError):
    """A negative status from the C ABI (the JS facade throws an Error there)."""

    def __init__(self, status: int, func: str, message: str):
        super().__init__(f"{func}: {message} (status {status})")
        self.status = status


_LIB = None


def lib():
    """Load libs2d.so once; raise if it was never built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python {os.path.join(PKG_DIR, 'build.py')}` "
                "(CUDA toolkit with sm_100a support required)")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def check(status: int, func: str) -> int:
    if status < 0:
        msg = lib().s2d_last_error().decode(errors="replace") or lib().s2d_status_string(status).decode()
        raise S2DError(status, func, msg)
    return status


def call(name: str, *args) -> int:
    return check(getattr(lib(), name)(*args), name)
