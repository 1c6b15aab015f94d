"""ctypes binding of liblceqcd_gpu.so (the C ABI in include/lceqcd_gpu.h).

The library is the only compute path: there is no CPU fallback.  If the
shared object is missing, or no CUDA device is present when a context is
created, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblceqcd_gpu.so")

LCE_OK = 0
LCE_ERR_INVALID = -1
LCE_ERR_CUDA = -2
LCE_ERR_GF_NOT_CONVERGED = -3
LCE_ERR_STREAM = -4
LCE_ERR_NAN = -5
LCE_ERR_NOMEM = -6
LCE_ERR_UNSUPPORTED = -7

LCE_PREC_F32 = 0
LCE_PREC_F64 = 1
LCE_RNG_PHILOX = 0
LCE_RNG_STREAM = 1
LCE_GF_ACOS = 0
LCE_GF_ATAN2 = 1
LCE_SWEEP_AUTO = 0
LCE_SWEEP_PASSES = 1
LCE_SWEEP_PERSISTENT = 2
LCE_SWEEP_PASSES2 = 3
LCE_SWEEP_DIRECT = 4
LCE_FIELDS = 0
LCE_FIELDS_FIXED = 1
LCE_GF_START_IDENTITY = 0
LCE_GF_START_TRANSFORM = 1
LCE_GF_START_NET = 2
LCE_ITGF_FIX_COMPONENT = 1
LCE_ITGF_ASCEND = 2
LCE_ITGF_TRACK = 4
LCE_WARM_NET = 1
LCE_WARM_JUDGE = 2
LCE_WARM_RECORD = 4
LCE_WARM_FOURIER = 8
LCE_WARM_CG = 16


class LceParams(C.Structure):
    _fields_ = [
        ("L", C.c_int * 3),
        ("beta", C.c_double), ("x", C.c_double), ("y", C.c_double),
        ("lambda_", C.c_double), ("alpha", C.c_double), ("limit_or", C.c_double),
        ("imode", C.c_int), ("precision", C.c_int), ("rng", C.c_int),
        ("seed", C.c_ulonglong), ("device", C.c_int),
        ("n_link_or", C.c_int), ("n_higgs_metro", C.c_int),
        ("delta0", C.c_double), ("gf_angle", C.c_int), ("sweep_mode", C.c_int),
        ("agauge_hits", C.c_int), ("tile_threads", C.c_int), ("tile_registers", C.c_int),
    ]


class LceMeas(C.Structure):
    _fields_ = [
        ("plaq", C.c_double), ("akin", C.c_double), ("a2", C.c_double), ("a4", C.c_double),
        ("acc_gauge", C.c_double), ("acc_hb", C.c_double), ("acc_or", C.c_double),
        ("acc_metro", C.c_double), ("acc_link_or", C.c_double), ("delta", C.c_double),
        ("af", C.c_double * 3),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "af"}
        d["af"] = list(self.af)
        return d


# name -> (restype, argtypes); every symbol declared in include/lceqcd_gpu.h
P, I, D, F = C.c_void_p, C.c_int, C.c_double, C.c_float
SIGNATURES = {
    "lce_version": (C.c_char_p, []),
    "lce_strerror": (C.c_char_p, [I]),
    "lce_last_error": (C.c_char_p, [P]),
    "lce_default_params": (None, [P]),
    "lce_couplings": (I, [P, P]),
    "lce_geometry_tables": (I, [I, I, I, P, P]),
    "lce_create": (P, [P]),
    "lce_create_batch": (P, [P, I]),
    "lce_destroy": (None, [P]),
    "lce_nchains": (I, [P]),
    "lce_get_extents": (I, [P, I, P]),
    "lce_confsave": (I, [P, I, C.c_char_p, C.c_char_p]),
    "lce_confget": (I, [P, I, C.c_char_p, C.c_char_p]),
    "lce_conf_filename": (I, [C.c_char_p, C.c_size_t, C.c_char_p, I, D, D, D, I]),
    "lce_set_stream": (I, [P, P]),
    "lce_synchronize": (I, [P]),
    "lce_upload": (I, [P, I, I, P, P, C.c_long]),
    "lce_upload_async": (I, [P, I, I, P, P, C.c_long]),
    "lce_upload_stage": (I, [P, I, I, P, P, C.c_long]),
    "lce_upload_apply": (I, [P]),
    "lce_upload_f64": (I, [P, I, I, P, P, C.c_long]),
    "lce_download": (I, [P, I, I, P, P, C.c_long]),
    "lce_download_f64": (I, [P, I, I, P, P, C.c_long]),
    "lce_init_unit": (I, [P, D]),
    "lce_init_hot": (I, [P, C.c_ulonglong]),
    "lce_set_rng_stream": (I, [P, P, C.c_size_t]),
    "lce_get_rng_position": (I, [P, P, P]),
    "lce_set_rng_position": (I, [P, C.c_ulonglong, C.c_ulonglong]),
    "lce_ahiggs1": (I, [P, P, I, P]),
    "lce_ahiggs2": (I, [P, I, P]),
    "lce_ahiggs3": (I, [P, I, P]),
    "lce_agauge": (I, [P, I, P]),
    "lce_agauge1": (I, [P, I, P]),
    "lce_link_or": (I, [P, I, P]),
    "lce_renorm": (I, [P]),
    "lce_sweep": (I, [P, I, P]),
    "lce_sweeps": (I, [P, I, I]),
    "lce_get_sweep_mode": (I, [P]),
    "lce_get_tile_shape": (I, [P, P, P, P]),
    "lce_get_meas": (I, [P, I, P]),
    "lce_get_meas_batch": (I, [P, P]),
    "lce_landau_gauge": (I, [P, I, P, P, I]),
    "lce_gauge_fix_continue": (I, [P, I, P, P, I]),
    "lce_it_gauge_fixing": (I, [P, I, D, I, P]),
    "lce_slabs_create": (P, [P, I, P]),
    "lce_slabs_destroy": (None, [P]),
    "lce_slabs_upload": (I, [P, P, P, C.c_long]),
    "lce_slabs_upload_f64": (I, [P, P, P, C.c_long]),
    "lce_slabs_download": (I, [P, P, P, C.c_long]),
    "lce_slabs_download_f64": (I, [P, P, P, C.c_long]),
    "lce_slabs_sweep": (I, [P, I, P]),
    "lce_slabs_set_rng_stream": (I, [P, P, C.c_size_t]),
    "lce_slabs_download_fixed": (I, [P, P, P, C.c_long]),
    "lce_slabs_download_fixed_f64": (I, [P, P, P, C.c_long]),
    "lce_slabs_landau_gauge_from": (I, [P, I, P, P, I]),
    "lce_slabs_landau_gauge_fourier": (I, [P, I, D, D, P, P, P, I]),
    "lce_slabs_it_landau_gauge": (I, [P, D, I, P, P, I]),
    "lce_slabs_landau_gauge_fourier_cg": (I, [P, I, D, P, P, P, I]),
    "lce_slabs_landau_gauge": (I, [P, P, P, I]),
    "lce_slabs_correlator": (I, [P, P, P, P, P]),
    "lce_slabs_polyakov": (I, [P, P, P, P]),
    "lce_slabs_scalarcorr": (I, [P, P, P, P]),
    "lce_it_landau_gauge": (I, [P, I, D, I, P, P, I]),
    "lce_landau_gauge_from": (I, [P, I, I, P, P, P, I]),
    "lce_apply_transform": (I, [P, I]),
    "lce_landau_gauge_fourier": (I, [P, I, I, D, D, P, P, P, I]),
    "lce_landau_gauge_fourier_cg": (I, [P, I, I, D, P, P, P, I]),
    "lce_debug_fourier_step": (I, [P, I, D, P]),
    "lce_set_transform": (I, [P, I, P, C.c_long]),
    "lce_get_transform": (I, [P, I, P, C.c_long]),
    "lce_gauge_functional": (I, [P, I, P]),
    "lce_theta": (I, [P, I, P]),
    "lce_correlator": (I, [P, I, P, P, P, P]),
    "lce_polyakov": (I, [P, I, P, P, P]),
    "lce_scalarcorr": (I, [P, I, P, P, P]),
    "lce_plaquette": (I, [P, I, P]),
    "lce_debug_staple": (I, [P, I, I, P]),
    "lce_debug_force": (I, [P, I, P]),
    "lce_flush_l2": (I, [P]),
    "lce_profile_sweep": (I, [P, I, P, I]),
    "lce_timer_start": (I, [P]),
    "lce_timer_stop": (I, [P, P]),
    "lce_plaquette_noalloc": (I, [P, C.c_long, I, I, I, P, P]),
    "lce_net_create": (P, [I, C.c_ulonglong]),
    "lce_net_destroy": (None, [P]),
    "lce_net_num_params": (I, [P]),
    "lce_net_get_params": (I, [P, P]),
    "lce_net_set_params": (I, [P, P]),
    "lce_net_save": (I, [P, C.c_char_p]),
    "lce_net_load": (I, [P, C.c_char_p]),
    "lce_net_eval": (I, [P, I, I, I, P, P, P, P, P]),
    "lce_net_num_pairs": (I, [P]),
    "lce_net_clear_pairs": (I, [P]),
    "lce_net_train": (I, [P, I, D, P]),
    "lce_landau_gauge_warm": (I, [P, I, P, I, P, P, P, P, I]),
}

_lib = None


def load() -> C.CDLL:
    """Load liblceqcd_gpu.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m lceqcd_b200.build` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class LceError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def check(rc: int, ctx=None) -> int:
    if rc < 0:
        lib = load()
        detail = lib.lce_last_error(ctx).decode() if ctx is not None else ""
        raise LceError(rc, f"{lib.lce_strerror(rc).decode()}: {detail}")
    return rc
