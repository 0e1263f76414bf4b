"""ctypes binding of libpcomgpu.so (include/pcom_gpu.h, include/pcom_host.h).

The library is the product: there is no CPU fallback.  If the shared object
is missing this module raises, and every compute call goes to the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

dbl_p = C.POINTER(C.c_double)
i32_p = C.POINTER(C.c_int32)

PCOM_OK = 0
ERRORS = {1: "PCOM_ERR_ARG", 2: "PCOM_ERR_CUDA", 3: "PCOM_ERR_STATE", 4: "PCOM_ERR_NUMERIC", 5: "PCOM_ERR_TIMEOUT"}
PCOM_PREC_FP64 = 0x0
PCOM_PREC_MIXED = 0x1
PCOM_LIT_R8 = 0x10
PCOM_MODEL_HOST_ONLY = 0x100


class Dims(C.Structure):
    _fields_ = [("glo_ni", C.c_int32), ("glo_nj", C.c_int32), ("nk", C.c_int32), ("ni", C.c_int32),
                ("nj", C.c_int32), ("dtbt", C.c_int32), ("dtbc", C.c_int32), ("flags", C.c_int32),
                ("rst", C.c_int32), ("reserved", C.c_int32 * 3)]


class Static(C.Structure):
    _fields_ = [("rh", dbl_p * 4), ("tn", dbl_p * 4), ("dx", dbl_p * 4),
                ("z1", dbl_p), ("pr1", dbl_p), ("dz1", dbl_p), ("dpr1", dbl_p),
                ("z2", dbl_p), ("pr2", dbl_p), ("dz2", dbl_p), ("dpr2", dbl_p),
                ("msk_t", i32_p), ("lev_t", i32_p), ("msk_u", i32_p), ("lev_u", i32_p),
                ("phih_t", dbl_p), ("prh_t", dbl_p), ("phih_u", dbl_p), ("prh_u", dbl_p),
                ("cv1", dbl_p), ("cv2", dbl_p), ("cor", dbl_p), ("km", dbl_p), ("kh", dbl_p),
                ("graphihx", dbl_p), ("graphihy", dbl_p)]


STATE_FIELDS = ["tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "auc", "aup", "aupp", "avc", "avp", "avpp",
                "ubc", "vbc", "ubp", "vbp", "chc", "chp", "mch", "mch2", "am", "prho", "alpha", "adp", "wm"]


class State(C.Structure):
    _fields_ = [(n, dbl_p) for n in STATE_FIELDS]


class Forcing(C.Structure):
    _fields_ = [(n, dbl_p) for n in ("taux", "tauy", "t", "s", "pa", "fw")]


ACCUM_FIELDS = ["act", "acs", "acr", "acu", "acv", "acw", "acch", "acssh"]


class Accum(C.Structure):
    _fields_ = [(n, dbl_p) for n in ACCUM_FIELDS] + [(n, C.c_int32) for n in ("n_ts", "n_uv", "n_w", "n_ch", "n_ssh")]


class CnnStats(C.Structure):
    _fields_ = [("in_mean", C.c_float * 5), ("in_std", C.c_float * 5), ("out_std", C.c_float * 4),
                ("out_gain", C.c_float * 4), ("out_clip", C.c_float), ("alpha_ref", C.c_double * 64)]


class TropIO(C.Structure):
    _fields_ = [("glo_ni", C.c_int32), ("glo_nj", C.c_int32), ("dtbt", C.c_int32), ("dtbc", C.c_int32),
                ("flags", C.c_int32), ("lev_t", C.c_void_p), ("lev_u", C.c_void_p),
                ("prh_t", C.c_void_p), ("prh_u", C.c_void_p), ("cor", C.c_void_p), ("am1", C.c_void_p),
                ("graphihx", C.c_void_p), ("graphihy", C.c_void_p),
                ("dxx", C.c_void_p * 4), ("dxy", C.c_void_p * 4), ("rh", C.c_void_p * 4),
                ("ut", C.c_void_p), ("vt", C.c_void_p), ("bphi", C.c_void_p * 4), ("bgraphi", C.c_void_p * 4),
                ("chc", C.c_void_p), ("chp", C.c_void_p), ("mch", C.c_void_p), ("mch2", C.c_void_p),
                ("ubc", C.c_void_p), ("vbc", C.c_void_p), ("ubp", C.c_void_p), ("vbp", C.c_void_p),
                ("acch", C.c_void_p)]


class Case(C.Structure):
    _fields_ = [("glo_ni", C.c_int32), ("glo_nj", C.c_int32), ("nk", C.c_int32), ("dtbt", C.c_int32),
                ("dtbc", C.c_int32), ("r8", C.c_int32), ("rst", C.c_int32), ("year", C.c_int32),
                ("month", C.c_int32), ("day", C.c_int32), ("hour", C.c_int32),
                ("lon", dbl_p), ("lat", dbl_p), ("z", dbl_p), ("tmn", dbl_p), ("smn", dbl_p), ("itn", i32_p),
                ("pt", dbl_p), ("sa", dbl_p), ("taux", dbl_p), ("tauy", dbl_p), ("bct", dbl_p), ("bcs", dbl_p),
                ("pa", dbl_p), ("fw", dbl_p), ("vmix", dbl_p)]


# name -> (restype, argtypes) for every entry point declared in include/*.h
SIGNATURES = {
    "pcom_gpu_create": (C.c_int, [C.POINTER(Dims), C.POINTER(C.c_void_p)]),
    "pcom_gpu_destroy": (C.c_int, [C.c_void_p]),
    "pcom_gpu_upload_static": (C.c_int, [C.c_void_p, C.POINTER(Static)]),
    "pcom_gpu_set_state": (C.c_int, [C.c_void_p, C.POINTER(State)]),
    "pcom_gpu_get_state": (C.c_int, [C.c_void_p, C.POINTER(State)]),
    "pcom_gpu_set_forcing": (C.c_int, [C.c_void_p, C.POINTER(Forcing)]),
    "pcom_gpu_get_accum": (C.c_int, [C.c_void_p, C.POINTER(Accum)]),
    "pcom_gpu_reset_accum": (C.c_int, [C.c_void_p]),
    "pcom_gpu_den_prho": (C.c_int, [C.c_void_p]),
    "pcom_gpu_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "pcom_gpu_step_async": (C.c_int, [C.c_void_p, C.c_int64]),
    "pcom_gpu_phase": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64]),
    "pcom_gpu_get_field": (C.c_int, [C.c_void_p, C.c_char_p, dbl_p, C.c_int64]),
    "pcom_gpu_field_size": (C.c_int64, [C.c_void_p, C.c_char_p]),
    "pcom_gpu_field_ptr": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int32)]),
    "pcom_gpu_set_rows": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "pcom_gpu_check_finite": (C.c_int, [C.c_void_p]),
    "pcom_gpu_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pcom_gpu_sync": (C.c_int, [C.c_void_p]),
    "pcom_gpu_trop_floor": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "pcom_gpu_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcom_gpu_profile_read": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64), dbl_p, C.c_int32]),
    "pcom_gpu_launch_count": (C.c_int64, [C.c_void_p]),
    "pcom_gpu_last_error": (C.c_int, [C.c_char_p, C.c_int32]),
    "pcom_gpu_trop_noalloc": (C.c_int, [C.POINTER(TropIO), C.c_void_p]),
    "pcom_gpu_global_sums": (C.c_int, [C.c_void_p, dbl_p]),
    "pcom_gpu_set_trop_kernel": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcom_gpu_set_overlap": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcom_gpu_set_wait_limit": (C.c_int, [C.c_void_p, C.c_double]),
    "pcom_gpu_set_forcing_async": (C.c_int, [C.c_void_p, C.POINTER(Forcing)]),
    "pcom_gpu_get_state_async": (C.c_int, [C.c_void_p, C.POINTER(State)]),
    "pcom_gpu_set_forcing_months": (C.c_int, [C.c_void_p, C.POINTER(Forcing)]),
    "pcom_gpu_int_bnd": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double]),
    "pcom_gpu_coarsen": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "pcom_gpu_cnn_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pcom_gpu_cnn_target": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "pcom_gpu_cnn_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "pcom_gpu_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    "pcom_gpu_batch_destroy": (C.c_int, [C.c_void_p]),
    "pcom_gpu_batch_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "pcom_gpu_batch_step_async": (C.c_int, [C.c_void_p, C.c_int64]),
    "pcom_gpu_batch_den_prho": (C.c_int, [C.c_void_p]),
    "pcom_gpu_batch_sync": (C.c_int, [C.c_void_p]),
    "pcom_gpu_batch_set_tiles": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "pcom_gpu_batch_launch_count": (C.c_int64, [C.c_void_p]),
    "pcom_gpu_batch_use_graphs": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcom_gpu_batch_autotune": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    # closure network (include/pcom_cnn.h)
    "pcom_cnn_last_error": (C.c_int, [C.c_char_p, C.c_int32]),
    "pcom_cnn_param_count": (C.c_int64, []),
    "pcom_cnn_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "pcom_cnn_destroy": (C.c_int, [C.c_void_p]),
    "pcom_cnn_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pcom_cnn_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "pcom_cnn_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "pcom_cnn_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pcom_cnn_forward_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pcom_cnn_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                    C.POINTER(C.c_double)]),
    "pcom_cnn_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_float,
                                      C.POINTER(C.c_double)]),
    "pcom_cnn_conv_layer": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_void_p]),
    "pcom_cnn_wgrad_layer": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "pcom_model_create": (C.c_int, [C.POINTER(Case), C.c_int32, C.POINTER(C.c_void_p)]),
    "pcom_model_destroy": (C.c_int, [C.c_void_p]),
    "pcom_model_handle": (C.c_void_p, [C.c_void_p]),
    "pcom_model_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "pcom_model_begin_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pcom_model_end_step": (C.c_int, [C.c_void_p]),
    "pcom_model_run_batch": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_void_p, C.c_int64]),
    "pcom_model_iter": (C.c_int64, [C.c_void_p]),
    "pcom_model_date": (C.c_int, [C.c_void_p, i32_p]),
    "pcom_model_static": (C.c_int, [C.c_void_p, C.POINTER(Static)]),
    "pcom_model_int_bnd": (C.c_int, [C.c_void_p] + [dbl_p] * 6),
    "pcom_model_initial_state": (C.c_int, [C.c_void_p, C.POINTER(State)]),
}

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libpcomgpu.so, building it first if it is missing or stale."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if build_if_missing and not _build.up_to_date():
        try:
            _build.build()
        except Exception as e:  # no nvcc: an existing library is still usable
            if not os.path.exists(path):
                raise RuntimeError(f"libpcomgpu.so is missing and could not be built: {e}") from e
    if not os.path.exists(path):
        raise RuntimeError(f"libpcomgpu.so not found at {path}; run pcom_b200.build.build()")
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class PcomError(RuntimeError):
    pass


def check(rc: int, what: str = ""):
    if rc != PCOM_OK:
        buf = C.create_string_buffer(512)
        load().pcom_gpu_last_error(buf, 512)
        raise PcomError(f"{what}: {ERRORS.get(rc, rc)}: {buf.value.decode(errors='replace')}")
