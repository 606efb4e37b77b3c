"""ctypes binding of liblcurve_b200.so (declarations in include/lcurve_b200.h).

The library must exist: there is no CPU fallback.  Loading fails loudly with
the build command when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
# LCB_LIBRARY selects another build of the library, e.g. the index-checking
# liblcurve_b200_bounds.so of `make bounds`
LIB_PATH = pathlib.Path(os.environ["LCB_LIBRARY"]) if os.environ.get("LCB_LIBRARY") else HERE / "liblcurve_b200.so"

LCB_OK = 0
ERR_NAMES = {
    1: "LCB_ERR_INVALID", 2: "LCB_ERR_PARSE", 3: "LCB_ERR_IO", 4: "LCB_ERR_MODEL", 5: "LCB_ERR_CUDA",
    6: "LCB_ERR_UNKNOWN_PARAM", 7: "LCB_ERR_NO_DEVICE", 8: "LCB_ERR_EMPTY", 9: "LCB_ERR_DEVICE_CHECK",
}

DATUM_DTYPE = np.dtype([("time", "<f8"), ("expose", "<f8"), ("flux", "<f8"), ("ferr", "<f8"),
                        ("weight", "<f8"), ("ndiv", "<i4"), ("pad", "<i4")])
assert DATUM_DTYPE.itemsize == 48


class Result(C.Structure):
    _fields_ = [("wdwarf", C.c_double), ("chisq", C.c_double), ("wnok", C.c_double), ("logg1", C.c_double),
                ("logg2", C.c_double), ("rv1", C.c_double), ("rv2", C.c_double), ("sfac", C.c_double * 5)]


class LcbError(RuntimeError):
    """Raised for a non-zero status of the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


SYMBOLS = [
    "lcb_version", "lcb_last_error", "lcb_device_count", "lcb_ctx_create", "lcb_ctx_destroy", "lcb_ctx_set_stream",
    "lcb_ctx_last_error", "lcb_model_load", "lcb_model_parse", "lcb_model_clone", "lcb_model_destroy",
    "lcb_model_set_param", "lcb_model_get_param", "lcb_model_get_pparam", "lcb_model_set_pparam",
    "lcb_model_set_comp", "lcb_model_get_comp", "lcb_param_name", "lcb_read_data", "lcb_free_data",
    "lcb_light_curve", "lcb_chisq_batch", "lcb_chisq_batch_ragged", "lcb_batch_create", "lcb_batch_destroy",
    "lcb_batch_set_params", "lcb_batch_run", "lcb_batch_results", "lcb_batch_stats", "lcb_batch_profile", "lcb_batch_stage_ms",
    "lcb_ctx_transfer_bytes", "lcb_measure_fma_peak", "lcb_model_grid", "lcb_batch_search_counts",
    "lcb_light_curve_noalloc", "lcb_batch_set_tuning", "lcb_batch_get_tuning", "lcb_ctx_set_search_cap",
    "lcb_wait_probe", "lcb_model_work", "lcb_model_elements", "lcb_light_curve_elements", "lcb_stream_points",
    # surrogate (lcurve_b200_surrogate.h)
    "lcb_mlp_last_error", "lcb_mlp_create", "lcb_mlp_destroy", "lcb_mlp_set_stream", "lcb_mlp_num_params",
    "lcb_mlp_get_params", "lcb_mlp_set_params", "lcb_mlp_get_grads", "lcb_mlp_forward", "lcb_mlp_backward",
    "lcb_mlp_train_step", "lcb_mlp_grads_device", "lcb_mlp_adam_step", "lcb_mlp_take_loss", "lcb_mlp_sync",
    "lcb_mlp_gemm", "lcb_logflux_chisq", "lcb_surrogate_subchain", "lcb_surrogate_subchain_host",
    "lcb_mlp_state_size", "lcb_mlp_get_state", "lcb_mlp_set_state",
]

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing; build it with `make -C {HERE}` "
                          "(or __graft_entry__.build()). There is no CPU fallback.")
    L = C.CDLL(str(LIB_PATH))
    vp, cp, i, i64, d = C.c_void_p, C.c_char_p, C.c_int, C.c_int64, C.c_double
    dp, i64p = C.POINTER(C.c_double), C.POINTER(C.c_int64)
    sig = {
        "lcb_version": ([], cp), "lcb_last_error": ([], cp), "lcb_device_count": ([C.POINTER(i)], i),
        "lcb_ctx_create": ([i, C.POINTER(vp)], i), "lcb_ctx_destroy": ([vp], None),
        "lcb_ctx_set_stream": ([vp, vp], i), "lcb_ctx_last_error": ([vp], cp),
        "lcb_model_load": ([cp, C.POINTER(vp)], i), "lcb_model_parse": ([cp, C.POINTER(vp)], i),
        "lcb_model_clone": ([vp, C.POINTER(vp)], i), "lcb_model_destroy": ([vp], None),
        "lcb_model_set_param": ([vp, cp, d], i), "lcb_model_get_param": ([vp, cp, dp], i),
        "lcb_model_get_pparam": ([vp, cp, dp, dp, dp, C.POINTER(i), C.POINTER(i)], i),
        "lcb_model_set_pparam": ([vp, cp, dp, dp, dp, C.POINTER(i)], i),
        "lcb_model_set_comp": ([vp, cp, cp], i), "lcb_model_get_comp": ([vp, cp, cp, i], i),
        "lcb_param_name": ([i], cp),
        "lcb_read_data": ([cp, C.POINTER(vp), i64p], i), "lcb_free_data": ([vp], None),
        "lcb_light_curve": ([vp, vp, vp, i64, i, i, dp, C.POINTER(Result)], i),
        "lcb_chisq_batch": ([vp, vp, vp, i64, C.POINTER(cp), i, dp, i64, i, dp], i),
        "lcb_chisq_batch_ragged": ([vp, C.POINTER(vp), i64, vp, i64p, i, dp, dp, C.POINTER(Result)], i),
        "lcb_batch_create": ([vp, C.POINTER(vp), i64, vp, i64p, C.POINTER(vp)], i),
        "lcb_batch_destroy": ([vp], None),
        "lcb_batch_set_params": ([vp, C.POINTER(cp), i, dp], i),
        "lcb_batch_run": ([vp, i], i),
        "lcb_batch_results": ([vp, dp, dp, C.POINTER(Result)], i),
        "lcb_batch_stats": ([vp, i64p], i),
        "lcb_batch_profile": ([vp, i], i),
        "lcb_batch_stage_ms": ([vp, dp], i),
        "lcb_ctx_transfer_bytes": ([vp, i64p, i64p], i),
        "lcb_measure_fma_peak": ([vp, i, dp], i),
        "lcb_model_grid": ([vp, vp, i, i64p, dp, dp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                            C.POINTER(C.c_float), dp], i),
        "lcb_batch_search_counts": ([vp, i64p], i),
        "lcb_batch_set_tuning": ([vp, i, i, i], i),
        "lcb_batch_get_tuning": ([vp, C.POINTER(i)], i),
        "lcb_light_curve_noalloc": ([vp, vp, vp, i64, i, i, dp, C.POINTER(Result)], i),
        "lcb_ctx_set_search_cap": ([vp, i], i),
        "lcb_wait_probe": ([vp, i64, i64p], i),
        "lcb_model_work": ([vp, vp, i64, i64p], i),
        "lcb_stream_points": ([vp, dp, dp, i64, i, dp], i),
        "lcb_model_elements": ([vp, vp, i64, i64, vp, vp, vp, vp, vp, i64p], i),
        "lcb_light_curve_elements": ([vp, vp, vp, i64, i, i, vp, vp, vp, vp, vp, dp, C.POINTER(Result)], i),
        "lcb_mlp_last_error": ([], cp),
        "lcb_mlp_create": ([i, i, i, i, i, i64, C.c_uint64, C.POINTER(vp)], i),
        "lcb_mlp_destroy": ([vp], None),
        "lcb_mlp_set_stream": ([vp, vp], i),
        "lcb_mlp_num_params": ([vp, i64p], i),
        "lcb_mlp_get_params": ([vp, vp, i64], i),
        "lcb_mlp_set_params": ([vp, vp, i64], i),
        "lcb_mlp_get_grads": ([vp, vp, i64], i),
        "lcb_mlp_state_size": ([vp, i64p], i),
        "lcb_mlp_get_state": ([vp, vp, i64, i64p], i),
        "lcb_mlp_set_state": ([vp, vp, i64, i64], i),
        "lcb_mlp_forward": ([vp, vp, i64, vp], i),
        "lcb_mlp_backward": ([vp, vp, vp, i64], i),
        "lcb_mlp_train_step": ([vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float], i),
        "lcb_mlp_grads_device": ([vp, C.POINTER(C.POINTER(C.c_float)), i64p], i),
        "lcb_mlp_adam_step": ([vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float], i),
        "lcb_mlp_take_loss": ([vp, dp], i),
        "lcb_mlp_sync": ([vp], i),
        "lcb_mlp_gemm": ([i, i64, i64, i64, vp, vp, vp, vp, vp, vp, vp, vp], i),
        "lcb_logflux_chisq": ([i64, i, vp, vp, vp, vp, vp, i, vp, vp], i),
        "lcb_surrogate_subchain": ([vp, i64, i64, i, vp, vp, vp, vp, i, d, dp, dp, C.POINTER(i),
                                    C.POINTER(C.c_float), C.POINTER(C.c_float), vp, vp, vp, vp, i, i, dp, dp], i),
        "lcb_surrogate_subchain_host": ([vp, i64, i64, i, vp, vp, vp, vp, i, d, dp, dp, C.POINTER(i),
                                         C.POINTER(C.c_float), C.POINTER(C.c_float), vp, vp, vp, vp, i, i, dp, dp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != LCB_OK:
        msg = load().lcb_last_error()
        raise LcbError(rc, msg.decode() if msg else "")


def check_mlp(rc: int) -> None:
    """Status check for the surrogate entry points (their own error slot)."""
    if rc != LCB_OK:
        msg = load().lcb_mlp_last_error()
        raise LcbError(rc, msg.decode() if msg else "")


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def i64ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))
