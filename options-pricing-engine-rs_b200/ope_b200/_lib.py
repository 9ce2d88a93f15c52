"""ctypes loader for libope_b200.so (the sm_100a product library).

There is no CPU fallback: if the shared library is missing or cannot be
loaded this module raises, and every pricing call fails loudly.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libope_b200.so")

OPE_OK = 0
STATUS_NAMES = {
    0: "OPE_OK",
    1: "OPE_ERR_INVALID_ARG",
    2: "OPE_ERR_OUT_OF_MEMORY",
    3: "OPE_ERR_DEVICE",
    4: "OPE_ERR_NO_DEVICE",
    5: "OPE_ERR_TIMEOUT",
    6: "OPE_ERR_REJECTED",
    7: "OPE_ERR_CANCELLED",
    8: "OPE_ERR_NOT_FOUND",
}
FLAG_DEVICE_PTRS = 1
FLAG_ANALYTIC_GREEKS = 2
MODEL_HESTON, MODEL_BATES = 0, 1


class OpeError(RuntimeError):
    """A non-zero status from the C ABI (the reference would panic here)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class Options(ctypes.Structure):
    _fields_ = [
        ("tol", ctypes.c_double),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("stream", ctypes.c_void_p),
    ]


# Exported symbols and their signatures; the CPU tests check that every
# symbol declared in include/ope.h is exported by the built library.
_SIGS: dict = {}


def _sig(name, res, args):
    _SIGS[name] = (res, args)


_vp, _d, _i32, _sz, _u64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int32, ctypes.c_size_t, ctypes.c_uint64
_sig("ope_last_error", ctypes.c_char_p, [])
_sig("ope_version", ctypes.c_char_p, [])
_sig("ope_kernel_launch_count", _u64, [])
_sig("ope_set_workspace_limit", ctypes.c_int, [_u64])
_sig("ope_workspace_bytes", _u64, [])
_sig("ope_check_word", ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_i32)])
_sig("ope_device_info", ctypes.c_int, [ctypes.POINTER(_i32)] * 3)
_sig("ope_heston_price", ctypes.c_int, [_d, _d, _d, _d, _d, _vp, _i32, ctypes.POINTER(_d)])
_sig("ope_bates_price", ctypes.c_int, [_d, _d, _d, _d, _d, _vp, _i32, ctypes.POINTER(_d)])
_sig("ope_batch_heston", ctypes.c_int, [_vp, _sz, _vp, _vp])
_sig("ope_batch_bates", ctypes.c_int, [_vp, _sz, _vp, _vp])
_sig("ope_batch_heston_greeks", ctypes.c_int, [_vp, _sz, _vp, _vp])
_sig("ope_batch_bates_greeks", ctypes.c_int, [_vp, _sz, _vp, _vp])
_sig("ope_batch_price_ex", ctypes.c_int, [_i32, _vp, _sz, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_batch_greeks_ex", ctypes.c_int, [_i32, _vp, _sz, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_batch_greeks_ad", ctypes.c_int, [_i32, _vp, _sz, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_price_surfaces", ctypes.c_int, [_i32, _vp, _sz, _vp, _sz, _vp, _vp, ctypes.POINTER(Options)])

_sig("ope_price_surfaces_stats", ctypes.c_int,
     [_i32, _vp, _sz, _vp, _sz, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_price_gradient_surfaces", ctypes.c_int,
     [_i32, _vp, _sz, _vp, _sz, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_selftest_math", ctypes.c_int, [ctypes.POINTER(_u64), ctypes.POINTER(_u64)])
_sig("ope_selftest_atan2", ctypes.c_int, [ctypes.POINTER(_u64)])
_sig("ope_selftest_log", ctypes.c_int, [ctypes.POINTER(_u64)])
_sig("ope_selftest_log_cr", ctypes.c_int, [_vp, _sz, _vp, _vp])
_sig("ope_selftest_node_u", ctypes.c_int, [ctypes.POINTER(_u64)])
_sig("ope_calibrate_surfaces", ctypes.c_int,
     [_i32, _vp, _vp, _vp, _sz, _vp, _sz, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_calibrate_surfaces_reg", ctypes.c_int,
     [_i32, _vp, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_calibrate_multistart", ctypes.c_int,
     [_i32, _vp, _vp, _vp, _sz, _vp, _sz, _vp, _i32, _u64, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_calibrate_global", ctypes.c_int,
     [_i32, _vp, _vp, _vp, _sz, _vp, _sz, _i32, _i32, _u64, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_calib_jacobian", ctypes.c_int, [_i32, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_batch_implied_vol", ctypes.c_int, [_vp, _sz, _vp, _vp, _vp, ctypes.POINTER(Options)])
_sig("ope_server_create", ctypes.c_int, [_vp, _vp])
_sig("ope_server_destroy", ctypes.c_int, [_vp])
_sig("ope_server_submit_price", ctypes.c_int, [_vp, _i32, _vp, _sz, _vp, ctypes.POINTER(_u64)])
_sig("ope_server_submit_calibrate", ctypes.c_int, [_vp, _i32, _vp, _vp, _sz, _vp, ctypes.POINTER(_u64)])
_sig("ope_server_wait", ctypes.c_int, [_vp, _u64, _d, _vp, _vp, ctypes.POINTER(_d)])
_sig("ope_server_cancel", ctypes.c_int, [_vp, _u64])
_sig("ope_server_get_stats", ctypes.c_int, [_vp, _vp])
_sig("ope_price_surfaces_noalloc", ctypes.c_int, [_i32, _vp, _sz, _vp, _sz, _vp, _vp, _d, _vp])
_sig("ope_measure_fp64_peak", ctypes.c_int, [ctypes.POINTER(_d), ctypes.POINTER(_d)])
_sig("ope_trace_integral", ctypes.c_int, [_i32, _vp, _vp, _i32, _d, _vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_d)])

class LaunchShape(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int32), ("deepest_first", ctypes.c_int32), ("occupancy", ctypes.c_double),
                ("per_unit", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class TuneEntry(ctypes.Structure):
    _fields_ = [("max_contracts", ctypes.c_uint64), ("shape", LaunchShape), ("ms_default", ctypes.c_double),
                ("ms_tuned", ctypes.c_double)]


TUNE_CLASSES = 16  # OPE_TUNE_CLASSES
TUNE_QUICK = 1    # OPE_TUNE_QUICK
_sig("ope_autotune", ctypes.c_int, [_i32, ctypes.c_uint32, ctypes.POINTER(TuneEntry)])
_sig("ope_set_autotune", ctypes.c_int, [_i32])
_sig("ope_get_tune_table", ctypes.c_int, [_i32, ctypes.POINTER(TuneEntry), ctypes.POINTER(_i32)])
_sig("ope_last_per_unit", ctypes.c_int, [ctypes.POINTER(_i32)])
_sig("ope_set_tune_table", ctypes.c_int, [_i32, ctypes.POINTER(TuneEntry)])

_lib = None


CHECKED_LIB_PATH = os.path.join(PKG_ROOT, "lib", "checked", "libope_b200.so")


def open_library(path: str) -> ctypes.CDLL:
    """A separate handle on a build of the library at `path` (e.g. the
    bounds-checked build), with the ABI signatures applied."""
    L = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return L


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(
                f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build` "
                "(or `make -C options-pricing-engine-rs_b200/csrc`); there is no CPU fallback"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OPE_OK:
        msg = load().ope_last_error()
        raise OpeError(status, msg.decode() if msg else "")


def declared_symbols(header: str) -> list[str]:
    """Names of the functions include/ope.h declares."""
    import re

    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ope_[a-z0-9_]+)\s*\(", text)))
