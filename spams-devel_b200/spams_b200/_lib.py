"""ctypes bindings of libspams_b200.so (the C ABI in include/spams_b200.h).

The library is loaded from spams-devel_b200/lib/ (built in-tree by
spams-devel_b200/build.py).  There is no CPU fallback: a missing library is an
ImportError, a missing GPU an error status from every coding call.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libspams_b200.so")

SC_OK = 0
SC_ERR_INVALID_ARG = 1
SC_ERR_DIMENSIONS = 2
SC_ERR_NO_CRITERION = 3
SC_ERR_CUDA = 4
SC_ERR_OUT_OF_MEMORY = 5
SC_ERR_NO_DEVICE = 6
SC_ERR_CAPACITY = 7
SC_ERR_TIMEOUT = 8
SC_ERR_UNSUPPORTED = 9

SC_L1COEFFS, SC_L2ERROR, SC_PENALTY = 0, 1, 2
SC_PREC_FP32, SC_PREC_BF16X3 = 0, 1
SC_KERNEL_AUTO, SC_KERNEL_WARP, SC_KERNEL_CTA = 0, 1, 2

# every entry point the header declares (checked by the CPU test suite)
EXPORTS = (
    "sc_version", "sc_last_error", "sc_device_count", "sc_csc_free_f32", "sc_csc_free_f64",
    "sc_release_all", "sc_omp_f32", "sc_omp_f64", "sc_lasso_f32", "sc_lasso_f64",
    "sc_lasso_gram_f32", "sc_lasso_gram_f64", "sc_lasso_gram_chol_f32",
    "sc_lasso_gram_chol_f64", "sc_omp_f32_dev", "sc_lasso_f32_dev",
    "sc_last_profile", "sc_corr_f32_dev", "sc_corr_bf16x3_noalloc_f32",
    "sc_server_create", "sc_server_destroy", "sc_server_add_dictionary_f32",
    "sc_server_remove_dictionary", "sc_server_submit", "sc_server_wait", "sc_server_replay",
    "sc_server_stats_get", "sc_dl_create", "sc_dl_destroy", "sc_dl_step_f32", "sc_dl_codes",
    "sc_dl_profile", "sc_omp_mask_f32", "sc_omp_mask_f64", "sc_lasso_mask_f32",
    "sc_lasso_mask_f64",
)

SC_REQ_OMP, SC_REQ_LASSO = 0, 1
SC_REQ_DISCARD = 1


class CscF32(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
                ("colptr", C.POINTER(C.c_int64)), ("rows", C.POINTER(C.c_int32)),
                ("vals", C.POINTER(C.c_float))]


class CscF64(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
                ("colptr", C.POINTER(C.c_int64)), ("rows", C.POINTER(C.c_int32)),
                ("vals", C.POINTER(C.c_double))]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("profile", C.c_int),
                ("refine", C.c_int), ("kernel", C.c_int), ("refactor", C.c_int),
                ("reserved", C.c_int * 2)]


class Profile(C.Structure):
    _fields_ = [("ms_gram", C.c_double), ("ms_norms", C.c_double), ("ms_corr", C.c_double),
                ("ms_code", C.c_double), ("ms_refine", C.c_double), ("ms_csc", C.c_double),
                ("ms_total", C.c_double),
                ("launches", C.c_int64), ("signals", C.c_int64), ("steps", C.c_int64),
                ("overflowed", C.c_int64), ("kernel", C.c_int32), ("lcap", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(C.Structure):
    _fields_ = [("dict_id", C.c_int64), ("algo", C.c_int), ("X", C.c_void_p), ("n", C.c_int64),
                ("L", C.c_int), ("eps", C.c_float), ("lambda1", C.c_float), ("mode", C.c_int),
                ("pos", C.c_int), ("precision", C.c_int), ("refine", C.c_int), ("flags", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("signals", C.c_int64), ("batches", C.c_int64),
                ("rejected", C.c_int64), ("pending", C.c_int64),
                ("lat_p50_ms", C.c_double), ("lat_p99_ms", C.c_double),
                ("lat_mean_ms", C.c_double), ("lat_max_ms", C.c_double), ("busy_s", C.c_double),
                ("peak_device_bytes", C.c_int64), ("mean_batch_requests", C.c_double),
                ("last_error", C.c_char * 256)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["last_error"] = self.last_error.decode(errors="replace")
        return d


class ScError(RuntimeError):
    """A non-OK status from the engine; `.status` holds the sc_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python spams-devel_b200/build.py` "
            "(the engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    p = C.c_void_p
    i32, i64 = C.c_int, C.c_int64
    f32p, f64p = C.POINTER(C.c_float), C.POINTER(C.c_double)
    i32p, i64p = C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    f, d = C.c_float, C.c_double
    opt = C.POINTER(Options)
    sigs = {
        "sc_version": (C.c_char_p, []),
        "sc_last_error": (C.c_char_p, []),
        "sc_device_count": (i32, [C.POINTER(C.c_int)]),
        "sc_csc_free_f32": (None, [C.POINTER(CscF32)]),
        "sc_csc_free_f64": (None, [C.POINTER(CscF64)]),
        "sc_release_all": (None, []),
        "sc_last_profile": (i32, [C.POINTER(Profile)]),
        "sc_omp_f32": (i32, [f32p, i32, i64, f32p, i32, i32p, i64, f32p, i64, f32p, i64, i32,
                             f32p, opt, C.POINTER(CscF32)]),
        "sc_omp_f64": (i32, [f64p, i32, i64, f64p, i32, i32p, i64, f64p, i64, f64p, i64, i32,
                             f64p, opt, C.POINTER(CscF64)]),
        "sc_lasso_f32": (i32, [f32p, i32, i64, f32p, i32, i32, f, f, i32, i32, i32, i32, i32, i32,
                               f32p, opt, C.POINTER(CscF32)]),
        "sc_lasso_f64": (i32, [f64p, i32, i64, f64p, i32, i32, d, d, i32, i32, i32, i32, i32, i32,
                               f64p, opt, C.POINTER(CscF64)]),
        "sc_lasso_gram_f32": (i32, [f32p, i32, i64, f32p, i32, f32p, i32, f, f, i32, i32, i32, i32,
                                    f32p, opt, C.POINTER(CscF32)]),
        "sc_lasso_gram_f64": (i32, [f64p, i32, i64, f64p, i32, f64p, i32, d, d, i32, i32, i32, i32,
                                    f64p, opt, C.POINTER(CscF64)]),
        "sc_lasso_gram_chol_f32": (i32, [f32p, i32, i64, f32p, i32, f32p, i32, f, f, i32, i32,
                                         i32, i32, i32, i32, f32p, opt, C.POINTER(CscF32)]),
        "sc_lasso_gram_chol_f64": (i32, [f64p, i32, i64, f64p, i32, f64p, i32, d, d, i32, i32,
                                         i32, i32, i32, i32, f64p, opt, C.POINTER(CscF64)]),
        "sc_omp_f32_dev": (i32, [p, i32, i64, p, i32, i32, f, f, p, p, p, p, p, p, i64, i64p, p,
                                 opt]),
        "sc_lasso_f32_dev": (i32, [p, i32, i64, p, i32, i32, f, f, i32, i32, i32, p, p, p, i64,
                                   i64p, p, opt]),
        "sc_corr_f32_dev": (i32, [p, i32, i32, p, i64, p, i32, i32, p]),
        "sc_corr_bf16x3_noalloc_f32": (i32, [p, i32, i32, p, i64, p, i32, p]),
        "sc_server_create": (i32, [i32, i64, i32, i64, C.POINTER(p)]),
        "sc_server_destroy": (i32, [p]),
        "sc_server_add_dictionary_f32": (i32, [p, i64, f32p, i32, i32]),
        "sc_server_remove_dictionary": (i32, [p, i64]),
        "sc_server_submit": (i32, [p, C.POINTER(Request), i64p]),
        "sc_server_wait": (i32, [p, i64, d, C.POINTER(CscF32), C.POINTER(C.c_double)]),
        "sc_server_replay": (i32, [p, C.POINTER(Request), f64p, i64]),
        "sc_server_stats_get": (i32, [p, i32, C.POINTER(ServerStats)]),
        "sc_dl_create": (i32, [i32, i32, i32, i32, i32, f, f, i32, i32, C.POINTER(p)]),
        "sc_dl_destroy": (i32, [p]),
        "sc_dl_step_f32": (i32, [p, p, p, i64, p, p, p, p, f, f, p]),
        "sc_dl_codes": (i32, [p, C.POINTER(p), C.POINTER(p), C.POINTER(p)]),
        "sc_dl_profile": (i32, [p, i32]),
        "sc_omp_mask_f32": (i32, [f32p, i32, i64, f32p, i32, C.POINTER(C.c_uint8), i32p, i64, f32p, i64, f32p,
                                  i64, i32, f32p, opt, C.POINTER(CscF32)]),
        "sc_omp_mask_f64": (i32, [f64p, i32, i64, f64p, i32, C.POINTER(C.c_uint8), i32p, i64, f64p, i64, f64p,
                                  i64, i32, f64p, opt, C.POINTER(CscF64)]),
        "sc_lasso_mask_f32": (i32, [f32p, i32, i64, f32p, i32, C.POINTER(C.c_uint8), i32, f, f, i32, i32, i32,
                                    opt, C.POINTER(CscF32)]),
        "sc_lasso_mask_f64": (i32, [f64p, i32, i64, f64p, i32, C.POINTER(C.c_uint8), i32, d, d, i32, i32, i32,
                                    opt, C.POINTER(CscF64)]),
    }
    missing = sorted(set(EXPORTS) - set(sigs))
    if missing:  # every exported entry point is called with a declared signature
        raise ImportError(f"spams_b200: no ctypes signature for {missing}")
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    s = lib().sc_last_error()
    return s.decode() if s else ""


def check(status: int) -> None:
    if status != SC_OK:
        raise ScError(status, last_error())


def last_profile() -> dict:
    """Profile of this thread's last coding call (stage times need profile=1)."""
    p = Profile()
    check(lib().sc_last_profile(C.byref(p)))
    return p.as_dict()


def device_count() -> int:
    c = C.c_int(0)
    st = lib().sc_device_count(C.byref(c))
    return c.value if st == SC_OK else 0
