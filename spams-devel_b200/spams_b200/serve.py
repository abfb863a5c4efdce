"""Serving loop over dictionaries kept resident on one GPU.

    with spams_b200.Server(hbm_budget=150e9, slots=3) as srv:
        srv.add_dictionary(7, D)                       # D: m x K float32
        t = srv.submit(7, X, algo="omp", L=10)         # returns at once
        alpha = srv.result(t)                          # K x n scipy CSC

Requests against the same dictionary with the same options are merged into
one GPU launch; every signal is coded exactly as spams_b200.omp / .lasso code
it in float32, whichever requests share its launch.  The loop itself (slots,
batching, admission by device-memory budget, latency accounting) is native
code behind the C ABI (sc_server_* in include/spams_b200.h).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .api import _csc_from

_ALGOS = {"omp": _lib.SC_REQ_OMP, "lasso": _lib.SC_REQ_LASSO}


def _signals(X) -> np.ndarray:
    X = np.asarray(X)
    if X.ndim != 2:
        raise ValueError("serving: X must be a matrix (m x n)")
    return np.asfortranarray(X, dtype=np.float32)


def request(dict_id: int, X: np.ndarray, algo: str = "omp", L: Optional[int] = None,
            eps: Optional[float] = None, lambda1: Optional[float] = None, mode: int = 2,
            pos: bool = False, precision: Optional[int] = None, refine: Optional[int] = None,
            discard: bool = False) -> _lib.Request:
    """The C request record for signals X (Fortran float32, kept alive by the
    caller until the request completes).  OMP: at least one of L / eps /
    lambda1 (facade defaults otherwise); Lasso: lambda1, mode, pos, L (-1 = K)."""
    if algo not in _ALGOS:
        raise ValueError(f"serving: algo must be 'omp' or 'lasso', not {algo!r}")
    if not (X.flags.f_contiguous and X.dtype == np.float32):
        raise ValueError("serving: X must be a Fortran-ordered float32 array")
    r = _lib.Request()
    r.dict_id = int(dict_id)
    r.algo = _ALGOS[algo]
    r.X = X.ctypes.data if X.size else None
    r.n = X.shape[1]
    if algo == "omp":
        if L is None and eps is None and lambda1 is None:
            raise ValueError("omp : You should either provide L, eps or lambda")
        r.L = int(L) if L is not None else 0
        r.eps = float(eps) if eps is not None else 0.0
        r.lambda1 = float(lambda1) if lambda1 is not None else 0.0
    else:
        if lambda1 is None:
            raise ValueError("lasso : lambda1 must be defined")
        r.L = int(L) if L is not None else -1
        r.lambda1 = float(lambda1)
        r.mode = int(mode)
        r.pos = int(bool(pos))
    r.precision = _lib.SC_PREC_FP32 if precision is None else int(precision)
    r.refine = int(refine or 0)
    r.flags = _lib.SC_REQ_DISCARD if discard else 0
    return r


class Server:
    """A request loop on one GPU (see the module docstring)."""

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, slots: int = 3,
                 max_batch_signals: int = 1 << 18):
        h = C.c_void_p()
        _lib.check(_lib.lib().sc_server_create(int(device), int(hbm_budget), int(slots),
                                               int(max_batch_signals), C.byref(h)))
        self._h = h
        self._keep = {}   # ticket -> signals kept alive until the result is collected
        self._dims = {}   # dictionary id -> (m, K)

    def close(self) -> None:
        if self._h:
            _lib.check(_lib.lib().sc_server_destroy(self._h))
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_dictionary(self, dict_id: int, D: np.ndarray) -> None:
        D = _signals(D)
        m, K = D.shape
        _lib.check(_lib.lib().sc_server_add_dictionary_f32(
            self._h, int(dict_id), D.ctypes.data_as(C.POINTER(C.c_float)), m, K))
        self._dims[int(dict_id)] = (m, K)

    def remove_dictionary(self, dict_id: int) -> None:
        _lib.check(_lib.lib().sc_server_remove_dictionary(self._h, int(dict_id)))
        self._dims.pop(int(dict_id), None)

    def submit(self, dict_id: int, X, algo: str = "omp", **kw) -> int:
        X = _signals(X)
        m = self._dims.get(int(dict_id), (None, None))[0]
        if m is not None and X.shape[0] != m:
            raise ValueError(f"{algo} : incompatible matrix dimensions")
        r = request(dict_id, X, algo, **kw)
        t = C.c_int64()
        _lib.check(_lib.lib().sc_server_submit(self._h, C.byref(r), C.byref(t)))
        if not (r.flags & _lib.SC_REQ_DISCARD):
            self._keep[t.value] = X
        return t.value

    def result(self, ticket: int, timeout: float = 600.0, with_latency: bool = False):
        out = _lib.CscF32()
        lat = C.c_double()
        st = _lib.lib().sc_server_wait(self._h, int(ticket), float(timeout), C.byref(out),
                                       C.byref(lat))
        if st != _lib.SC_ERR_TIMEOUT:
            self._keep.pop(int(ticket), None)
        _lib.check(st)
        a = _csc_from(out, False)
        return (a, lat.value) if with_latency else a

    def code(self, dict_id: int, X, algo: str = "omp", **kw):
        return self.result(self.submit(dict_id, X, algo, **kw))

    def replay(self, requests: Sequence[_lib.Request], arrival_s: Sequence[float]) -> None:
        """Open-loop load: request i is submitted arrival_s[i] seconds after the
        call starts; results are discarded, latencies go to stats()."""
        n = len(requests)
        arr = (_lib.Request * n)(*requests)
        t = np.ascontiguousarray(np.asarray(arrival_s, dtype=np.float64))
        if t.size != n:
            raise ValueError("serving: one arrival time per request")
        _lib.check(_lib.lib().sc_server_replay(
            self._h, arr, t.ctypes.data_as(C.POINTER(C.c_double)), n))

    def stats(self, reset: bool = False) -> dict:
        s = _lib.ServerStats()
        _lib.check(_lib.lib().sc_server_stats_get(self._h, int(bool(reset)), C.byref(s)))
        return s.as_dict()
