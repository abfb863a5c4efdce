"""numpy / torch front ends over the C ABI.

`omp` and `lasso` keep the signatures of SPAMS' Python API
(swig/python/spams.py:109-142 `lasso`, :167-198 `omp`) and return
scipy.sparse.csc_matrix codes; their argument checks and error messages are
the facade's (cpp_library/spams.h:107-143, 145-188, 250-293).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import scipy.sparse as ssp

from . import _lib
from ._lib import (SC_ERR_DIMENSIONS, SC_ERR_INVALID_ARG, SC_ERR_NO_CRITERION, SC_PENALTY,
                   SC_PREC_FP32, CscF32, CscF64, Options, ScError)


def _fortran(a: np.ndarray, dtype) -> np.ndarray:
    return np.asfortranarray(a, dtype=dtype)


def _dtype_of(X: np.ndarray):
    if X.dtype == np.float32:
        return np.float32
    if X.dtype == np.float64:
        return np.float64
    raise ValueError("spams_b200: X must be float32 or float64")


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


_KERNELS = {None: 0, "auto": 0, "warp": 1, "cta": 2}


def _opts(precision: Optional[int], device: int, profile: bool = False,
          refine: Optional[bool] = None, kernel: Optional[str] = None,
          refactor: Optional[str] = None) -> Options:
    o = Options()
    if refactor not in (None, "pivot", "always", "never"):
        raise ValueError("spams_b200: refactor must be 'pivot', 'always' or 'never'")
    o.refactor = {None: 0, "pivot": 0, "always": 1, "never": -1}[refactor]
    o.precision = SC_PREC_FP32 if precision is None else int(precision)
    o.device = int(device)
    o.profile = int(bool(profile))
    o.refine = 0 if refine is None else (1 if refine else -1)
    if kernel not in _KERNELS:
        raise ValueError("spams_b200: kernel must be 'auto', 'warp' or 'cta'")
    o.kernel = _KERNELS[kernel]
    return o


def _raise(status: int) -> None:
    if status == 0:
        return
    msg = _lib.last_error()
    if status in (SC_ERR_DIMENSIONS, SC_ERR_NO_CRITERION, SC_ERR_INVALID_ARG):
        raise ValueError(msg)
    raise ScError(status, msg)


class _EngineCsc:
    """Owner of an engine-allocated CSC result: numpy arrays viewing its
    arrays keep it alive, and it is handed back to sc_csc_free_* when the
    last of them goes away (no copy of the result on the way out)."""

    def __init__(self, out, f64: bool):
        self.out = out
        self.f64 = f64

    def view(self, ptr, count: int, typestr: str) -> np.ndarray:
        holder = _Holder(self, C.cast(ptr, C.c_void_p).value, count, typestr)
        return np.asarray(holder)

    def __del__(self):
        try:
            (_lib.lib().sc_csc_free_f64 if self.f64 else _lib.lib().sc_csc_free_f32)(
                C.byref(self.out))
        except Exception:
            pass


class _Holder:
    def __init__(self, owner: _EngineCsc, addr: int, count: int, typestr: str):
        self.owner = owner
        self.__array_interface__ = {"data": (addr, False), "shape": (count,),
                                    "typestr": typestr, "version": 3}


def _csc_from(out, f64: bool) -> ssp.csc_matrix:
    m, n, nnz = int(out.m), int(out.n), int(out.nnz)
    own = _EngineCsc(out, f64)
    colptr = own.view(out.colptr, n + 1, "<i8")
    if nnz > 0:
        rows = own.view(out.rows, nnz, "<i4")
        vals = own.view(out.vals, nnz, "<f8" if f64 else "<f4")
    else:
        rows = np.zeros(0, np.int32)
        vals = np.zeros(0, np.float64 if f64 else np.float32)
    # one index type for both arrays, as scipy's sparse kernels expect
    if nnz < 2**31 - 1 and max(m, n) < 2**31 - 1:
        colptr = colptr.astype(np.int32)
    else:
        rows = rows.astype(np.int64)
    a = ssp.csc_matrix((vals, rows, colptr), shape=(m, n), copy=False)
    a.has_sorted_indices = True  # rows ascend within every column
    return a


def _vec(v, dtype, n: int):
    """None -> not given; scalar -> 1 entry; array -> n entries (per signal)."""
    if v is None:
        return None, 0
    a = np.ascontiguousarray(np.atleast_1d(np.asarray(v, dtype=dtype)).ravel())
    return a, a.size


def omp(X, D, L=None, eps=None, lambda1=None, return_reg_path=False, numThreads=-1,
        precision=None, device=0, refine=None, kernel=None, refactor=None):
    """Orthogonal Matching Pursuit of every column of X on D (unit-norm atoms).

    Mirrors spams.omp (swig/python/spams.py:167-198): L / eps / lambda1 are
    scalars or per-signal arrays; at least one must be given.  Returns a
    K x n csc_matrix, and the K x min(m,K) path of the first signal when
    return_reg_path is set."""
    dt = _dtype_of(np.asarray(X))
    X = _fortran(X, dt)
    D = _fortran(D, dt)
    if X.ndim != 2 or D.ndim != 2 or X.shape[0] != D.shape[0]:
        raise ValueError("omp : incompatible matrix dimensions")
    m, n = X.shape
    K = D.shape[1]
    Lv, nL = _vec(L, np.int32, n)
    ev, nE = _vec(eps, dt, n)
    lv, nLa = _vec(lambda1, dt, n)
    path = np.zeros((K, min(m, K)), dtype=dt, order="F") if return_reg_path else None
    f64 = dt == np.float64
    out = CscF64() if f64 else CscF32()
    ct = C.c_double if f64 else C.c_float
    fn = _lib.lib().sc_omp_f64 if f64 else _lib.lib().sc_omp_f32
    o = _opts(precision, device, refine=refine, kernel=kernel, refactor=refactor)
    st = fn(_ptr(X, ct), m, n, _ptr(D, ct), K, _ptr(Lv, C.c_int32), nL, _ptr(ev, ct), nE,
            _ptr(lv, ct), nLa, numThreads, _ptr(path, ct), C.byref(o), C.byref(out))
    _raise(st)
    alpha = _csc_from(out, f64)
    return (alpha, path) if return_reg_path else alpha


def lasso(X, D=None, Q=None, q=None, return_reg_path=False, L=-1, lambda1=None, lambda2=0.,
          mode=SC_PENALTY, pos=False, ols=False, numThreads=-1, max_length_path=-1,
          verbose=False, cholesky=False, precision=None, device=0, refine=None,
          kernel=None, refactor=None):
    """LARS-Lasso of every column of X (swig/python/spams.py:109-142).

    mode 0: ||a||_1 <= lambda1; 1: ||x - D a||^2 <= lambda1; 2 (default):
    0.5 ||x - D a||^2 + lambda1 ||a||_1 (+ 0.5 lambda2 ||a||^2).  With Q and q
    the products D^T D and D^T X are given instead of D."""
    if Q is not None:
        if q is None:
            raise ValueError("lasso : q is needed when Q is given")
    elif D is None:
        raise ValueError("lasso : you must give D or Q and q")
    if lambda1 is None:
        raise ValueError("lasso : lambda1 must be defined")
    dt = _dtype_of(np.asarray(X))
    X = _fortran(X, dt)
    m, n = X.shape
    f64 = dt == np.float64
    ct = C.c_double if f64 else C.c_float
    out = CscF64() if f64 else CscF32()
    o = _opts(precision, device, refine=refine, kernel=kernel, refactor=refactor)
    if Q is not None:
        Q = _fortran(Q, dt)
        q = _fortran(q, dt)
        if Q.shape[0] != Q.shape[1]:
            raise ValueError("lasso : Q must be square")
        K = Q.shape[0]
        if q.shape[0] != K or q.shape[1] != n:
            raise ValueError("lasso : incompatible matrix dimensions")
    else:
        D = _fortran(D, dt)
        if D.shape[0] != m:
            raise ValueError("lasso : incompatible matrix dimensions")
        K = D.shape[1]
    L0 = K if L < 0 else L
    mlp = 4 * L0 if max_length_path < 0 else max_length_path
    path = np.zeros((K, max(mlp, 0)), dtype=dt, order="F") if return_reg_path else None
    if Q is not None and (ols or cholesky):
        fn = _lib.lib().sc_lasso_gram_chol_f64 if f64 else _lib.lib().sc_lasso_gram_chol_f32
        st = fn(_ptr(X, ct), m, n, _ptr(Q, ct), K, _ptr(q, ct), int(L), float(lambda1),
                float(lambda2), int(mode), int(bool(pos)), int(bool(ols)), int(bool(cholesky)),
                numThreads, int(max_length_path), _ptr(path, ct), C.byref(o), C.byref(out))
    elif Q is not None:
        fn = _lib.lib().sc_lasso_gram_f64 if f64 else _lib.lib().sc_lasso_gram_f32
        st = fn(_ptr(X, ct), m, n, _ptr(Q, ct), K, _ptr(q, ct), int(L), float(lambda1),
                float(lambda2), int(mode), int(bool(pos)), numThreads, int(max_length_path),
                _ptr(path, ct), C.byref(o), C.byref(out))
    else:
        fn = _lib.lib().sc_lasso_f64 if f64 else _lib.lib().sc_lasso_f32
        st = fn(_ptr(X, ct), m, n, _ptr(D, ct), K, int(L), float(lambda1), float(lambda2),
                int(mode), int(bool(pos)), int(bool(ols)), numThreads, int(max_length_path),
                int(bool(cholesky)), _ptr(path, ct), C.byref(o), C.byref(out))
    _raise(st)
    alpha = _csc_from(out, f64)
    return (alpha, path) if return_reg_path else alpha


def _mask_of(B, m: int, n: int, name: str) -> np.ndarray:
    B = np.asarray(B)
    if B.shape != (m, n):
        raise ValueError(f"{name} : Mash has non acceptable dimensions")
    return np.asfortranarray(B != 0, dtype=np.uint8)


def ompMask(X, D, B, L=None, eps=None, lambda1=None, return_reg_path=False, numThreads=-1,
            precision=None, device=0, kernel=None):
    """OMP of every column of X on its observed rows (swig/python/spams.py:201-232).

    B (m x n, boolean) marks the observed rows of each signal; a signal is
    coded against the rows of D its mask keeps (eps scaled by the observed
    fraction), an all-false column gives an empty code."""
    dt = _dtype_of(np.asarray(X))
    X = _fortran(X, dt)
    D = _fortran(D, dt)
    if X.ndim != 2 or D.ndim != 2 or X.shape[0] != D.shape[0]:
        raise ValueError("ompMask : incompatible matrix dimensions")
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask_of(B, m, n, "ompMask")
    if L is None and eps is None and lambda1 is None:
        raise ValueError("omp : You should either provide L, eps or lambda")
    Lv, nL = _vec(L, np.int32, n)
    ev, nE = _vec(eps, dt, n)
    lv, nLa = _vec(lambda1, dt, n)
    path = np.zeros((K, min(m, K)), dtype=dt, order="F") if return_reg_path else None
    f64 = dt == np.float64
    out = CscF64() if f64 else CscF32()
    ct = C.c_double if f64 else C.c_float
    fn = _lib.lib().sc_omp_mask_f64 if f64 else _lib.lib().sc_omp_mask_f32
    o = _opts(precision, device, kernel=kernel)
    st = fn(_ptr(X, ct), m, n, _ptr(D, ct), K, _ptr(Bm, C.c_uint8), _ptr(Lv, C.c_int32), nL,
            _ptr(ev, ct), nE, _ptr(lv, ct), nLa, numThreads, _ptr(path, ct), C.byref(o),
            C.byref(out))
    _raise(st)
    alpha = _csc_from(out, f64)
    return (alpha, path) if return_reg_path else alpha


def lassoMask(X, D, B, L=-1, lambda1=None, lambda2=0., mode=SC_PENALTY, pos=False,
              numThreads=-1, verbose=False, precision=None, device=0, kernel=None):
    """LARS-Lasso of every column of X on its observed rows
    (swig/python/spams.py:144-153): B (m x n, boolean) marks the observed rows;
    PENALTY / L2ERROR constraints scale by the observed fraction."""
    if lambda1 is None:
        raise ValueError("lassoMask : lambda1 must be defined")
    dt = _dtype_of(np.asarray(X))
    X = _fortran(X, dt)
    D = _fortran(D, dt)
    if X.ndim != 2 or D.ndim != 2 or X.shape[0] != D.shape[0]:
        raise ValueError("lassoMask : incompatible matrix dimensions")
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask_of(B, m, n, "lassoMask")
    f64 = dt == np.float64
    out = CscF64() if f64 else CscF32()
    ct = C.c_double if f64 else C.c_float
    fn = _lib.lib().sc_lasso_mask_f64 if f64 else _lib.lib().sc_lasso_mask_f32
    o = _opts(precision, device, kernel=kernel)
    st = fn(_ptr(X, ct), m, n, _ptr(D, ct), K, _ptr(Bm, C.c_uint8), int(L), float(lambda1),
            float(lambda2), int(mode), int(bool(pos)), numThreads, C.byref(o), C.byref(out))
    _raise(st)
    return _csc_from(out, f64)


# ---------------------------------------------------------------------------
# device-resident front ends (torch CUDA tensors in and out)

def _clamp_lasso_L(m: int, K: int, L: int, lambda1: float, lambda2: float, mode: int,
                   pos: bool) -> int:
    if L < 0:
        L = K
    if L > m and not (mode == SC_PENALTY and abs(lambda1) < 1e-99 and not pos and lambda2 > 0):
        L = m
    return min(L, K)


def lasso_device(X, D, lambda1, L=-1, lambda2=0.0, mode=SC_PENALTY, pos=False,
                 max_length_path=-1, stream=None, precision=None, out=None, sync=True,
                 profile=False, refine=None, kernel=None):
    """LARS-Lasso with X (m x n) and D (m x K) as column-major float32 CUDA
    tensors (i.e. the .t() views of row-major n x m / K x m tensors, or any
    tensor whose column j is contiguous).  Returns (colptr, rows, vals, nnz)
    CUDA tensors; nnz is None when sync is False."""
    import torch
    assert X.is_cuda and D.is_cuda and X.dtype == torch.float32 and D.dtype == torch.float32
    m, n = X.shape
    K = D.shape[1]
    _check_colmajor(X)
    _check_colmajor(D)
    Lc = _clamp_lasso_L(m, K, int(L), float(lambda1), float(lambda2), int(mode), bool(pos))
    cap = max(1, n * max(Lc, 0))
    if out is None:
        out = (torch.empty(n + 1, dtype=torch.int64, device=X.device),
               torch.empty(cap, dtype=torch.int32, device=X.device),
               torch.empty(cap, dtype=torch.float32, device=X.device))
    colptr, rows, vals = out
    nnz = C.c_int64(0)
    s = stream if stream is not None else torch.cuda.current_stream(X.device)
    o = _opts(precision, X.device.index or 0, profile, refine, kernel)
    st = _lib.lib().sc_lasso_f32_dev(
        C.c_void_p(X.data_ptr()), m, n, C.c_void_p(D.data_ptr()), K, int(L), float(lambda1),
        float(lambda2), int(mode), int(bool(pos)), int(max_length_path),
        C.c_void_p(colptr.data_ptr()), C.c_void_p(rows.data_ptr()), C.c_void_p(vals.data_ptr()),
        rows.numel(), C.byref(nnz) if sync else None, C.c_void_p(s.cuda_stream), C.byref(o))
    _raise(st)
    return colptr, rows, vals, (int(nnz.value) if sync else None)


def omp_device(X, D, L=None, eps=None, lambda1=None, L_vec=None, eps_vec=None,
               lambda_vec=None, stream=None, precision=None, out=None, sync=True,
               profile=False, refine=None, kernel=None):
    """OMP with CUDA tensors (see lasso_device).  Scalars L / eps / lambda1
    follow the facade defaults; *_vec are optional per-signal CUDA tensors
    (int32 / float32) of n entries, with L then the maximum of L_vec."""
    import torch
    assert X.is_cuda and D.is_cuda and X.dtype == torch.float32 and D.dtype == torch.float32
    m, n = X.shape
    K = D.shape[1]
    _check_colmajor(X)
    _check_colmajor(D)
    if L is None and eps is None and lambda1 is None and L_vec is None and eps_vec is None \
            and lambda_vec is None:
        raise ValueError("omp : You should either provide L, eps or lambda")
    if L is None:
        L = int(L_vec.max().item()) if L_vec is not None else min(m, K)
    Lc = min(m, min(int(L), K))
    cap = max(1, n * max(Lc, 0))
    if out is None:
        out = (torch.empty(n + 1, dtype=torch.int64, device=X.device),
               torch.empty(cap, dtype=torch.int32, device=X.device),
               torch.empty(cap, dtype=torch.float32, device=X.device))
    colptr, rows, vals = out
    nnz = C.c_int64(0)
    s = stream if stream is not None else torch.cuda.current_stream(X.device)
    o = _opts(precision, X.device.index or 0, profile, refine, kernel)

    def vp(t):
        return C.c_void_p(t.data_ptr()) if t is not None else None

    st = _lib.lib().sc_omp_f32_dev(
        C.c_void_p(X.data_ptr()), m, n, C.c_void_p(D.data_ptr()), K, int(L),
        float(eps or 0.0), float(lambda1 or 0.0), vp(L_vec), vp(eps_vec), vp(lambda_vec),
        C.c_void_p(colptr.data_ptr()), C.c_void_p(rows.data_ptr()), C.c_void_p(vals.data_ptr()),
        rows.numel(), C.byref(nnz) if sync else None, C.c_void_p(s.cuda_stream), C.byref(o))
    _raise(st)
    return colptr, rows, vals, (int(nnz.value) if sync else None)


def _check_colmajor(t) -> None:
    if t.dim() != 2 or t.stride(0) != 1 or t.stride(1) != t.shape[0]:
        raise ValueError("spams_b200: device matrices must be dense column-major "
                         "(stride (1, rows))")


def corr_device(D, X, precision=None, out=None, stream=None):
    """Correlations D^T X for column-major float32 CUDA tensors D (m x K) and
    X (m x n); returns a K x n column-major tensor (a .t() view)."""
    import torch
    _check_colmajor(X)
    _check_colmajor(D)
    m, K = D.shape
    n = X.shape[1]
    if X.shape[0] != m:
        raise ValueError("corr : incompatible matrix dimensions")
    res = out if out is not None else torch.empty((n, K), dtype=torch.float32, device=X.device).t()
    s = stream if stream is not None else torch.cuda.current_stream(X.device)
    st = _lib.lib().sc_corr_f32_dev(
        C.c_void_p(D.data_ptr()), m, K, C.c_void_p(X.data_ptr()), n, C.c_void_p(res.data_ptr()),
        res.stride(1), SC_PREC_FP32 if precision is None else int(precision),
        C.c_void_p(s.cuda_stream))
    _raise(st)
    return res
