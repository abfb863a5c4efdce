"""The oracle (test infrastructure only): CPU ground truth for the coding path.

Two implementations, both CPU-only:
  * ``ref_*``  - the SPAMS reference's own omp / lasso facade compiled from its
    header sources into oracle/_ref/libspams_ref.so (oracle/build_ref.sh,
    FP64 or FP32 templates, OpenMP + OpenBLAS).
  * ``orc_*``  - the plain-C restatement in oracle/sc_oracle_impl.h
    (oracle/liborc.so), pinned against ``ref_*`` through tests/golden/.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The shipped engine never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as ssp

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_SO = os.path.join(HERE, "liborc.so")
REF_SO = os.path.join(HERE, "_ref", "libspams_ref.so")
# The reference checkout: SPAMS_REFERENCE_DIR (or build_ref's argument).
REFERENCE_DIR = os.environ.get("SPAMS_REFERENCE_DIR")


def build_orc() -> str:
    src = [os.path.join(HERE, "sc_oracle.c"), os.path.join(HERE, "sc_oracle_impl.h")]
    if not os.path.exists(ORC_SO) or any(os.path.getmtime(s) > os.path.getmtime(ORC_SO) for s in src):
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", src[0], "-o", ORC_SO, "-lm"],
                       check=True)
    return ORC_SO


def build_ref(reference_dir: str | None = REFERENCE_DIR) -> str | None:
    """Compile oracle/_ref from the reference sources when they are present.

    ``reference_dir`` (or SPAMS_REFERENCE_DIR) names the checkout; without
    either nothing is built.  The script exits 2 when
    it finds no sources, and an existing build is then kept as it is.
    """
    deps = [os.path.join(HERE, "ref_driver.cpp"), os.path.join(HERE, "build_ref.sh")]
    fresh = os.path.exists(REF_SO) and all(os.path.getmtime(d) <= os.path.getmtime(REF_SO) for d in deps)
    if fresh:
        return REF_SO
    cmd = ["bash", os.path.join(HERE, "build_ref.sh")] + ([reference_dir] if reference_dir else [])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode == 2:
        return REF_SO if os.path.exists(REF_SO) else None
    if r.returncode != 0:
        raise RuntimeError(f"build_ref.sh failed:\n{r.stderr[-2000:]}")
    return REF_SO


def have_ref() -> bool:
    return os.path.exists(REF_SO)


class _RefCsc(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
                ("colptr", C.POINTER(C.c_int64)), ("rows", C.POINTER(C.c_int32)),
                ("vals", C.c_void_p), ("err", C.c_char * 128)]


_ref = None
_orc = None


def _ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: run oracle/build_ref.sh")
        # one OpenBLAS thread per OpenMP thread, as the reference's build notes ask
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        _ref = C.CDLL(REF_SO)
        _ref.ref_free.argtypes = [C.c_void_p]
    return _ref


def _orc_lib():
    global _orc
    if _orc is None:
        build_orc()
        _orc = C.CDLL(ORC_SO)
    return _orc


def _f(a, dt):
    return np.asfortranarray(a, dtype=dt)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _csc_out(out: _RefCsc, dt) -> ssp.csc_matrix:
    if out.err:
        raise ValueError(out.err.decode())
    n, nnz = int(out.n), int(out.nnz)
    colptr = np.ctypeslib.as_array(out.colptr, shape=(n + 1,)).copy()
    rows = np.ctypeslib.as_array(out.rows, shape=(max(nnz, 1),))[:nnz].copy()
    vals = np.ctypeslib.as_array(C.cast(out.vals, C.POINTER(C.c_double if dt == np.float64 else C.c_float)),
                                 shape=(max(nnz, 1),))[:nnz].copy()
    lib = _ref_lib()
    for p in (C.cast(out.colptr, C.c_void_p), C.cast(out.rows, C.c_void_p), out.vals):
        lib.ref_free(p)
    return ssp.csc_matrix((vals, rows, colptr), shape=(int(out.m), n))


def ref_omp(X, D, L=None, eps=None, lambda1=None, numThreads=-1, return_reg_path=False):
    """The reference _omp<T> (cpp_library/spams.h:250-293) on X, D."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]

    def vec(v, t):
        if v is None:
            return None, 0
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(v, dtype=t)).ravel())
        return a, a.size
    Lv, nL = vec(L, np.int32)
    ev, nE = vec(eps, dt)
    lv, nLa = vec(lambda1, dt)
    path = np.zeros((K, min(m, K)), dtype=dt, order="F") if return_reg_path else None
    lib = _ref_lib()
    fn = lib.ref_omp_f64 if dt == np.float64 else lib.ref_omp_f32
    out = _RefCsc()
    fn(_p(X), C.c_int(m), C.c_int(n), _p(D), C.c_int(K), _p(Lv), C.c_int(nL), _p(ev), C.c_int(nE),
       _p(lv), C.c_int(nLa), C.c_int(numThreads), _p(path), C.byref(out))
    a = _csc_out(out, dt)
    return (a, path) if return_reg_path else a


def ref_lasso(X, D=None, Q=None, q=None, L=-1, lambda1=0.0, lambda2=0.0, mode=2, pos=False,
              ols=False, cholesky=False, numThreads=-1, max_length_path=-1, return_reg_path=False):
    """The reference _lassoD<T> / _lassoQq<T> (cpp_library/spams.h:107-188)."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X = _f(X, dt)
    m, n = X.shape
    lib = _ref_lib()
    out = _RefCsc()
    if Q is not None:
        Q, q = _f(Q, dt), _f(q, dt)
        K = Q.shape[0]
    else:
        D = _f(D, dt)
        K = D.shape[1]
    L0 = K if L < 0 else L
    mlp = 4 * L0 if max_length_path < 0 else max_length_path
    path = np.zeros((K, max(mlp, 0)), dtype=dt, order="F") if return_reg_path else None
    ct = C.c_double if dt == np.float64 else C.c_float
    if Q is not None:
        fn = lib.ref_lassoQq_f64 if dt == np.float64 else lib.ref_lassoQq_f32
        fn(_p(X), C.c_int(m), C.c_int(n), _p(Q), C.c_int(K), _p(q), C.c_int(L), ct(lambda1),
           C.c_int(mode), C.c_int(int(pos)), C.c_int(int(ols)), C.c_int(int(cholesky)),
           C.c_int(numThreads), C.c_int(max_length_path), _p(path), C.byref(out))
    else:
        fn = lib.ref_lasso_f64 if dt == np.float64 else lib.ref_lasso_f32
        fn(_p(X), C.c_int(m), C.c_int(n), _p(D), C.c_int(K), C.c_int(L), ct(lambda1), ct(lambda2),
           C.c_int(mode), C.c_int(int(pos)), C.c_int(int(ols)), C.c_int(int(cholesky)),
           C.c_int(numThreads), C.c_int(max_length_path), _p(path), C.byref(out))
    a = _csc_out(out, dt)
    return (a, path) if return_reg_path else a


def ref_dl_minibatch(D, X, perm, it, batch, lambda1, A, B, beta=1.0, gamma=1.0, numThreads=-1):
    """One minibatch of the reference's online dictionary learning (coding and
    accumulations, dictLearn/dicts.h:526-603, PENALTY mode) in float32: A and
    B (Fortran float32 arrays K x K and m x K) are updated in place."""
    D = _f(D, np.float32)
    X = _f(X, np.float32)
    perm = np.ascontiguousarray(perm, np.int32)
    m, K = D.shape
    assert A.dtype == np.float32 and A.flags.f_contiguous and A.shape == (K, K)
    assert B.dtype == np.float32 and B.flags.f_contiguous and B.shape == (m, K)
    lib = _ref_lib()
    lib.ref_dl_minibatch_f32(_p(D), C.c_int(m), C.c_int(K), _p(X), C.c_int(X.shape[1]), _p(perm),
                             C.c_int(it), C.c_int(batch), C.c_float(lambda1), C.c_int(numThreads),
                             _p(A), _p(B), C.c_float(beta), C.c_float(gamma))


# ---------------------------------------------------------------------------
# the C restatement

def _convert(vM, rM, L, n, K, dt) -> ssp.csc_matrix:
    lib = _orc_lib()
    fn = lib.orc_convert_f64 if dt == np.float64 else lib.orc_convert_f32
    fn.restype = C.c_int64
    colptr = np.zeros(n + 1, np.int64)
    rows = np.zeros(max(1, L * n), np.int32)
    vals = np.zeros(max(1, L * n), dt)
    nnz = fn(_p(vM), _p(rM), C.c_int(L), C.c_int64(n), _p(colptr), _p(rows), _p(vals))
    return ssp.csc_matrix((vals[:nnz], rows[:nnz], colptr), shape=(K, n))


def orc_omp(X, D, L=None, eps=None, lambda1=None, return_reg_path=False):
    """C restatement of _omp / omp / coreORMP (same facade defaults)."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]
    if L is None and eps is None and lambda1 is None:
        raise ValueError("omp : You should either provide L, eps or lambda")
    Lv = np.atleast_1d(np.asarray(min(m, K) if L is None else L, np.int32)).ravel().copy()
    ev = np.atleast_1d(np.asarray(0.0 if eps is None else eps, dt)).ravel().copy()
    lv = np.atleast_1d(np.asarray(0.0 if lambda1 is None else lambda1, dt)).ravel().copy()
    Ld = int(Lv.max()) if Lv.size > 1 else int(Lv[0])
    if Ld <= 0:
        a = ssp.csc_matrix((0, 0), dtype=dt)
        return (a, np.zeros((K, min(m, K)), dt, order="F")) if return_reg_path else a
    Lc = min(m, min(Ld, K))
    vM = np.zeros(max(1, Lc * n), dt)
    rM = np.full(max(1, Lc * n), -1, np.int32)
    path = np.zeros((K, min(m, K)), dt, order="F") if return_reg_path else None
    lib = _orc_lib()
    fn = lib.orc_omp_f64 if dt == np.float64 else lib.orc_omp_f32
    fn(_p(X), C.c_int(m), C.c_int64(n), _p(D), C.c_int(K), _p(Lv), C.c_int(Lv.size), _p(ev),
       C.c_int(ev.size), _p(lv), C.c_int(lv.size), _p(vM), _p(rM), _p(path), C.c_int(0))
    a = _convert(vM, rM, Lc, n, K, dt)
    return (a, path) if return_reg_path else a


def orc_lasso(X, D, L=-1, lambda1=0.0, lambda2=0.0, mode=2, pos=False, max_length_path=-1,
              return_reg_path=False, ols=False, cholesky=False, Q=None, q=None):
    """C restatement of _lassoD / _lassoQq: lasso2 / coreLARS2, or with
    cholesky / ols the Cholesky implementation lasso<T> / coreLARS +
    downDateLasso (decomp/decomp.h:735-1203).  With Q and q the products are
    given (Q used as given, X supplies ||x||^2); D is then unused."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X = _f(X, dt)
    m, n = X.shape
    if Q is not None:
        Q, q = _f(Q, dt), _f(q, dt)
        K = Q.shape[0]
    else:
        D = _f(D, dt)
        K = D.shape[1]
    lib = _orc_lib()
    ct = C.c_double if dt == np.float64 else C.c_float
    clamp = lib.orc_lasso_clamp_f64 if dt == np.float64 else lib.orc_lasso_clamp_f32
    mlp = C.c_int(max_length_path)
    Lc = clamp(C.c_int(m), C.c_int(K), C.c_int(L), ct(lambda1), ct(lambda2), C.c_int(mode),
               C.c_int(int(pos)), C.byref(mlp))
    path = np.zeros((K, max(mlp.value, 0)), dt, order="F") if return_reg_path else None
    if Lc <= 0:
        a = ssp.csc_matrix((0, 0), dtype=dt)
        return (a, path) if return_reg_path else a
    vM = np.zeros(max(1, Lc * n), dt)
    rM = np.full(max(1, Lc * n), -1, np.int32)
    if ols or cholesky or Q is not None:
        if not (ols or cholesky):
            raise NotImplementedError("the restatement takes (Q, q) with the Cholesky variant; "
                                      "the homotopy computes its products from D")
        fn = lib.orc_lasso_chol_f64 if dt == np.float64 else lib.orc_lasso_chol_f32
        fn(_p(X), C.c_int(m), C.c_int64(n), _p(D) if Q is None else None,
           _p(Q) if Q is not None else None, _p(q) if Q is not None else None, C.c_int(K),
           C.c_int(Lc), ct(lambda1), ct(lambda2), C.c_int(mode), C.c_int(int(pos)),
           C.c_int(int(bool(ols))), C.c_int(mlp.value), _p(vM), _p(rM), _p(path))
    else:
        fn = lib.orc_lasso_f64 if dt == np.float64 else lib.orc_lasso_f32
        fn(_p(X), C.c_int(m), C.c_int64(n), _p(D), C.c_int(K), C.c_int(Lc), ct(lambda1),
           ct(lambda2), C.c_int(mode), C.c_int(int(pos)), C.c_int(mlp.value), _p(vM), _p(rM),
           _p(path))
    a = _convert(vM, rM, Lc, n, K, dt)
    return (a, path) if return_reg_path else a


def _mask(B, m, n):
    B = np.asarray(B)
    if B.shape != (m, n):
        raise ValueError("ompMask : Mash has non acceptable dimensions")
    return np.asfortranarray(B != 0, dtype=np.uint8)


def ref_omp_mask(X, D, B, L=None, eps=None, lambda1=None, numThreads=-1, return_reg_path=False):
    """The reference _ompMask<T> (cpp_library/spams.h:296-343) on X, D, B."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask(B, m, n)

    def vec(v, t):
        if v is None:
            return None, 0
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(v, dtype=t)).ravel())
        return a, a.size
    Lv, nL = vec(L, np.int32)
    ev, nE = vec(eps, dt)
    lv, nLa = vec(lambda1, dt)
    path = np.zeros((K, min(m, K)), dtype=dt, order="F") if return_reg_path else None
    lib = _ref_lib()
    fn = lib.ref_omp_mask_f64 if dt == np.float64 else lib.ref_omp_mask_f32
    out = _RefCsc()
    fn(_p(X), C.c_int(m), C.c_int(n), _p(D), C.c_int(K), _p(Bm), _p(Lv), C.c_int(nL), _p(ev),
       C.c_int(nE), _p(lv), C.c_int(nLa), C.c_int(numThreads), _p(path), C.byref(out))
    a = _csc_out(out, dt)
    return (a, path) if return_reg_path else a


def ref_lasso_mask(X, D, B, L=-1, lambda1=0.0, lambda2=0.0, mode=2, pos=False, numThreads=-1):
    """The reference _lassoMask<T> (cpp_library/spams.h:191-214) on X, D, B."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask(B, m, n)
    ct = C.c_double if dt == np.float64 else C.c_float
    lib = _ref_lib()
    fn = lib.ref_lasso_mask_f64 if dt == np.float64 else lib.ref_lasso_mask_f32
    out = _RefCsc()
    fn(_p(X), C.c_int(m), C.c_int(n), _p(D), C.c_int(K), _p(Bm), C.c_int(L), ct(lambda1),
       ct(lambda2), C.c_int(mode), C.c_int(int(pos)), C.c_int(numThreads), C.byref(out))
    return _csc_out(out, dt)


def orc_omp_mask(X, D, B, L=None, eps=None, lambda1=None, return_reg_path=False):
    """C restatement of _ompMask / omp_mask (same facade defaults)."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask(B, m, n)
    if L is None and eps is None and lambda1 is None:
        raise ValueError("omp : You should either provide L, eps or lambda")
    Lv = np.atleast_1d(np.asarray(min(m, K) if L is None else L, np.int32)).ravel().copy()
    ev = np.atleast_1d(np.asarray(0.0 if eps is None else eps, dt)).ravel().copy()
    lv = np.atleast_1d(np.asarray(0.0 if lambda1 is None else lambda1, dt)).ravel().copy()
    Ld = int(Lv.max()) if Lv.size > 1 else int(Lv[0])
    if Ld <= 0:
        a = ssp.csc_matrix((0, 0), dtype=dt)
        return (a, np.zeros((K, min(m, K)), dt, order="F")) if return_reg_path else a
    Lc = min(m, min(Ld, K))
    vM = np.zeros(max(1, Lc * n), dt)
    rM = np.full(max(1, Lc * n), -1, np.int32)
    path = np.zeros((K, min(m, K)), dt, order="F") if return_reg_path else None
    lib = _orc_lib()
    fn = lib.orc_omp_mask_f64 if dt == np.float64 else lib.orc_omp_mask_f32
    fn(_p(X), C.c_int(m), C.c_int64(n), _p(D), C.c_int(K), _p(Bm), _p(Lv), C.c_int(Lv.size),
       _p(ev), C.c_int(ev.size), _p(lv), C.c_int(lv.size), _p(vM), _p(rM), _p(path))
    a = _convert(vM, rM, Lc, n, K, dt)
    return (a, path) if return_reg_path else a


def orc_lasso_mask(X, D, B, L=-1, lambda1=0.0, lambda2=0.0, mode=2, pos=False):
    """C restatement of _lassoMask / lasso_mask (including the reference's
    L explicit zeros at row 0 for a column with no observed row)."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X, D = _f(X, dt), _f(D, dt)
    m, n = X.shape
    K = D.shape[1]
    Bm = _mask(B, m, n)
    lib = _orc_lib()
    ct = C.c_double if dt == np.float64 else C.c_float
    clamp = lib.orc_lasso_clamp_f64 if dt == np.float64 else lib.orc_lasso_clamp_f32
    mlp = C.c_int(-1)
    Lc = clamp(C.c_int(m), C.c_int(K), C.c_int(L), ct(lambda1), ct(lambda2), C.c_int(mode),
               C.c_int(int(pos)), C.byref(mlp))
    if Lc <= 0:
        return ssp.csc_matrix((0, 0), dtype=dt)
    vM = np.zeros(max(1, Lc * n), dt)
    rM = np.zeros(max(1, Lc * n), np.int32)
    fn = lib.orc_lasso_mask_f64 if dt == np.float64 else lib.orc_lasso_mask_f32
    fn(_p(X), C.c_int(m), C.c_int64(n), _p(D), C.c_int(K), _p(Bm), C.c_int(Lc), ct(lambda1),
       ct(lambda2), C.c_int(mode), C.c_int(int(pos)), _p(vM), _p(rM))
    return _convert(vM, rM, Lc, n, K, dt)
