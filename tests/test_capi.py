"""CPU checks of the C ABI library: it loads, exports every entry point the
header declares, and fails loudly (no CPU fallback) where no GPU is present.
No compute call runs here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import spams_b200
from spams_b200 import _lib


def _declared():
    with open(os.path.join(ROOT, "include", "spams_b200.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_match_binding_list():
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name


def test_version_string():
    assert spams_b200.lib().sc_version().decode().startswith("spams_b200")


def test_no_device_is_an_error_not_a_fallback():
    if spams_b200.device_count() > 0:
        pytest.skip("a GPU is present")
    X = np.asfortranarray(np.random.randn(8, 4).astype(np.float32))
    D = np.asfortranarray(np.random.randn(8, 6).astype(np.float32))
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.lasso(X, D, lambda1=0.1)
    assert e.value.status == _lib.SC_ERR_NO_DEVICE
    with pytest.raises(spams_b200.ScError):
        spams_b200.omp(X, D, L=2)


def test_facade_argument_errors_need_no_device():
    X = np.asfortranarray(np.random.randn(8, 4))
    D = np.asfortranarray(np.random.randn(9, 6))
    with pytest.raises(ValueError, match="incompatible matrix dimensions"):
        spams_b200.omp(X, D, L=2)
    with pytest.raises(ValueError, match="incompatible matrix dimensions"):
        spams_b200.lasso(X, D, lambda1=0.1)
    D = np.asfortranarray(np.random.randn(8, 6))
    with pytest.raises(ValueError, match="either provide L, eps or lambda"):
        spams_b200.omp(X, D)
    with pytest.raises(ValueError, match="lambda1 must be defined"):
        spams_b200.lasso(X, D)
    with pytest.raises(ValueError, match="q is needed"):
        spams_b200.lasso(X, Q=np.eye(6), lambda1=0.1)
    with pytest.raises(ValueError, match="Q must be square"):
        spams_b200.lasso(X, Q=np.ones((6, 5)), q=np.ones((6, 4)), lambda1=0.1)


def test_c_abi_rejects_bad_counts_before_touching_the_device():
    lib = spams_b200.lib()
    X = np.asfortranarray(np.random.randn(8, 4).astype(np.float32))
    D = np.asfortranarray(np.random.randn(8, 6).astype(np.float32))
    L = np.array([2, 3], np.int32)  # neither 1 nor n entries
    out = _lib.CscF32()
    fp = C.POINTER(C.c_float)
    st = lib.sc_omp_f32(X.ctypes.data_as(fp), 8, 4, D.ctypes.data_as(fp), 6,
                        L.ctypes.data_as(C.POINTER(C.c_int32)), 2, None, 0, None, 0, -1, None,
                        None, C.byref(out))
    assert st == _lib.SC_ERR_INVALID_ARG
    st = lib.sc_omp_f32(X.ctypes.data_as(fp), 8, 4, D.ctypes.data_as(fp), 6, None, 0, None, 0,
                        None, 0, -1, None, None, C.byref(out))
    assert st == _lib.SC_ERR_NO_CRITERION
    assert "either provide L, eps or lambda" in _lib.last_error()


def test_dictionaries_beyond_16384_atoms_are_rejected_before_the_device():
    """Up to 1024 atoms one warp codes a signal, up to 16384 one CTA; larger
    dictionaries are refused with SC_ERR_UNSUPPORTED (not coded on the CPU)."""
    X = np.asfortranarray(np.random.randn(8, 3).astype(np.float32))
    D = np.asfortranarray(np.random.randn(8, 16385).astype(np.float32))
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.omp(X, D, L=2)
    assert e.value.status == _lib.SC_ERR_UNSUPPORTED
    assert "16384" in str(e.value)
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.lasso(X, D, lambda1=0.1)
    assert e.value.status == _lib.SC_ERR_UNSUPPORTED


def test_kernel_choice_is_validated():
    X = np.asfortranarray(np.random.randn(8, 4).astype(np.float32))
    D = np.asfortranarray(np.random.randn(8, 6).astype(np.float32))
    with pytest.raises(ValueError, match="kernel must be"):
        spams_b200.omp(X, D, L=2, kernel="block")
    o = _lib.Options()
    o.kernel = 7
    out = _lib.CscF32()
    fp = C.POINTER(C.c_float)
    st = spams_b200.lib().sc_omp_f32(X.ctypes.data_as(fp), 8, 4, D.ctypes.data_as(fp), 6,
                                     (C.c_int32 * 1)(2), 1, None, 0, None, 0, -1, None,
                                     C.byref(o), C.byref(out))
    assert st == _lib.SC_ERR_INVALID_ARG
    assert "kernel" in _lib.last_error()


def test_mask_front_ends_check_arguments_without_a_device():
    X = np.asfortranarray(np.random.randn(8, 4))
    D = np.asfortranarray(np.random.randn(8, 6))
    B = np.ones((8, 4), bool)
    with pytest.raises(ValueError, match="non acceptable dimensions"):
        spams_b200.ompMask(X, D, B[:, :3], L=2)
    with pytest.raises(ValueError, match="either provide L, eps or lambda"):
        spams_b200.ompMask(X, D, B)
    with pytest.raises(ValueError, match="lambda1 must be defined"):
        spams_b200.lassoMask(X, D, B)
    with pytest.raises(ValueError, match="incompatible matrix dimensions"):
        spams_b200.lassoMask(X, np.asfortranarray(np.random.randn(9, 6)), B, lambda1=0.1)


def test_refactor_choice_is_validated():
    X = np.asfortranarray(np.random.randn(8, 4).astype(np.float32))
    D = np.asfortranarray(np.random.randn(8, 6).astype(np.float32))
    with pytest.raises(ValueError, match="refactor must be"):
        spams_b200.lasso(X, D, lambda1=0.1, refactor="sometimes")
