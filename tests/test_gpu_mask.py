"""Masked variants on the GPU (ompMask / lassoMask): each signal coded from
its observed rows only.  FP64 results match the oracle's restatement of
omp_mask / lasso_mask (itself pinned to the reference by the golden
fixtures) with identical supports; all-observed masks reproduce the plain
calls bit for bit; unobserved signals give empty columns."""
import numpy as np
import pytest

from conftest import rel_err, support_match

import spams_b200
from spams_b200 import _lib
from spams_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = a.tocsc(), b.tocsc()
    assert a.shape == b.shape
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    np.testing.assert_array_equal(a.data, b.data)


def _draw(m, K, n, seed, density=0.7):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = W.gaussian_dictionary(m, K, rng)
    X, _, _ = W.sparse_signals(D, n, 8, 0.05, rng)
    B = rng.random((m, n)) < density
    B[:, 0] = True
    B[:, 1] = False
    return X, D, B


def _nz(a):
    a = a.tocsc().copy()
    a.eliminate_zeros()
    return a


@pytest.mark.parametrize("m,K", [(64, 300), (48, 1000)])
def test_masked_omp_and_lasso_f64(m, K):
    X, D, B = _draw(m, K, 400, K + m)
    L = np.random.default_rng(1).integers(2, 12, size=X.shape[1]).astype(np.int32)
    eps = np.full(X.shape[1], 0.01)
    for kw in (dict(L=10), dict(L=L, eps=eps), dict(L=15, lambda1=0.01)):
        ref = O.orc_omp_mask(X, D, B, **kw)
        a = spams_b200.ompMask(X, D, B, **kw)
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    for kw in (dict(lambda1=0.05), dict(lambda1=0.3, mode=1, pos=True), dict(lambda1=1.5, mode=0),
               dict(lambda1=0.02, lambda2=0.1), dict(lambda1=0.004)):
        ref = _nz(O.orc_lasso_mask(X, D, B, **kw))
        a = _nz(spams_b200.lassoMask(X, D, B, **kw))
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    assert np.diff(a.indptr)[1] == 0  # the unobserved signal


def test_masked_f32_and_bf16x3_close_to_f64():
    X, D, B = _draw(96, 512, 2000, 5)
    ref = O.orc_omp_mask(X, D, B, L=10)
    a = spams_b200.ompMask(X.astype(np.float32), D.astype(np.float32), B, L=10)
    assert support_match(a, ref) >= 0.99
    b = spams_b200.ompMask(X.astype(np.float32), D.astype(np.float32), B, L=10,
                           precision=spams_b200.SC_PREC_BF16X3)
    assert support_match(b, ref) >= 0.99
    ref = _nz(O.orc_lasso_mask(X, D, B, lambda1=0.05))
    a = _nz(spams_b200.lassoMask(X.astype(np.float32), D.astype(np.float32), B, lambda1=0.05))
    assert support_match(a, ref) >= 0.99


def test_full_masks_reproduce_the_plain_calls():
    X, D, _ = _draw(64, 256, 300, 7)
    full = np.ones(X.shape, bool)
    for dt in (np.float64, np.float32):
        Xd, Dd = X.astype(dt), D.astype(dt)
        _same(spams_b200.ompMask(Xd, Dd, full, L=9), spams_b200.omp(Xd, Dd, L=9))
        _same(spams_b200.lassoMask(Xd, Dd, full, lambda1=0.05),
              spams_b200.lasso(Xd, Dd, lambda1=0.05, L=min(Xd.shape[0], Dd.shape[1])))
    none = np.zeros(X.shape, bool)
    assert spams_b200.ompMask(X, D, none, L=9).nnz == 0
    assert spams_b200.lassoMask(X, D, none, lambda1=0.05).nnz == 0


def test_masked_path_of_the_first_signal():
    X, D, B = _draw(40, 120, 30, 11)
    B[:, 0] = B[:, 2]  # a partially observed first signal
    ref, rpath = O.orc_omp_mask(X, D, B, L=8, return_reg_path=True)
    a, path = spams_b200.ompMask(X, D, B, L=8, return_reg_path=True)
    assert support_match(a, ref) == 1.0
    np.testing.assert_allclose(path, rpath, rtol=1e-8, atol=1e-10)


@pytest.mark.parametrize("m,K", [(32, 1500), (40, 2048), (24, 5000)])
def test_masked_on_the_cta_kernels_f64(m, K):
    """Beyond 1024 atoms the masked products run on the CTA-per-signal
    kernels (Kp / 512 warps per signal): the same exact supports and FP64
    values against the oracle."""
    X, D, B = _draw(m, K, 60, K + 3)
    for kw in (dict(L=6), dict(L=12, lambda1=0.01)):
        ref = O.orc_omp_mask(X, D, B, **kw)
        a = spams_b200.ompMask(X, D, B, **kw)
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    for kw in (dict(lambda1=0.05), dict(lambda1=0.3, mode=1, pos=True)):
        ref = _nz(O.orc_lasso_mask(X, D, B, **kw))
        a = _nz(spams_b200.lassoMask(X, D, B, **kw))
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_masked_warp_and_cta_kernels_give_the_same_bits(dt):
    """Masked coding on the warp kernel (the default up to 1024 atoms) and
    on the CTA kernel when asked for."""
    X, D, B = _draw(48, 512, 300, 17)
    Xd, Dd = X.astype(dt), D.astype(dt)
    w = spams_b200.ompMask(Xd, Dd, B, L=10, kernel="warp")
    _same(w, spams_b200.ompMask(Xd, Dd, B, L=10))
    _same(w, spams_b200.ompMask(Xd, Dd, B, L=10, kernel="cta"))
    w = spams_b200.lassoMask(Xd, Dd, B, lambda1=0.05, kernel="warp")
    _same(w, spams_b200.lassoMask(Xd, Dd, B, lambda1=0.05))
    _same(w, spams_b200.lassoMask(Xd, Dd, B, lambda1=0.05, kernel="cta"))


def test_masked_limits():
    X, D, B = _draw(32, 150, 10, 3)
    with pytest.raises(ValueError, match="non acceptable dimensions"):
        spams_b200.lassoMask(X, D, B[:, :5], lambda1=0.1)
