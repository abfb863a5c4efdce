"""The two coding-kernel families (one warp per signal, one CTA per signal)
run the same arithmetic in the same order: forcing either gives the same bits,
and so does the autotuned choice."""
import numpy as np
import pytest

import spams_b200
from spams_b200 import _lib
from spams_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = a.tocsc(), b.tocsc()
    assert a.shape == b.shape
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    np.testing.assert_array_equal(a.data, b.data)


def _draw(m, K, n, seed, dt):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = W.gaussian_dictionary(m, K, rng)
    X, _, _ = W.sparse_signals(D, n, 10, 0.05, rng)
    return np.asfortranarray(X, dt), np.asfortranarray(D, dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("m,K", [(64, 200), (96, 512), (128, 1000)])
def test_warp_and_cta_give_the_same_bits(dt, m, K):
    X, D = _draw(m, K, 700, K + m, dt)
    runs = [
        (spams_b200.lasso, dict(lambda1=0.05)),
        (spams_b200.lasso, dict(lambda1=0.005)),           # active sets past 32 atoms
        (spams_b200.lasso, dict(lambda1=2.0, mode=0, pos=True)),
        (spams_b200.lasso, dict(lambda1=0.5, mode=1)),
        (spams_b200.omp, dict(L=12)),
        (spams_b200.omp, dict(L=60, eps=1e-3)),            # OMP past 32 atoms
    ]
    for fn, kw in runs:
        w = fn(X, D, kernel="warp", **kw)
        c = fn(X, D, kernel="cta", **kw)
        a = fn(X, D, **kw)
        _same(w, c)
        _same(w, a)


def test_paths_and_bf16x3_match_across_kernels():
    X, D = _draw(96, 512, 300, 9, np.float32)
    pw = spams_b200.lasso(X, D, lambda1=0.02, return_reg_path=True, kernel="warp")
    pc = spams_b200.lasso(X, D, lambda1=0.02, return_reg_path=True, kernel="cta")
    _same(pw[0], pc[0])
    np.testing.assert_array_equal(pw[1], pc[1])
    bw = spams_b200.omp(X, D, L=20, precision=spams_b200.SC_PREC_BF16X3, kernel="warp")
    bc = spams_b200.omp(X, D, L=20, precision=spams_b200.SC_PREC_BF16X3, kernel="cta")
    _same(bw, bc)


def test_warp_kernel_refuses_large_dictionaries():
    X, D = _draw(64, 1500, 10, 1, np.float32)
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.omp(X, D, L=4, kernel="warp")
    assert e.value.status == _lib.SC_ERR_UNSUPPORTED
    _same(spams_b200.omp(X, D, L=4, kernel="cta"), spams_b200.omp(X, D, L=4))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("m,K", [(64, 200), (128, 1000)])
def test_cholesky_variant_warp_and_cta_give_the_same_bits(dt, m, K):
    """The Cholesky implementation (cholesky / ols) in its two forms: the
    warp kernel and, forced here at a size the warp kernel takes, the CTA
    kernel that codes dictionaries beyond 1024 atoms."""
    X, D = _draw(m, K, 300, K + m + 1, dt)
    runs = [
        dict(lambda1=0.05, cholesky=True),
        dict(lambda1=0.005, cholesky=True),                 # past the 32-atom state
        dict(lambda1=2.0, mode=0, pos=True, cholesky=True),
        dict(lambda1=0.5, mode=1, cholesky=True),
        dict(lambda1=0.05, ols=True),
        dict(lambda1=0.5, mode=1, ols=True),
    ]
    for kw in runs:
        w = spams_b200.lasso(X, D, kernel="warp", **kw)
        c = spams_b200.lasso(X, D, kernel="cta", **kw)
        _same(w, c)
    pw = spams_b200.lasso(X, D, lambda1=0.02, cholesky=True, return_reg_path=True, kernel="warp")
    pc = spams_b200.lasso(X, D, lambda1=0.02, cholesky=True, return_reg_path=True, kernel="cta")
    _same(pw[0], pc[0])
    np.testing.assert_array_equal(pw[1], pc[1])
