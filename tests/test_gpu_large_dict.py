"""Dictionaries of 1025 to 16384 atoms: the CTA-per-signal kernels.

Beyond 1024 atoms the correlations of one signal no longer fit one warp's
registers, so one CTA of Kp / 512 warps codes a signal (Kp = K rounded up to
512 up to 4096 atoms, then to 6144, 8192, 12288 or 16384).  The same seeded-oracle parity as the warp kernels: exact support and
1e-9 relative error in FP64, every constraint mode, pos, the path of signal
0, per-signal L / eps, the rerun of active sets beyond the shared-memory
capacity, and the (Q, q) form."""
import numpy as np
import pytest

from conftest import rel_err, support_match

import spams_b200
from spams_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _draw(m, K, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = W.gaussian_dictionary(m, K, rng)
    X = np.asfortranarray(rng.standard_normal((m, n)))
    return X, D


@pytest.mark.parametrize("K", [1025, 1100, 1536, 2048, 2500, 4096])
def test_lasso_and_omp_exact_support_f64(K):
    X, D = _draw(64, K, 60, K)
    ref = O.orc_lasso(X, D, lambda1=0.1)
    a = spams_b200.lasso(X, D, lambda1=0.1)
    assert a.shape == ref.shape
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    ref = O.orc_omp(X, D, L=8)
    a = spams_b200.omp(X, D, L=8)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9


@pytest.mark.parametrize("K", [4097, 7000, 10000, 16384])
def test_beyond_4096_atoms_exact_support_f64(K):
    """12, 16, 24 and 32 warps per signal (Kp 6144 .. 16384), double and
    single precision."""
    X, D = _draw(48, K, 24, K)
    ref = O.orc_lasso(X, D, lambda1=0.1)
    a = spams_b200.lasso(X, D, lambda1=0.1)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    ref = O.orc_omp(X, D, L=8)
    if K <= 12288:
        a = spams_b200.omp(X, D, L=8)
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    else:  # two K-vectors of doubles per signal no longer fit a block's shared memory
        with pytest.raises(spams_b200.ScError, match="at most 12288"):
            spams_b200.omp(X, D, L=8)
    a32 = spams_b200.omp(X.astype(np.float32), D.astype(np.float32), L=8)
    assert support_match(a32, ref) >= 0.95


@pytest.mark.parametrize("K", [1536, 4097])
@pytest.mark.parametrize("variant", ["cholesky", "ols"])
def test_cholesky_variant_beyond_1024_atoms_f64(K, variant):
    """The Cholesky implementation (coreLARS + downDateLasso) on the CTA
    kernel: every constraint mode, pos, and the active sets past the
    shared-memory capacity (about 61 atoms at lambda 0.1 here)."""
    X, D = _draw(64, K, 40, K + 5)
    for mode, lam in [(2, 0.1), (0, 1.5), (1, 20.0)]:
        for pos in (False, True):
            ref = O.orc_lasso(X, D, lambda1=lam, mode=mode, pos=pos, **{variant: True})
            a = spams_b200.lasso(X, D, lambda1=lam, mode=mode, pos=pos, **{variant: True})
            assert a.shape == ref.shape
            assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9, (mode, pos)


def test_cholesky_variant_large_active_sets_and_path():
    """120-atom active sets (the rerun with the state in global memory), the
    path of signal 0, and the largest dictionary."""
    X, D = _draw(160, 2048, 8, 77)
    for variant in ("cholesky", "ols"):
        ref, rpath = O.orc_lasso(X, D, L=120, lambda1=0.01, return_reg_path=True,
                                 **{variant: True})
        a, path = spams_b200.lasso(X, D, L=120, lambda1=0.01, return_reg_path=True,
                                   **{variant: True})
        assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
        np.testing.assert_allclose(path, rpath, rtol=1e-8, atol=1e-10)
    X, D = _draw(48, 16384, 8, 16384)
    ref = O.orc_lasso(X, D, lambda1=0.1, cholesky=True)
    a = spams_b200.lasso(X, D, lambda1=0.1, cholesky=True)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    a32 = spams_b200.lasso(X.astype(np.float32), D.astype(np.float32), lambda1=0.1,
                           cholesky=True)
    assert support_match(a32, ref) >= 0.95


def test_more_than_16384_atoms_refused():
    X, D = _draw(16, 16385, 2, 3)
    with pytest.raises(spams_b200.ScError, match="16384"):
        spams_b200.omp(X.astype(np.float32), D.astype(np.float32), L=4)


@pytest.mark.parametrize("mode,lam", [(0, 1.5), (1, 20.0), (2, 0.05)])
def test_lasso_modes_and_pos(mode, lam):
    X, D = _draw(48, 2048, 40, 7 + mode)
    for pos in (False, True):
        ref = O.orc_lasso(X, D, lambda1=lam, mode=mode, pos=pos)
        a = spams_b200.lasso(X, D, lambda1=lam, mode=mode, pos=pos)
        assert support_match(a, ref) == 1.0
        assert rel_err(a, ref) <= 1e-9


def test_regularisation_paths():
    X, D = _draw(64, 1536, 10, 21)
    ref, rpath = O.orc_lasso(X, D, lambda1=0.05, return_reg_path=True)
    a, path = spams_b200.lasso(X, D, lambda1=0.05, return_reg_path=True)
    assert support_match(a, ref) == 1.0
    np.testing.assert_allclose(path, rpath, rtol=1e-8, atol=1e-10)
    ref, rpath = O.orc_omp(X, D, L=12, return_reg_path=True)
    a, path = spams_b200.omp(X, D, L=12, return_reg_path=True)
    assert support_match(a, ref) == 1.0
    np.testing.assert_allclose(path, rpath, rtol=1e-8, atol=1e-10)


def test_overflow_rerun_cta():
    """Active sets beyond the CTA's shared-memory capacity (80 atoms) take the
    rerun with per-CTA global state."""
    X, D = _draw(128, 2048, 40, 31)
    ref = O.orc_omp(X, D, L=100)
    assert (np.diff(ref.indptr) > 80).any()
    a = spams_b200.omp(X, D, L=100)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-8
    ref = O.orc_lasso(X, D, lambda1=0.002)
    assert (np.diff(ref.indptr) > 80).any()
    a = spams_b200.lasso(X, D, lambda1=0.002)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-8


def test_uneven_omp_f64_and_f32():
    """The batched uneven OMP workload's shape (D 512 x 2048, L_i = s_i + 4,
    eps_i = 0.5 ||noise_i||^2) on a sample of signals."""
    X, D, L, eps = W.config_uneven_omp(n=600, seed=5)
    ref = O.orc_omp(X, D, L=L, eps=eps)
    a = spams_b200.omp(X, D, L=L, eps=eps)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-9
    X32, D32 = X.astype(np.float32), D.astype(np.float32)
    # single precision: a column whose residual ends within rounding of its
    # eps may stop one atom earlier or later (at most 3 of the 600 here)
    a32 = spams_b200.omp(X32, D32, L=L, eps=eps.astype(np.float32))
    assert support_match(a32, ref) >= 0.995
    b32 = spams_b200.omp(X32, D32, L=L, eps=eps.astype(np.float32),
                         precision=spams_b200.SC_PREC_BF16X3, refine=1)
    assert support_match(b32, ref) >= 0.995


def test_gram_form_matches_dictionary_form():
    X, D = _draw(64, 1536, 30, 41)
    Q = np.asfortranarray(D.T @ D)
    q = np.asfortranarray(D.T @ X)
    ref = O.orc_lasso(X, D, lambda1=0.1, lambda2=0.0)
    a = spams_b200.lasso(X, Q=Q, q=q, lambda1=0.1)
    assert support_match(a, ref) == 1.0 and rel_err(a, ref) <= 1e-8


def test_device_entry_matches_host_entry():
    torch = pytest.importorskip("torch")
    X, D = _draw(96, 3000, 200, 51)
    X32, D32 = X.astype(np.float32), D.astype(np.float32)
    host = spams_b200.lasso(X32, D32, lambda1=0.1)
    dev = torch.device("cuda:0")
    Xt = torch.from_numpy(np.ascontiguousarray(X32.T)).to(dev).t()
    Dt = torch.from_numpy(np.ascontiguousarray(D32.T)).to(dev).t()
    colptr, rows, vals, nnz = spams_b200.lasso_device(Xt, Dt, 0.1)
    assert nnz == host.nnz
    np.testing.assert_array_equal(colptr.cpu().numpy(), host.indptr)
    np.testing.assert_array_equal(rows[:nnz].cpu().numpy(), host.indices)
    np.testing.assert_array_equal(vals[:nnz].cpu().numpy(), host.data)
