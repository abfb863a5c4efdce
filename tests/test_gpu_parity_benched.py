"""Parity of the configurations the benchmark runs, in the form it runs them,
against the FP64 reference (the reference's own omp / lasso2 compiled from
its sources, or the C restatement pinned to it where that build is absent).

Each test reports the support match, the Frobenius relative error over the
columns whose supports agree, and the 99.9th percentile and maximum of the
per-column relative error on those columns.
"""
import numpy as np
import pytest

from conftest import err_report

import spams_b200
from spams_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

BF16 = spams_b200.SC_PREC_BF16X3
FP32 = spams_b200.SC_PREC_FP32


def _ref_lasso(X, D, **kw):
    if O.have_ref():
        return O.ref_lasso(np.asfortranarray(X, np.float64), np.asfortranarray(D, np.float64),
                           numThreads=-1, **kw)
    return O.orc_lasso(np.asfortranarray(X, np.float64), np.asfortranarray(D, np.float64), **kw)


def _ref_omp(X, D, **kw):
    if O.have_ref():
        return O.ref_omp(np.asfortranarray(X, np.float64), np.asfortranarray(D, np.float64),
                         numThreads=-1, **kw)
    return O.orc_omp(np.asfortranarray(X, np.float64), np.asfortranarray(D, np.float64), **kw)


def _report(tag, rep):
    sm, fro, p999, mx = rep
    print(f"\n{tag}: support {sm:.5f}, rel err {fro:.2e}, per-column p99.9 {p999:.2e}, "
          f"max {mx:.2e}")


@pytest.mark.parametrize("prec", [BF16, FP32], ids=["bf16x3", "fp32"])
def test_lasso_workload_full_size_vs_reference_f64(prec):
    """D 256 x 512, all 100 000 signals, lambda1 = 0.15, as the benchmark codes
    them (BF16 hi/lo correlations, or plain FP32), against the FP64 reference."""
    X, D = W.config_lasso(100000)
    ref = _ref_lasso(X, D, lambda1=0.15)
    a = spams_b200.lasso(X.astype(np.float32), D.astype(np.float32), lambda1=0.15,
                         precision=prec, kernel="warp")
    rep = err_report(a, ref)
    _report(f"lasso 256x512 n=1e5 prec={prec}", rep)
    sm, fro, p999, _ = rep
    assert sm >= 0.999
    assert fro <= 1e-5
    assert p999 <= 1e-4


def test_uneven_omp_as_benched_vs_reference_f64():
    """The batched uneven OMP workload exactly as the benchmark draws and codes
    it (device-drawn X 512 x 1e6, D 512 x 2048, s ~ U{1..64}, L = s + 4,
    eps = 0.5 ||noise||^2, BF16 hi/lo correlations, no refinement), its first
    10 000 columns compared with the FP64 reference."""
    dev = torch.device("cuda", 0)
    n = 1000000
    X, D, Lv, eps = W.config_uneven_omp_device(n=n, seed=0, device=dev)
    Lmax = int(Lv.max().item())
    colptr, rows, vals, nnz = spams_b200.omp_device(X, D, L=Lmax, L_vec=Lv, eps_vec=eps,
                                                     precision=BF16)
    ns = 10000
    cp = colptr[:ns + 1].cpu().numpy()
    import scipy.sparse as ssp
    a = ssp.csc_matrix((vals[:cp[-1]].cpu().numpy(), rows[:cp[-1]].cpu().numpy(), cp),
                       shape=(D.shape[1], ns))
    Xs = X[:, :ns].double().cpu().numpy()
    Dh = D.double().cpu().numpy()
    ref = _ref_omp(Xs, Dh, L=Lv[:ns].cpu().numpy(), eps=eps[:ns].double().cpu().numpy())
    rep = err_report(a, ref)
    _report("uneven omp 512x2048 first 1e4 of 1e6, bf16x3", rep)
    sm, fro, p999, _ = rep
    assert sm >= 0.999
    assert fro <= 1e-5
    assert p999 <= 1e-4


def test_dictlearn_step_codes_vs_reference_f64():
    """Codes of the dictionary-learning minibatch step at the benchmarked shape
    (12x12 smooth patches, D 144 x 1024 drawn from the signals as the
    benchmark does, batch 1024, lambda1 = 0.1) against the FP64 reference
    lasso2 on the same minibatch and dictionary."""
    m, K, batch = 144, 1024, 1024
    rng = np.random.Generator(np.random.PCG64(0))
    pool = 20000
    Xnp = W.smooth_patches(pool, rng, side=12).astype(np.float32)
    D0 = Xnp[:, rng.choice(pool, K, replace=False)]
    D0 = np.asfortranarray(D0 / np.linalg.norm(D0, axis=0, keepdims=True), dtype=np.float32)
    perm = rng.permutation(pool).astype(np.int32)

    def cm(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda().t()

    for prec in (BF16, FP32):
        step = spams_b200.MinibatchStep(m, K, batch, lambda1=0.1, precision=prec)
        it = torch.zeros(1, dtype=torch.int64, device="cuda")
        step(cm(D0), cm(Xnp), it, perm=torch.from_numpy(perm).cuda())
        torch.cuda.synchronize()
        cp, r, v = (t.cpu().numpy() for t in step.codes())
        import scipy.sparse as ssp
        a = ssp.csc_matrix((v, r, cp), shape=(K, batch))
        Xb = Xnp[:, perm[:batch]]
        ref = _ref_lasso(Xb, D0, lambda1=0.1, L=min(m, K))
        rep = err_report(a, ref)
        _report(f"dictlearn step 144x1024 batch 1024 prec={prec}", rep)
        sm, fro, p999, _ = rep
        assert sm >= 0.995
        # smooth patches make a correlated dictionary, which amplifies the
        # BF16 hi/lo correlation error (the BF16-split tolerance is 1e-3)
        assert fro <= (1e-5 if prec == FP32 else 1e-4)


def _tie_case(dt):
    """A Gram-entry lasso case in which two inactive atoms (1 and 2, owned by
    the same lane of the coding kernels) offer joining steps whose rounded
    quotients (C - c)/(1 - a) are equal while their cross products order
    them the other way: the reference's cblas_iamin takes the first index.

    G = I with G[0,1] = g1, G[0,2] = g2; D^T x = (1, c1, c2, 0, ...).  Atom 0
    enters first with u = 1, so A_j = g_j exactly and the candidates are
    fl(fl(1 - c_j) / fl(1 - g_j))."""
    rng = np.random.default_rng(0)
    one = dt(1)
    for _ in range(200000):
        c1 = dt(0.45 + 0.1 * rng.random())
        g1 = dt(0.25 + 0.1 * rng.random())
        n1, d1 = one - c1, one - g1
        for _ in range(20):
            c2 = c1 + dt(rng.integers(-8, 9)) * np.spacing(c1)
            g2 = g1 + dt(rng.integers(-8, 9)) * np.spacing(g1)
            n2, d2 = one - c2, one - g2
            if n1 / d1 == n2 / d2 and n2 * d1 < n1 * d2:
                K = 8
                Q = np.eye(K, dtype=dt)
                Q[1, 0] = Q[0, 1] = g1
                Q[2, 0] = Q[0, 2] = g2
                q = np.zeros((K, 1), dt)
                q[0, 0], q[1, 0], q[2, 0] = 1, c1, c2
                X = np.full((K, 1), np.sqrt(10.0 / K), dt)
                return X, Q, q
    raise AssertionError("no tie case found")


@pytest.mark.parametrize("kernel", ["warp", "cta"])
def test_joining_screen_exact_tie_takes_first_index(kernel):
    """Equal rounded joining steps go to the first index, as cblas_iamin
    (linalg/cblas_alt_template.h:1094-1105) in the reference's coreLARS2
    (decomp/decomp.h:1823) decides them."""
    X, Q, q = _tie_case(np.float64)
    ref = O.ref_lasso(X, Q=Q, q=q, lambda1=0.05) if O.have_ref() else None
    orc_first = [0, 1]
    if ref is not None:
        ref.sort_indices()
        assert list(ref.indices) == orc_first
    a = spams_b200.lasso(X, Q=Q, q=q, lambda1=0.05, kernel=kernel)
    a.sort_indices()
    assert list(a.indices) == orc_first
    if ref is not None:
        np.testing.assert_allclose(a.toarray(), ref.toarray(), rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("prec", [FP32, BF16], ids=["fp32", "bf16x3"])
def test_dictlearn_step_accumulations_vs_reference_loop(prec):
    """A <- beta A + gamma sum a a^T and B <- beta B + gamma sum x a^T of one
    minibatch at the benchmarked shape, against the reference's own loop body
    (Trainer::train, dictLearn/dicts.h:526-603: Gram + ridge, multTrans,
    coreLARS2, sort, rank-1 updates; float build) on the same minibatch.

    The accumulation is exact arithmetic on the step's own codes (checked in
    double); the codes match the reference's float codes column by column,
    where one column whose last atom is picked differently moves A by ~5e-3
    (an atom of a smooth-patch dictionary), so A and B against the
    reference's own loop are held to that scale."""
    if not O.have_ref():
        pytest.skip("the reference build is absent")
    import scipy.sparse as ssp
    m, K, batch = 144, 1024, 1024
    rng = np.random.Generator(np.random.PCG64(1))
    pool = 8192
    Xnp = np.asfortranarray(W.smooth_patches(pool, rng, side=12).astype(np.float32))
    D0 = Xnp[:, rng.choice(pool, K, replace=False)]
    D0 = np.asfortranarray(D0 / np.linalg.norm(D0, axis=0, keepdims=True), dtype=np.float32)
    perm = rng.permutation(pool).astype(np.int32)
    A0 = np.asfortranarray(0.01 * rng.standard_normal((K, K)).astype(np.float32))
    B0 = np.asfortranarray(0.01 * rng.standard_normal((m, K)).astype(np.float32))
    beta, gamma, it0 = 0.9, 1.5, 3

    def cm(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda().t()

    step = spams_b200.MinibatchStep(m, K, batch, lambda1=0.1, precision=prec)
    it = torch.full((1,), it0, dtype=torch.int64, device="cuda")
    A, B = cm(A0), cm(B0)
    step(cm(D0), cm(Xnp), it, perm=torch.from_numpy(perm).cuda(), A=A, B=B, beta=beta,
         gamma=gamma)
    torch.cuda.synchronize()
    assert int(it.item()) == it0 + 1
    Ag, Bg = A.cpu().numpy().astype(np.float64), B.cpu().numpy().astype(np.float64)
    cp, r, v = (t.cpu().numpy() for t in step.codes())
    codes = ssp.csc_matrix((v, r, cp), shape=(K, batch)).astype(np.float64)
    Xb = Xnp[:, perm[(np.arange(batch) + it0 * batch) % pool]].astype(np.float64)
    # the accumulation itself, on the step's own codes
    Ae = beta * A0.astype(np.float64) + gamma * (codes @ codes.T).toarray()
    Be = beta * B0.astype(np.float64) + gamma * (codes @ Xb.T).T
    assert np.linalg.norm(Ag - Ae) / np.linalg.norm(Ae) <= 1e-6
    assert np.linalg.norm(Bg - Be) / np.linalg.norm(Be) <= 1e-6
    # the codes against the reference's float coreLARS2 on the same minibatch
    refc = O.ref_lasso(np.asfortranarray(Xb, np.float32), D0, lambda1=0.1, L=min(m, K),
                       numThreads=-1)
    sm, fro, _, _ = err_report(codes, refc)
    # A and B against the reference's own loop
    Ar, Br = A0.copy(order="F"), B0.copy(order="F")
    O.ref_dl_minibatch(D0, Xnp, perm, it0, batch, 0.1, Ar, Br, beta=beta, gamma=gamma)
    ea = np.linalg.norm(Ag - Ar) / np.linalg.norm(Ar)
    eb = np.linalg.norm(Bg - Br) / np.linalg.norm(Br)
    print(f"\ndictlearn step prec={prec}: codes vs reference float support {sm:.4f}, "
          f"rel err {fro:.2e}; A rel err {ea:.2e}, B rel err {eb:.2e}")
    assert sm >= 0.995
    assert fro <= (1e-4 if prec == FP32 else 1e-3)
    assert ea <= 2e-2 and eb <= 2e-2
