"""The minibatch step of online dictionary learning on the GPU: its codes are
the coding path's codes of the selected minibatch, A and B are the rank-1
accumulations of those codes, the minibatch index comes from the device
counter, and a CUDA-graph replay reproduces the eager loop bit for bit."""
import numpy as np
import pytest
import scipy.sparse as ssp

import spams_b200
from spams_b200 import dictlearn as DL
from spams_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _cm(a):
    """Column-major float32 CUDA tensor of a numpy matrix."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda().t()


def _setup(m=144, K=256, M=3000, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = W.smooth_patches(M, rng, side=12)[:m]
    X = X / np.linalg.norm(X, axis=0, keepdims=True)
    D = X[:, rng.choice(M, K, replace=False)]
    D = D + 0.05 * rng.standard_normal(D.shape)
    D = D / np.linalg.norm(D, axis=0, keepdims=True)
    perm = rng.permutation(M).astype(np.int32)
    return np.asfortranarray(X, np.float32), np.asfortranarray(D, np.float32), perm


def _csc(codes, K, n):
    cp, r, v = (t.cpu().numpy() for t in codes)
    return ssp.csc_matrix((v, r, cp), shape=(K, n))


def _same(a, b):
    a, b = a.tocsc(), b.tocsc()
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    np.testing.assert_array_equal(a.data, b.data)


@pytest.mark.parametrize("mode,lam", [(DL.PENALTY, 0.1), (DL.L1COEFFS, 1.0), (DL.L2ERROR, 0.2),
                                      (DL.SPARSITY, 6), (DL.L2ERROR2, 0.1), (DL.PENALTY2, 0.01)])
def test_step_codes_and_accumulations(mode, lam):
    m, K, batch = 144, 256, 200
    X, D, perm = _setup(m, K)
    Xd, Dd, pd = _cm(X), _cm(D), torch.from_numpy(perm).cuda()
    it = torch.zeros(1, dtype=torch.int64, device="cuda")
    A = torch.zeros((K, K), device="cuda").t()
    B = torch.zeros((K, m), device="cuda").t()
    step = spams_b200.MinibatchStep(m, K, batch, mode=mode, lambda1=lam)
    A0 = np.random.default_rng(1).standard_normal((K, K)).astype(np.float32)
    B0 = np.random.default_rng(2).standard_normal((m, K)).astype(np.float32)
    A.copy_(_cm(A0))
    B.copy_(_cm(B0))
    for i in range(3):
        step(Dd, Xd, it, perm=pd, A=A, B=B, beta=0.5, gamma=2.0)
        torch.cuda.synchronize()
        cols = perm[(np.arange(batch) + i * batch) % X.shape[1]]
        Xb = np.asfortranarray(X[:, cols])
        a = _csc(step.codes(), K, batch)
        # the coding path's codes of the same minibatch
        L = min(m, K)
        if mode <= 2:
            ref = spams_b200.lasso(Xb, D, lambda1=lam, mode=mode, L=L)
        elif mode == DL.SPARSITY:
            ref = spams_b200.omp(Xb, D, L=int(lam))
        elif mode == DL.L2ERROR2:
            ref = spams_b200.omp(Xb, D, L=L, eps=lam)
        else:
            ref = spams_b200.omp(Xb, D, L=L, lambda1=lam)
        _same(a, ref)
        # the accumulations of those codes
        ad = a.astype(np.float64).toarray()
        A0 = 0.5 * A0.astype(np.float64) + 2.0 * ad @ ad.T
        B0 = 0.5 * B0.astype(np.float64) + 2.0 * Xb.astype(np.float64) @ ad.T
        np.testing.assert_allclose(A.cpu().numpy(), A0, rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(B.cpu().numpy(), B0, rtol=1e-5, atol=1e-5)
        A0, B0 = A.cpu().numpy(), B.cpu().numpy()
    assert int(it.item()) == 3


def test_graph_replay_matches_eager_loop():
    m, K, batch, steps = 144, 512, 256, 6
    X, D, perm = _setup(m, K, M=4000, seed=3)
    Xd, pd = _cm(X), torch.from_numpy(perm).cuda()

    def run(graph):
        Dd = _cm(D)
        it = torch.zeros(1, dtype=torch.int64, device="cuda")
        A = torch.zeros((K, K), device="cuda").t()
        B = torch.zeros((K, m), device="cuda").t()
        step = spams_b200.MinibatchStep(m, K, batch, lambda1=0.1)
        rng = np.random.default_rng(7)
        U = torch.from_numpy(rng.standard_normal((m, steps)).astype(np.float32)).cuda()
        V = torch.from_numpy(rng.standard_normal((K, steps)).astype(np.float32)).cuda()

        def body():
            # the dictionary changes every minibatch: a rank-1 perturbation
            # (the minibatch's column of U and V, picked by the device
            # counter), then unit columns again
            u = U.index_select(1, it).squeeze(1)
            v = V.index_select(1, it).squeeze(1)
            Dd.add_(0.01 * torch.outer(u, v))
            Dd.div_(Dd.norm(dim=0, keepdim=True))
            step(Dd, Xd, it, perm=pd, A=A, B=B, beta=0.9, gamma=1.0 / batch)

        if not graph:
            for _ in range(steps):
                body()
        else:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                body()  # eager first step: sizes the workspaces
            torch.cuda.current_stream().wait_stream(s)
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg):
                body()
            for _ in range(steps - 1):
                cg.replay()
        torch.cuda.synchronize()
        return Dd.cpu().numpy(), A.cpu().numpy(), B.cpu().numpy(), int(it.item()), \
            _csc(step.codes(), K, batch)

    e = run(False)
    g = run(True)
    assert e[3] == g[3] == steps
    for x, y in zip(e[:3], g[:3]):
        np.testing.assert_array_equal(x, y)
    _same(e[4], g[4])


def test_bf16x3_step_matches_fp32_support():
    m, K, batch = 144, 1024, 512
    X, D, perm = _setup(m, K, M=2000, seed=5)
    Xd, Dd, pd = _cm(X), _cm(D), torch.from_numpy(perm).cuda()
    res = []
    for prec in (None, spams_b200.SC_PREC_BF16X3):
        it = torch.zeros(1, dtype=torch.int64, device="cuda")
        step = spams_b200.MinibatchStep(m, K, batch, lambda1=0.1, precision=prec)
        step(Dd, Xd, it, perm=pd)
        torch.cuda.synchronize()
        res.append(_csc(step.codes(), K, batch))
    a, b = res[0].tocsc(), res[1].tocsc()
    same = sum(np.array_equal(a.indices[a.indptr[j]:a.indptr[j + 1]],
                              b.indices[b.indptr[j]:b.indptr[j + 1]]) for j in range(batch))
    assert same / batch >= 0.99
