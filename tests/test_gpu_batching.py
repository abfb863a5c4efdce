"""The batching form of the uneven-OMP workload: signals with per-signal step
caps L_i are scheduled longest first within each launch, and the whole device
call can be captured once as a CUDA graph and replayed per batch.  Results do
not depend on either: every signal is coded on its own."""
import numpy as np
import pytest

import spams_b200
from spams_b200 import workloads as W
from oracle import oracle as O

from conftest import matched_columns, rel_err, support_match

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _csc(colptr, rows, vals, K, n):
    import scipy.sparse as ssp
    cp = colptr.cpu().numpy()
    return ssp.csc_matrix((vals[:cp[-1]].cpu().numpy(), rows[:cp[-1]].cpu().numpy(), cp),
                          shape=(K, n))


@pytest.mark.parametrize("prec", [spams_b200.SC_PREC_FP32, spams_b200.SC_PREC_BF16X3],
                         ids=["fp32", "bf16x3"])
def test_graph_replay_of_uneven_omp_matches_eager_call(prec):
    dev = torch.device("cuda", 0)
    n, m, K = 20000, 128, 512
    X, D, Lv, eps = W.config_uneven_omp_device(n=n, seed=3, m=m, K=K, smax=32, device=dev)
    Lmax = int(Lv.max().item())
    cap = n * Lmax
    outs = (torch.empty(n + 1, dtype=torch.int64, device=dev),
            torch.empty(cap, dtype=torch.int32, device=dev),
            torch.empty(cap, dtype=torch.float32, device=dev))

    def call(s, sync):
        return spams_b200.omp_device(X, D, L=Lmax, L_vec=Lv, eps_vec=eps, stream=s,
                                     precision=prec, out=outs, sync=sync)

    call(torch.cuda.current_stream(dev), True)
    eager = _csc(*outs, K, n)
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        call(side, False)
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        call(torch.cuda.current_stream(dev), False)
    for _ in range(2):
        for t in outs:
            t.fill_(0)
        graph.replay()
        torch.cuda.synchronize()
        got = _csc(*outs, K, n)
        assert got.nnz == eager.nnz
        np.testing.assert_array_equal(got.indptr, eager.indptr)
        np.testing.assert_array_equal(got.indices, eager.indices)
        np.testing.assert_array_equal(got.data, eager.data)
    # and the codes are the reference's (longest-first order changes nothing)
    if prec == spams_b200.SC_PREC_FP32:
        ns = 3000
        ref = O.orc_omp(X[:, :ns].double().cpu().numpy(), D.double().cpu().numpy(),
                        L=Lv[:ns].cpu().numpy(), eps=eps[:ns].double().cpu().numpy())
        a = eager[:, :ns]
        assert support_match(a, ref) >= 0.995
        assert rel_err(*matched_columns(a, ref)) <= 1e-4


def test_workspace_growth_between_calls_keeps_the_codes():
    """Workspaces grow through the stream-ordered allocator on the call's
    stream: a small call, a much larger one (every workspace grows), then the
    small one again, on host arrays and on a caller's torch stream, give the
    codes that each gives in isolation."""
    rng = np.random.Generator(np.random.PCG64(41))
    m, K = 96, 700
    D = W.gaussian_dictionary(m, K, rng).astype(np.float32)
    Xs, _, _ = W.sparse_signals(D, 300, 8, 0.01, rng)
    Xb, _, _ = W.sparse_signals(D, 60000, 8, 0.01, rng)
    Xs, Xb = np.asfortranarray(Xs, np.float32), np.asfortranarray(Xb, np.float32)
    for prec in (spams_b200.SC_PREC_FP32, spams_b200.SC_PREC_BF16X3):
        a1 = spams_b200.lasso(Xs, D, lambda1=0.05, precision=prec)
        b1 = spams_b200.lasso(Xb, D, lambda1=0.05, precision=prec)
        a2 = spams_b200.lasso(Xs, D, lambda1=0.05, precision=prec)
        assert (a1 != a2).nnz == 0
        b2 = spams_b200.lasso(Xb[:, :300], D, lambda1=0.05, precision=prec)
        assert (b1[:, :300] != b2).nnz == 0
        o1 = spams_b200.omp(Xs, D, L=10, precision=prec)
        ob = spams_b200.omp(Xb, D, L=12, precision=prec)
        assert (o1 != spams_b200.omp(Xs, D, L=10, precision=prec)).nnz == 0
        assert (ob[:, -300:] != spams_b200.omp(Xb[:, -300:], D, L=12, precision=prec)).nnz == 0
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream()
    def cm(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).to(dev).t()
    Dd = cm(D)
    with torch.cuda.stream(st):
        small = spams_b200.lasso_device(cm(Xs), Dd, 0.05)
        big = spams_b200.lasso_device(cm(Xb), Dd, 0.05)
        again = spams_b200.lasso_device(cm(Xs), Dd, 0.05)
    st.synchronize()
    s1 = _csc(*small[:3], K, 300)
    s2 = _csc(*again[:3], K, 300)
    assert (s1 != s2).nnz == 0
    assert (s1 != spams_b200.lasso(Xs, D, lambda1=0.05)).nnz == 0
    assert _csc(*big[:3], K, 60000).nnz > 0


def test_release_all_returns_device_memory_and_recovers():
    """sc_release_all frees every cached workspace and returns the
    stream-ordered pool's blocks to the device; the next call rebuilds them
    and gives the same codes."""
    from spams_b200 import _lib
    rng = np.random.Generator(np.random.PCG64(43))
    D = W.gaussian_dictionary(128, 1024, rng).astype(np.float32)
    X, _, _ = W.sparse_signals(D, 50000, 8, 0.01, rng)
    X = np.asfortranarray(X, np.float32)
    a = spams_b200.lasso(X, D, lambda1=0.05, precision=spams_b200.SC_PREC_BF16X3)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    _lib.lib().sc_release_all()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after > free_before  # workspaces of ~0.5 GB came back
    b = spams_b200.lasso(X, D, lambda1=0.05, precision=spams_b200.SC_PREC_BF16X3)
    assert (a != b).nnz == 0
