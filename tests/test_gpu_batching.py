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
