"""The serving loop on the GPU: a request's result does not depend on the
requests it shares a launch with (alone vs mixed, bit for bit), equals the
direct float32 API's result, merges pending same-dictionary requests, respects
the device-memory budget, and reports latencies for an open-loop replay."""
import time

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


def _draw(m, K, n, seed, s=6):
    rng = np.random.Generator(np.random.PCG64(seed))
    D = W.gaussian_dictionary(m, K, rng).astype(np.float32)
    X, _, _ = W.sparse_signals(D.astype(np.float64), n, s, 0.01, rng)
    return np.asfortranarray(D), np.asfortranarray(X, dtype=np.float32)


def _requests(X):
    """Mixed OMP / Lasso requests over column windows of X."""
    return [
        ("omp", X[:, 0:300], dict(L=5)),
        ("omp", X[:, 300:700], dict(L=9, eps=0.05)),
        ("omp", X[:, 700:800], dict(lambda1=0.02)),
        ("lasso", X[:, 800:1400], dict(lambda1=0.1)),
        ("lasso", X[:, 1400:1500], dict(lambda1=0.25)),
        ("lasso", X[:, 1500:1700], dict(lambda1=0.3, mode=2, pos=True)),
        ("omp", X[:, 1700:2000], dict(L=12)),
    ]


def _direct(algo, Xs, D, kw):
    Xs = np.asfortranarray(Xs)
    if algo == "omp":
        return spams_b200.omp(Xs, D, **kw)
    return spams_b200.lasso(Xs, D, **kw)


@pytest.mark.parametrize("m,K,prec", [(64, 256, None), (144, 1024, spams_b200.SC_PREC_BF16X3),
                                      (96, 2048, None)])
def test_alone_vs_mixed_vs_direct(m, K, prec):
    D, X = _draw(m, K, 2000, K + m)
    big = np.asfortranarray(np.tile(X, (1, 40)))  # keeps the only slot busy
    reqs = _requests(X)
    with spams_b200.Server(hbm_budget=20e9, slots=1) as srv:
        srv.add_dictionary(1, D)
        alone = [srv.code(1, np.asfortranarray(x), algo, precision=prec, **kw)
                 for algo, x, kw in reqs]
        srv.stats(reset=True)
        # a long request first: the others queue behind it and are merged
        t_big = srv.submit(1, big, "omp", L=4, precision=prec)
        tickets = [srv.submit(1, np.asfortranarray(x), algo, precision=prec, **kw)
                   for algo, x, kw in reqs]
        mixed = [srv.result(t) for t in tickets]
        srv.result(t_big)
        st = srv.stats()
    assert st["completed"] == len(reqs) + 1
    assert st["batches"] < len(reqs) + 1, st  # some requests shared a launch
    for (algo, x, kw), a, b in zip(reqs, alone, mixed):
        _same(a, b)
        _same(a, _direct(algo, x, D, dict(kw, precision=prec)))


def test_results_follow_the_request_options():
    D, X = _draw(64, 256, 400, 3)
    with spams_b200.Server(hbm_budget=4e9, slots=2) as srv:
        srv.add_dictionary(5, D)
        a = srv.code(5, X, "lasso", lambda1=0.2, mode=spams_b200.SC_L1COEFFS)
        _same(a, spams_b200.lasso(X, D, lambda1=0.2, mode=spams_b200.SC_L1COEFFS))
        a = srv.code(5, X, "lasso", lambda1=0.15, L=3)
        assert np.diff(a.indptr).max() <= 3
        _same(a, spams_b200.lasso(X, D, lambda1=0.15, L=3))
        a = srv.code(5, X, "omp", eps=0.1)
        _same(a, spams_b200.omp(X, D, eps=0.1))
        # empty request: a K x 0 result
        a = srv.code(5, np.zeros((64, 0), np.float32), "omp", L=3)
        assert a.shape == (256, 0) and a.nnz == 0
        with pytest.raises(ValueError, match="incompatible matrix dimensions"):
            srv.submit(5, np.zeros((65, 3), np.float32), "omp", L=3)
        with pytest.raises(spams_b200.ScError, match="unknown dictionary"):
            srv.submit(9, X, "omp", L=3)


def test_device_memory_budget():
    D, X = _draw(64, 256, 1000, 4)
    with spams_b200.Server(hbm_budget=64 << 20, slots=2) as srv:
        srv.add_dictionary(1, D)
        a = srv.code(1, X, "omp", L=4)
        _same(a, spams_b200.omp(X, D, L=4))
        huge = np.asfortranarray(np.tile(X, (1, 200)))  # 200k signals: ~0.4 GB of workspaces
        with pytest.raises(spams_b200.ScError) as e:
            srv.code(1, huge, "omp", L=4)
        assert e.value.status == _lib.SC_ERR_OUT_OF_MEMORY
        # the server still serves requests that fit
        _same(srv.code(1, X, "omp", L=4), a)
        assert srv.stats()["peak_device_bytes"] <= 64 << 20
        with pytest.raises(spams_b200.ScError, match="does not fit"):
            srv.add_dictionary(2, np.asfortranarray(np.ones((512, 4096), np.float32)))


def test_concurrent_slots_with_every_kernel_shape():
    """Slots launch the same kernels with different shared-memory sizes at
    the same time (OMP requests of different L, Lasso with large active sets,
    large and small dictionaries): every request succeeds and equals the
    direct call."""
    cases = [(64, 256), (96, 1024), (128, 2048)]
    dicts, data = [], []
    for i, (m, K) in enumerate(cases):
        D, X = _draw(m, K, 600, 100 + i, s=20)
        dicts.append(D)
        data.append(X)
    with spams_b200.Server(hbm_budget=20e9, slots=4) as srv:
        for i, D in enumerate(dicts):
            srv.add_dictionary(i, D)
        jobs = []
        for rep in range(6):
            for i, X in enumerate(data):
                L = 4 + 9 * rep
                jobs.append((i, X, "omp", dict(L=L)))
                jobs.append((i, X, "lasso", dict(lambda1=0.3 / (rep + 1))))
        tickets = [srv.submit(i, X, algo, **kw) for i, X, algo, kw in jobs]
        outs = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["rejected"] == 0, st["last_error"]
    for (i, X, algo, kw), a in zip(jobs, outs):
        _same(a, _direct(algo, X, dicts[i], kw))


def test_remove_dictionary_and_timeouts():
    D, X = _draw(64, 256, 100, 5)
    srv = spams_b200.Server(hbm_budget=2e9, slots=1)
    try:
        srv.add_dictionary(1, D)
        with pytest.raises(spams_b200.ScError, match="exists"):
            srv.add_dictionary(1, D)
        t = srv.submit(1, X, "omp", L=3)
        srv.result(t)
        srv.remove_dictionary(1)
        with pytest.raises(spams_b200.ScError, match="unknown dictionary"):
            srv.submit(1, X, "omp", L=3)
        with pytest.raises(spams_b200.ScError, match="unknown ticket"):
            srv.result(t)
    finally:
        srv.close()


def test_replay_reports_latencies():
    dicts, pools, reqs = W.config_serving(rate=400.0, duration_s=0.5, seed=1, pool=4000,
                                          nmax=4000)
    with spams_b200.Server(hbm_budget=40e9, slots=3) as srv:
        for i, D in enumerate(dicts):
            srv.add_dictionary(i, D)
        recs = []
        for k in range(len(reqs["n"])):
            P = pools[reqs["dict"][k]]
            o, n = int(reqs["offset"][k]), int(reqs["n"][k])
            if reqs["algo"][k] == 0:
                recs.append(spams_b200.request(int(reqs["dict"][k]), P[:, o:o + n], "omp",
                                               L=int(reqs["L"][k]), discard=True))
            else:
                recs.append(spams_b200.request(int(reqs["dict"][k]), P[:, o:o + n], "lasso",
                                               lambda1=float(reqs["lambda1"][k]), discard=True))
        t0 = time.perf_counter()
        srv.replay(recs, reqs["arrival_s"])
        wall = time.perf_counter() - t0
        st = srv.stats()
    assert st["rejected"] == 0, st["last_error"]
    assert st["completed"] == len(recs) and st["pending"] == 0
    assert st["signals"] == int(np.sum(reqs["n"]))
    assert 0 < st["lat_p50_ms"] <= st["lat_p99_ms"] <= st["lat_max_ms"]
    assert wall >= float(reqs["arrival_s"][-1])
