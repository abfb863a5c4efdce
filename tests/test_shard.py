"""Multi-GPU column sharding with two gloo ranks.

On the CPU each rank codes its column block with the oracle standing in for
its GPU; on a GPU box both ranks code with the engine itself on the one GPU.
Either way the blocks travel as flat CSC arrays and the gathered result must
equal the unsharded coding of the whole batch."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse as ssp

from spams_b200.shard import concat_csc, shard_bounds


def test_shard_bounds_cover_and_balance():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            blocks = [shard_bounds(n, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in blocks]
            assert max(sizes) - min(sizes) <= 1


def test_concat_csc_matches_hstack():
    rng = np.random.default_rng(0)
    parts = [ssp.random(20, k, density=0.2, format="csc", random_state=i) for i, k in enumerate((3, 0, 5, 1))]
    got = concat_csc(parts, 20)
    ref = ssp.hstack(parts).tocsc()
    assert (got != ref).nnz == 0
    assert got.shape == (20, 9)
    del rng


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from spams_b200 import workloads as W
        from spams_b200.shard import code_sharded
        X, D = W.config_lasso(n=301, seed=9, m=32, K=64, s=4, noise=0.01)
        a = code_sharded(O.orc_lasso, X, D, lambda1=0.1)
        Xo, Do, Lv, ev = W.config_uneven_omp(n=157, seed=10, m=24, K=48, smax=6)
        b = code_sharded(O.orc_omp, Xo, Do, L=Lv, eps=ev, dst=None)
        if rank == 0:
            q.put(("ok", a, b))
        else:
            q.put(("ok", a, b))
    except Exception as e:  # report to the parent instead of hanging it
        q.put(("err", repr(e), None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_code_like_one():
    import multiprocessing as mp
    from oracle import oracle as O
    from spams_b200 import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(r[0] == "ok" for r in res), res
    X, D = W.config_lasso(n=301, seed=9, m=32, K=64, s=4, noise=0.01)
    ref = O.orc_lasso(X, D, lambda1=0.1)
    Xo, Do, Lv, ev = W.config_uneven_omp(n=157, seed=10, m=24, K=48, smax=6)
    refo = O.orc_omp(Xo, Do, L=Lv, eps=ev)
    gathered = [r[1] for r in res if r[1] is not None]
    assert len(gathered) == 1  # only the destination rank holds the lasso result
    assert abs(gathered[0] - ref).max() == 0
    for r in res:  # all ranks hold the all-gathered OMP result
        assert abs(r[2] - refo).max() == 0


def _gpu_worker(rank, world, port, q):
    """Two ranks on one GPU coding their blocks with the engine itself (the
    ranks never wait on each other inside a kernel)."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import spams_b200
        from spams_b200 import workloads as W
        from spams_b200.shard import code_sharded
        X, D = W.config_lasso(n=3001, seed=9, m=64, K=256, s=6, noise=0.01)
        a = code_sharded(spams_b200.lasso, X.astype(np.float32), D.astype(np.float32),
                         lambda1=0.1)
        Xo, Do, Lv, ev = W.config_uneven_omp(n=1577, seed=10, m=48, K=128, smax=12)
        b = code_sharded(spams_b200.omp, Xo, Do, L=Lv, eps=ev, dst=None)
        q.put(("ok", a, b))
    except Exception as e:
        q.put(("err", repr(e), None))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_gloo_ranks_with_the_engine_code_like_one():
    import multiprocessing as mp
    import spams_b200
    from spams_b200 import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(r[0] == "ok" for r in res), res
    X, D = W.config_lasso(n=3001, seed=9, m=64, K=256, s=6, noise=0.01)
    ref = spams_b200.lasso(X.astype(np.float32), D.astype(np.float32), lambda1=0.1)
    Xo, Do, Lv, ev = W.config_uneven_omp(n=1577, seed=10, m=48, K=128, smax=12)
    refo = spams_b200.omp(Xo, Do, L=Lv, eps=ev)
    gathered = [r[1] for r in res if r[1] is not None]
    assert len(gathered) == 1
    assert abs(gathered[0] - ref).max() == 0 and gathered[0].nnz == ref.nnz
    for r in res:
        assert abs(r[2] - refo).max() == 0 and r[2].nnz == refo.nnz
