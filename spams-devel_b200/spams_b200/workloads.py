"""Seeded synthetic workloads with the shapes of the engine's benchmark set.

SPAMS publishes no dataset for its coding path; its demos draw random
Gaussian signals (cpp_library/test_decomp.cpp:14-64, swig/python/test_decomp.py)
and its dictionary-learning demos use 8x8 / 12x12 image patches.  These
generators stand in for them: NumPy PCG64, seed 0 unless stated, column-major
float64 (cast as needed) so the CPU oracle and the GPU read the same numbers.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as ssp


def unit_columns(A: np.ndarray) -> np.ndarray:
    return A / np.linalg.norm(A, axis=0, keepdims=True)


def gaussian_dictionary(m: int, K: int, rng: np.random.Generator) -> np.ndarray:
    return np.asfortranarray(unit_columns(rng.standard_normal((m, K))))


def sparse_signals(D: np.ndarray, n: int, s, noise: float, rng: np.random.Generator,
                   chunk: int = 1 << 16):
    """X = D a + noise * N(0,1), a with s (scalar or per-column array) uniformly
    placed N(0,1) non-zeros.  Returns (X, A, noise_sq) with A K x n csc and
    noise_sq[i] = ||noise_i||^2."""
    m, K = D.shape
    s_arr = np.full(n, s, np.int64) if np.isscalar(s) else np.asarray(s, np.int64)
    X = np.empty((m, n), order="F")
    noise_sq = np.empty(n)
    rows_all, vals_all = [], []
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        cs = s_arr[c0:c1]
        # uniform supports without replacement: argsort of random keys
        keys = rng.random((c1 - c0, K))
        smax = int(cs.max()) if cs.size else 0
        idx = np.argpartition(keys, smax - 1, axis=1)[:, :smax] if smax > 0 else np.zeros((c1 - c0, 0), int)
        mask = np.arange(smax)[None, :] < cs[:, None]
        vals = rng.standard_normal((c1 - c0, smax))
        rows = idx[mask]
        v = vals[mask]
        cols = np.repeat(np.arange(c1 - c0), cs)
        A = ssp.csc_matrix((v, (rows, cols)), shape=(K, c1 - c0))
        E = noise * rng.standard_normal((m, c1 - c0))
        X[:, c0:c1] = (A.T @ D.T).T + E
        noise_sq[c0:c1] = (E * E).sum(axis=0)
        rows_all.append(A)
    A = ssp.hstack(rows_all).tocsc() if rows_all else ssp.csc_matrix((K, 0))
    return X, A, noise_sq


def config_omp_small(n: int = 10000, seed: int = 0):
    """Plain OMP: D 64x256 and X 64 x n, N(0,1) entries, unit-norm columns;
    L=10, eps=0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D = gaussian_dictionary(64, 256, rng)
    X = np.asfortranarray(unit_columns(rng.standard_normal((64, n))))
    return X, D


def config_lasso(n: int = 100000, seed: int = 0, m: int = 256, K: int = 512, s: int = 12,
                 noise: float = 0.01):
    """LARS-Lasso mode 2, lambda1=0.15: D 256x512 unit-norm N(0,1); each column
    of X is D a + 0.01 N(0,1) with 12 uniformly placed N(0,1) non-zeros."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D = gaussian_dictionary(m, K, rng)
    X, _, _ = sparse_signals(D, n, s, noise, rng)
    return X, D


def config_uneven_omp(n: int = 1000000, seed: int = 0, m: int = 512, K: int = 2048,
                      smax: int = 64, noise: float = 0.02):
    """Batched uneven OMP: D 512x2048; s_i ~ U{1..64}; x = D a + 0.02 N(0,1);
    per-column L_i = s_i + 4 and eps_i = 0.5 ||noise_i||^2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D = gaussian_dictionary(m, K, rng)
    s = rng.integers(1, smax + 1, size=n)
    X, _, nsq = sparse_signals(D, n, s, noise, rng)
    L = (s + 4).astype(np.int32)
    eps = 0.5 * nsq
    return X, D, L, eps


def smooth_patches(n: int, rng: np.random.Generator, side: int = 12) -> np.ndarray:
    """side x side patches of N(0,1) convolved with a 3x3 Gaussian, mean
    removed, unit norm (stand-in for image patches)."""
    k1 = np.array([1.0, 2.0, 1.0]) / 4.0
    Z = rng.standard_normal((n, side + 2, side + 2))
    Z = k1[0] * Z[:, :-2, :] + k1[1] * Z[:, 1:-1, :] + k1[2] * Z[:, 2:, :]
    Z = k1[0] * Z[:, :, :-2] + k1[1] * Z[:, :, 1:-1] + k1[2] * Z[:, :, 2:]
    P = Z.reshape(n, side * side).T
    P = P - P.mean(axis=0, keepdims=True)
    return np.asfortranarray(unit_columns(P))


# the eight resident dictionaries of the serving workload: every m of
# {64, 144, 256, 512} with two atom counts of {256, 1024, 2048, 4096}
SERVING_DICTS = ((64, 256), (64, 1024), (144, 256), (144, 1024), (256, 1024), (256, 2048),
                 (512, 2048), (512, 4096))


def config_serving(rate: float = 2000.0, duration_s: float = 10.0, seed: int = 0,
                   pool: int = 50000, nmax: int = 50000, noise: float = 0.01):
    """Serving stream: Poisson arrivals at `rate` requests/s for duration_s;
    each request picks one of the eight dictionaries uniformly (unit-norm
    N(0,1)), n ~ log-uniform on [1, nmax] signals, and OMP with L ~ U{4..32}
    or Lasso (mode 2) with lambda1 ~ U[0.05, 0.3] at equal odds.  Signals are
    sparse combinations D a + 0.01 N(0,1) with s ~ U{1..16} non-zeros, drawn
    once into a pool of `pool` float32 columns per dictionary; a request codes
    a random contiguous window of its dictionary's pool.

    Returns (dicts, pools, reqs) with dicts a list of m x K float32 arrays,
    pools the matching m x pool float32 arrays, and reqs a dict of per-request
    arrays: arrival_s, dict, n, offset, algo (0 OMP / 1 Lasso), L, lambda1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dicts, pools = [], []
    for m, K in SERVING_DICTS:
        D = gaussian_dictionary(m, K, rng)
        s = rng.integers(1, 17, size=pool)
        X, _, _ = sparse_signals(D, pool, s, noise, rng)
        dicts.append(np.asfortranarray(D, dtype=np.float32))
        pools.append(np.asfortranarray(X, dtype=np.float32))
    count = max(1, int(rng.poisson(rate * duration_s)))
    arrival = np.sort(rng.random(count) * duration_s)
    dsel = rng.integers(0, len(SERVING_DICTS), size=count)
    nreq = np.minimum(nmax, np.floor(np.exp(rng.random(count) * np.log(nmax + 1))).astype(np.int64))
    nreq = np.maximum(nreq, 1)
    nreq = np.minimum(nreq, pool)
    offset = (rng.random(count) * (pool - nreq + 1)).astype(np.int64)
    algo = rng.integers(0, 2, size=count)
    L = rng.integers(4, 33, size=count)
    lam = 0.05 + 0.25 * rng.random(count)
    reqs = {"arrival_s": arrival, "dict": dsel, "n": nreq, "offset": offset, "algo": algo,
            "L": L, "lambda1": lam}
    return dicts, pools, reqs


def config_uneven_omp_device(n: int = 1000000, seed: int = 0, m: int = 512, K: int = 2048,
                             smax: int = 64, noise: float = 0.02, device=None,
                             chunk: int = 1 << 16):
    """config_uneven_omp drawn on a CUDA device with torch (for the full-size
    run, whose host draw takes minutes): same shapes and distributions (unit
    D, s_i ~ U{1..smax} distinct atoms with N(0,1) values, 0.02 N(0,1) noise,
    L_i = s_i + 4, eps_i = 0.5 ||noise_i||^2), a different random stream.
    Returns float32 CUDA tensors X (m x n, column-major view), D (m x K,
    column-major view), L (int32) and eps."""
    import torch
    dev = torch.device(device if device is not None else "cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    D = torch.randn((K, m), generator=g, device=dev, dtype=torch.float32)
    D = D / D.norm(dim=1, keepdim=True)
    s = torch.randint(1, smax + 1, (n,), generator=g, device=dev)
    Xr = torch.empty((n, m), device=dev, dtype=torch.float32)
    eps = torch.empty(n, device=dev, dtype=torch.float32)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        w = torch.ones((c1 - c0, K), device=dev)
        idx = torch.multinomial(w, smax, replacement=False, generator=g)
        vals = torch.randn((c1 - c0, smax), generator=g, device=dev)
        vals = vals * (torch.arange(smax, device=dev)[None, :] < s[c0:c1, None])
        A = torch.zeros((c1 - c0, K), device=dev)
        A.scatter_(1, idx, vals)
        E = noise * torch.randn((c1 - c0, m), generator=g, device=dev)
        Xr[c0:c1] = A @ D + E
        eps[c0:c1] = 0.5 * (E * E).sum(dim=1)
    L = (s + 4).to(torch.int32)
    return Xr.t(), D.t(), L, eps
