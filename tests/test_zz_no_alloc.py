"""The allocation-free correlation entry point (sc_corr_bf16x3_noalloc_f32).

Some callers cannot allocate device memory: a serving process that has
already given its free memory to its own pool, or code that must not incur
the device synchronisation of cudaMalloc / cudaFree.  This entry point stages
its BF16 hi / lo operands in a fixed 16 MiB array inside the library instead
of the engine's allocations.  The test calls it through the C ABI twice in a
row and checks each result against the allocating entry point
(sc_corr_f32_dev with SC_PREC_BF16X3), checks that a warm call on a
non-default stream leaves the device's free memory unchanged, and that a call
too large for the fixed array is refused.  The file name makes pytest collect
it last.
"""
import ctypes as C

import numpy as np
import pytest

import spams_b200
from spams_b200 import _lib

pytestmark = pytest.mark.gpu

# the BF16x3 correlation tolerance of the other GPU tests, relative to ||x||
TOL = 2e-5


def _colmajor(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def _noalloc(torch, D, X, out=None, stream=None):
    m, K = D.shape
    n = X.shape[1]
    if out is None:
        out = torch.full((n, K), float("nan"), dtype=torch.float32, device=X.device).t()
    s = stream if stream is not None else torch.cuda.current_stream()
    st = _lib.lib().sc_corr_bf16x3_noalloc_f32(
        C.c_void_p(D.data_ptr()), m, K, C.c_void_p(X.data_ptr()), n, C.c_void_p(out.data_ptr()),
        out.stride(1), C.c_void_p(s.cuda_stream))
    return st, out


@pytest.mark.parametrize("shape", [((256, 512, 3000), (100, 200, 777))])
def test_noalloc_matches_allocating_entry_twice(shape):
    import torch
    for call, (m, K, n) in enumerate(shape):
        rng = np.random.Generator(np.random.PCG64(100 + call))
        D = rng.standard_normal((m, K)).astype(np.float32)
        D /= np.linalg.norm(D, axis=0, keepdims=True)
        X = rng.standard_normal((m, n)).astype(np.float32)
        Dt, Xt = _colmajor(torch, D), _colmajor(torch, X)
        st, got = _noalloc(torch, Dt, Xt)
        assert st == _lib.SC_OK, _lib.last_error()
        ref = spams_b200.corr_device(Dt, Xt, precision=spams_b200.SC_PREC_BF16X3)
        torch.cuda.synchronize()
        scale = np.linalg.norm(X, axis=0)[None, :]
        diff = np.abs(got.cpu().numpy() - ref.cpu().numpy()) / scale
        assert np.isfinite(got.cpu().numpy()).all()
        assert diff.max() <= TOL
        exact = D.astype(np.float64).T @ X.astype(np.float64)
        assert (np.abs(got.cpu().numpy() - exact) / scale).max() <= TOL


def test_noalloc_warm_call_allocates_no_device_memory():
    """A warm call on a non-default stream: the device's free memory (as the
    driver reports it) is the same before and after, and the result is the
    allocating entry point's."""
    import torch
    m, K, n = 144, 1024, 2000
    rng = np.random.Generator(np.random.PCG64(7))
    D = rng.standard_normal((m, K)).astype(np.float32)
    D /= np.linalg.norm(D, axis=0, keepdims=True)
    X = rng.standard_normal((m, n)).astype(np.float32)
    Dt, Xt = _colmajor(torch, D), _colmajor(torch, X)
    out = torch.empty((n, K), dtype=torch.float32, device="cuda").t()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    st, _ = _noalloc(torch, Dt, Xt, out, side)  # warm: address looked up, kernels loaded
    assert st == _lib.SC_OK, _lib.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    out.fill_(float("nan"))
    side.wait_stream(torch.cuda.current_stream())
    st, _ = _noalloc(torch, Dt, Xt, out, side)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert st == _lib.SC_OK, _lib.last_error()
    assert free1 == free0
    ref = spams_b200.corr_device(Dt, Xt, precision=spams_b200.SC_PREC_BF16X3)
    torch.cuda.synchronize()
    scale = np.linalg.norm(X, axis=0)[None, :]
    assert (np.abs(out.cpu().numpy() - ref.cpu().numpy()) / scale).max() <= TOL


def test_noalloc_rejects_calls_beyond_the_fixed_scratch():
    import torch
    m, K, n = 512, 1024, 8192  # 256 + 4 * 512 * (1024 + 8192) bytes > 16 MiB
    D = torch.zeros((K, m), dtype=torch.float32, device="cuda").t()
    X = torch.zeros((n, m), dtype=torch.float32, device="cuda").t()
    st, _ = _noalloc(torch, D, X)
    assert st == _lib.SC_ERR_CAPACITY
    assert "16777216" in _lib.last_error()
