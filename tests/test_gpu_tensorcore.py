"""The tcgen05 BF16-split correlation product against an FP64 reference."""
import numpy as np
import pytest
import torch

import spams_b200

pytestmark = pytest.mark.gpu


def _colmajor(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


# signal tiles of 128, 64, 32 and 16 signals (the resident split of a tile
# shrinks as m grows), atom tiles spread over groups when the signal tiles
# are few (n = 257, 50), and m = 2100, beyond the resident form, on the
# streaming kernel
@pytest.mark.parametrize("m,K,n", [(64, 128, 128), (256, 512, 1000), (100, 200, 333),
                                   (512, 2048, 4096), (144, 1024, 257), (1000, 256, 700),
                                   (2000, 128, 50), (2100, 256, 300)])
def test_bf16x3_correlation_close_to_fp64(m, K, n):
    rng = np.random.Generator(np.random.PCG64(m * 7 + K))
    D = rng.standard_normal((m, K)).astype(np.float32)
    D /= np.linalg.norm(D, axis=0, keepdims=True)
    X = rng.standard_normal((m, n)).astype(np.float32)
    ref = D.astype(np.float64).T @ X.astype(np.float64)
    C = spams_b200.corr_device(_colmajor(D), _colmajor(X), precision=spams_b200.SC_PREC_BF16X3)
    torch.cuda.synchronize()
    got = C.cpu().numpy().astype(np.float64)
    scale = np.linalg.norm(X, axis=0)[None, :]  # |d^T x| <= ||x||
    err = np.abs(got - ref) / scale
    assert err.max() < 2e-5, err.max()
    C32 = spams_b200.corr_device(_colmajor(D), _colmajor(X))
    err32 = np.abs(C32.cpu().numpy() - ref) / scale
    assert err32.max() < 2e-6
