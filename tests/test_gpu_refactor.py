"""FP64 refactor of the single-precision LARS inverse Gram.

By default it only triggers when an added atom's pivot falls below 1e-3 of
its diagonal, which well-conditioned dictionaries never reach (the codes are
the same bits as with the refactor off); on every add it costs about 3.5x the
coding time of the 100k-signal lasso workload and buys accuracy on
near-duplicate atoms, where the incremental single-precision update drifts."""
import numpy as np
import pytest

from conftest import rel_err, support_match

import spams_b200
from spams_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = a.tocsc(), b.tocsc()
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    np.testing.assert_array_equal(a.data, b.data)


def test_default_refactor_leaves_well_conditioned_codes_unchanged():
    X, D = W.config_lasso(20000)
    Xf, Df = X.astype(np.float32), D.astype(np.float32)
    _same(spams_b200.lasso(Xf, Df, lambda1=0.15), spams_b200.lasso(Xf, Df, lambda1=0.15,
                                                                  refactor="never"))


def test_refactor_on_every_add_tracks_the_fp64_path_on_near_duplicate_atoms():
    rng = np.random.Generator(np.random.PCG64(4))
    m, K0 = 64, 150
    D0 = W.gaussian_dictionary(m, K0, rng)
    dup = D0[:, :50] + 1e-2 * rng.standard_normal((m, 50))  # pairs with correlation ~0.9999
    D = np.hstack([D0, dup])
    D = np.asfortranarray(D / np.linalg.norm(D, axis=0, keepdims=True))
    X, _, _ = W.sparse_signals(D, 500, 8, 0.02, rng)
    ref = O.orc_lasso(X, D, lambda1=0.02)
    Xf, Df = X.astype(np.float32), D.astype(np.float32)
    never = spams_b200.lasso(Xf, Df, lambda1=0.02, refactor="never")
    always = spams_b200.lasso(Xf, Df, lambda1=0.02, refactor="always")
    assert support_match(always, ref) >= max(0.985, support_match(never, ref))
    assert rel_err(always, ref) <= rel_err(never, ref)
    # the warp and CTA kernels refactor alike
    _same(spams_b200.lasso(Xf, Df, lambda1=0.02, refactor="always", kernel="warp"),
          spams_b200.lasso(Xf, Df, lambda1=0.02, refactor="always", kernel="cta"))
