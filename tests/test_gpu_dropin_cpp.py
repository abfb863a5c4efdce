"""The drop-in C++ headers (include/spams_b200/*.h) compiled with g++ and run
like the reference's C++ demo, their outputs checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as ssp

from conftest import PKG, ROOT, matched_columns, rel_err, support_match
from oracle import oracle as O
from spams_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _read_csc(fn):
    with open(fn, "rb") as f:
        m, n, nnz = np.frombuffer(f.read(24), np.int64)
        colptr = np.frombuffer(f.read(8 * (n + 1)), np.int64)
        rows = np.frombuffer(f.read(4 * nnz), np.int32)
        vals = np.frombuffer(f.read(8 * nnz), np.float64)
    return ssp.csc_matrix((vals, rows, colptr), shape=(int(m), int(n)))


@pytest.mark.parametrize("std", ["c++14", "c++17"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_cpp_dropin(tmp_path, std, prec):
    exe = tmp_path / "dropin"
    lib = os.path.join(PKG, "lib")
    subprocess.run(["g++", f"-std={std}", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_demo.cpp"), "-o", str(exe),
                    "-L", lib, "-lspams_b200", f"-Wl,-rpath,{lib}"], check=True)
    X, D = W.config_lasso(n=400, seed=21, m=48, K=100, s=5, noise=0.01)
    dt = np.float64 if prec == "f64" else np.float32
    X = np.asfortranarray(X.astype(dt))
    D = np.asfortranarray(D.astype(dt))
    X.ravel(order="F").tofile(tmp_path / "X.bin")  # column-major, as Matrix<T>
    D.ravel(order="F").tofile(tmp_path / "D.bin")
    r = subprocess.run([str(exe), str(tmp_path), "48", "400", "100", prec], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caught: lasso : incompatible matrix dimensions" in r.stdout
    X64, D64 = X.astype(np.float64), D.astype(np.float64)
    tol_s, tol_v = (1.0, 1e-9) if prec == "f64" else (0.99, 1e-4)
    cases = {
        "omp": O.orc_omp(X64, D64, L=6, eps=0.0),
        "omp_eps": O.orc_omp(X64, D64, eps=0.05),
        "lasso_L10": O.orc_lasso(X64, D64, L=10, lambda1=0.15),
        "lasso_pos": O.orc_lasso(X64, D64, lambda1=0.1, pos=True),
        "lasso_gram": O.orc_lasso(X64, D64, lambda1=0.15),
        "lasso_qq": O.orc_lasso(X64, D64, lambda1=0.15),
        "lasso_chol_l2err": O.orc_lasso(X64, D64, lambda1=0.05, mode=1, cholesky=True),
    }
    # the Cholesky implementation on the demo's products G (+1e-10) and D^T X,
    # formed the same way (double sums rounded to the precision)
    Gq = (D64.T @ D64 + 1e-10 * np.eye(100)).astype(dt).astype(np.float64)
    qq = (D64.T @ X64).astype(dt).astype(np.float64)
    cases["lasso_gram_chol_l1"] = O.orc_lasso(X64, None, Q=Gq, q=qq, L=48, lambda1=1.0, mode=0,
                                              cholesky=True)
    cases["lasso_qq_ols_l2err"] = O.orc_lasso(X64, None, Q=Gq, q=qq, lambda1=0.05, mode=1,
                                              ols=True)
    rr, ii = np.meshgrid(np.arange(48), np.arange(400), indexing="ij")
    B = (7 * rr + 3 * ii) % 10 < 7
    B[:, 0] = True
    B[:, 1] = False
    cases["omp_mask"] = O.orc_omp_mask(X64, D64, B, L=6, eps=0.0, lambda1=0.0)
    lm = O.orc_lasso_mask(X64, D64, B, lambda1=0.1).copy()
    lm.eliminate_zeros()
    cases["lasso_mask"] = lm
    # In single precision the L1COEFFS stop of the Cholesky variant lands
    # within float rounding of ||alpha||_1 = lambda on a few columns (the
    # reference's float build leaves its double build there as well): those
    # columns may take one atom more or fewer; the others agree as usual.
    loose_f32 = {"lasso_gram_chol_l1": 0.95}
    for name, ref in cases.items():
        a = _read_csc(tmp_path / f"{name}.csc")
        assert a.shape == ref.shape, name
        ts = loose_f32.get(name, tol_s) if prec == "f32" else tol_s
        assert support_match(a, ref) >= ts, name
        gram = name.startswith(("lasso_gram", "lasso_qq"))
        am, bm = matched_columns(a, ref) if ts < tol_s else (a, ref)
        assert rel_err(am, bm) <= (1e-6 if gram and prec == "f64" else tol_v), name
        if name == "lasso_gram_chol_l1":
            l1 = np.asarray(abs(a).sum(axis=0)).ravel()
            assert l1.max() <= 1.0 * (1 + (1e-9 if prec == "f64" else 1e-5)), name
