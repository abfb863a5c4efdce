"""Generate the golden fixtures of tests/golden/ from the SPAMS reference itself.

    python tests/golden/make_golden.py        (needs oracle/_ref, i.e. the
                                               reference sources at build time)

Each case draws seeded inputs with spams_b200.workloads, stores them as
float32 (so the float64 run sees exactly the same numbers), and records the
reference's CSC output for T=double and T=float, plus the regularisation
path where the case asks for one.  The reference has no known-answer tests
of its own; these vectors are its outputs on our inputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spams-devel_b200"))

from oracle import oracle as O  # noqa: E402
from spams_b200 import workloads as W  # noqa: E402


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def cases():
    out = []
    # OMP, unit-norm Gaussian signals (the plain OMP workload at n=300)
    X, D = W.config_omp_small(300, seed=1)
    out.append(dict(name="omp_L10", algo="omp", X=X, D=D, kw=dict(L=10, eps=0.0), path=False))
    # OMP demo style: un-normalised X, eps only / L only, lambda stop, path
    r = rng(2)
    D = W.gaussian_dictionary(32, 96, r)
    X = np.asfortranarray(r.standard_normal((32, 120)))
    out.append(dict(name="omp_eps", algo="omp", X=X, D=D, kw=dict(eps=8.0), path=False))
    out.append(dict(name="omp_lambda", algo="omp", X=X, D=D, kw=dict(L=12, lambda1=0.3), path=False))
    out.append(dict(name="omp_path", algo="omp", X=X[:, :20], D=D, kw=dict(L=7, eps=0.5), path=True))
    # per-signal L / eps (the uneven batched workload at small size)
    X3, D3, L3, e3 = W.config_uneven_omp(n=150, seed=3, m=48, K=160, smax=10, noise=0.02)
    out.append(dict(name="omp_vec", algo="omp", X=X3, D=D3, kw=dict(L=L3, eps=e3), path=False))
    # L larger than m, K not a multiple of anything
    r = rng(4)
    D = W.gaussian_dictionary(9, 37, r)
    X = np.asfortranarray(r.standard_normal((9, 40)))
    out.append(dict(name="omp_L_gt_m", algo="omp", X=X, D=D, kw=dict(L=20), path=False))
    out.append(dict(name="omp_eps_all", algo="omp", X=X, D=D, kw=dict(eps=1e9), path=False))
    # LARS-Lasso: the sparse-signal workload at reduced size
    X, D = W.config_lasso(n=300, seed=5, m=64, K=128, s=8, noise=0.01)
    out.append(dict(name="lasso_pen", algo="lasso", X=X, D=D, kw=dict(lambda1=0.15), path=False))
    out.append(dict(name="lasso_pen_L10", algo="lasso", X=X, D=D, kw=dict(lambda1=0.05, L=10), path=False))
    out.append(dict(name="lasso_pos", algo="lasso", X=X, D=D, kw=dict(lambda1=0.1, pos=True), path=False))
    out.append(dict(name="lasso_l1", algo="lasso", X=X, D=D, kw=dict(lambda1=1.0, mode=0), path=False))
    out.append(dict(name="lasso_l2err", algo="lasso", X=X, D=D, kw=dict(lambda1=0.05, mode=1), path=False))
    out.append(dict(name="lasso_enet", algo="lasso", X=X, D=D, kw=dict(lambda1=0.1, lambda2=0.5), path=False))
    out.append(dict(name="lasso_path", algo="lasso", X=X[:, :10], D=D, kw=dict(lambda1=0.05, L=12), path=True))
    out.append(dict(name="lasso_big_lambda", algo="lasso", X=X[:, :30], D=D, kw=dict(lambda1=100.0), path=False))
    # the Cholesky implementation (lasso / coreLARS) and its ols projection
    out.append(dict(name="lasso_ols", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=0.1, ols=True), path=False))
    out.append(dict(name="lasso_chol_l1", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=1.0, mode=0, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_pen", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=0.15, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_l2err", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=0.05, mode=1, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_pos", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=0.1, pos=True, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_path", algo="lasso", X=X[:, :10], D=D, kw=dict(lambda1=0.05, L=12, cholesky=True), path=True))
    out.append(dict(name="lasso_ols_l2err", algo="lasso", X=X[:, :120], D=D, kw=dict(lambda1=0.05, mode=1, ols=True), path=False))
    # Gaussian signals, LARS runs long with drops (dense active sets, small lambda)
    r = rng(6)
    D = W.gaussian_dictionary(24, 70, r)
    X = np.asfortranarray(r.standard_normal((24, 80)))
    out.append(dict(name="lasso_dense", algo="lasso", X=X, D=D, kw=dict(lambda1=0.01), path=False))
    out.append(dict(name="lasso_dense_pos", algo="lasso", X=X, D=D, kw=dict(lambda1=0.01, pos=True), path=False))
    # the Cholesky implementation with drops (downDateLasso) in every mode
    out.append(dict(name="lasso_chol_dense", algo="lasso", X=X, D=D, kw=dict(lambda1=0.01, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_dense_pos", algo="lasso", X=X, D=D, kw=dict(lambda1=0.01, pos=True, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_dense_l2err", algo="lasso", X=X, D=D, kw=dict(lambda1=2.0, mode=1, cholesky=True), path=False))
    out.append(dict(name="lasso_chol_dense_l1", algo="lasso", X=X, D=D, kw=dict(lambda1=3.0, mode=0, cholesky=True), path=False))
    out.append(dict(name="lasso_ols_dense", algo="lasso", X=X, D=D, kw=dict(lambda1=0.01, ols=True), path=False))
    # precomputed products (Q, q)
    X, D = W.config_lasso(n=60, seed=7, m=40, K=100, s=6, noise=0.01)
    X = X.astype(np.float32).astype(np.float64)
    D = D.astype(np.float32).astype(np.float64)
    Q = D.T @ D
    q = D.T @ X
    out.append(dict(name="lassoQq", algo="lassoQq", X=X, D=D, Q=Q, q=q, kw=dict(lambda1=0.1), path=False))
    out.append(dict(name="lassoQq_ols", algo="lassoQq", X=X, D=D, Q=Q, q=q, kw=dict(lambda1=0.1, ols=True), path=False))
    out.append(dict(name="lassoQq_chol_l1", algo="lassoQq", X=X, D=D, Q=Q, q=q, kw=dict(lambda1=1.0, mode=0, cholesky=True), path=False))
    # masked variants: random observed rows (70 %), plus one fully observed,
    # one unobserved and one mostly observed column.  ompMask gets L, eps and
    # lambda explicitly: the reference facade points eps / lambda at an
    # out-of-scope local when they are not given (cpp_library/spams.h:323-333)
    r = rng(8)
    D = W.gaussian_dictionary(40, 120, r)
    X, _, _ = W.sparse_signals(D, 160, 6, 0.05, r)
    B = r.random((40, 160)) < 0.7
    B[:, 0] = True
    B[:, 1] = False
    B[:5, 2] = False
    B = B.astype(np.uint8)
    out.append(dict(name="omp_mask", algo="omp_mask", X=X, D=D, B=B,
                    kw=dict(L=8, eps=0.02, lambda1=0.0), path=True))
    out.append(dict(name="lasso_mask", algo="lasso_mask", X=X, D=D, B=B,
                    kw=dict(lambda1=0.05), path=False))
    out.append(dict(name="lasso_mask_l2err_pos", algo="lasso_mask", X=X, D=D, B=B,
                    kw=dict(lambda1=0.3, mode=1, pos=True), path=False))
    return out


def run(case, dt):
    X = case["X"].astype(np.float32).astype(dt)
    D = case["D"].astype(np.float32).astype(dt)
    kw = dict(case["kw"])
    for k in ("eps", "lambda1"):
        if case["algo"] == "omp" and k in kw and np.ndim(kw[k]) > 0:
            kw[k] = np.asarray(kw[k]).astype(np.float32).astype(dt)
    if case["algo"] == "omp":
        return O.ref_omp(X, D, return_reg_path=case["path"], **kw)
    if case["algo"] == "omp_mask":
        return O.ref_omp_mask(X, D, case["B"], return_reg_path=case["path"], **kw)
    if case["algo"] == "lasso_mask":
        return O.ref_lasso_mask(X, D, case["B"], **kw)
    if case["algo"] == "lassoQq":
        Q = case["Q"].astype(np.float32).astype(dt)
        q = case["q"].astype(np.float32).astype(dt)
        return O.ref_lasso(X, Q=Q, q=q, return_reg_path=case["path"], **kw)
    return O.ref_lasso(X, D, return_reg_path=case["path"], **kw)


def main():
    O.build_ref()
    for case in cases():
        rec = dict(X=case["X"].astype(np.float32), D=case["D"].astype(np.float32),
                   algo=np.asarray(case["algo"]))
        for k, v in case["kw"].items():
            v = np.asarray(v)
            # per-signal float arrays were rounded to float32 for both runs;
            # scalars were passed as given
            rec["kw_" + k] = v.astype(np.float32) if (v.dtype.kind == "f" and v.ndim > 0) else v
        if "B" in case:
            rec["B"] = case["B"]
        if "Q" in case:
            rec["Q"] = case["Q"].astype(np.float32)
            rec["q"] = case["q"].astype(np.float32)
        for tag, dt in (("f64", np.float64), ("f32", np.float32)):
            res = run(case, dt)
            a, path = res if case["path"] else (res, None)
            a = a.tocsc()
            rec[f"{tag}_shape"] = np.asarray(a.shape)
            rec[f"{tag}_indptr"] = a.indptr.astype(np.int64)
            rec[f"{tag}_indices"] = a.indices.astype(np.int32)
            rec[f"{tag}_data"] = a.data.astype(dt)
            if path is not None:
                rec[f"{tag}_path"] = path.astype(dt)
        fn = os.path.join(HERE, case["name"] + ".npz")
        np.savez_compressed(fn, **rec)
        print(fn, os.path.getsize(fn))


if __name__ == "__main__":
    main()
