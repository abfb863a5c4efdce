"""spams_b200: batched OMP / LARS-Lasso sparse coding on one B200.

Drop-in for SPAMS' Python coding entry points (swig/python/spams.py:109-198):

    alpha = spams_b200.omp(X, D, L=10, eps=0.)          # scipy.sparse.csc_matrix
    alpha = spams_b200.lasso(X, D, lambda1=0.15, mode=2)

X and D are Fortran-ordered float32/float64 numpy arrays (m x n, m x K).
Calls go through the C ABI of libspams_b200.so; all arithmetic runs on the
GPU.  `omp_device` / `lasso_device` take CUDA tensors and leave the CSC on the
device.  `Server` keeps dictionaries resident and codes a stream of requests
(continuous batching, device-memory admission, latency percentiles);
`MinibatchStep` is the graph-capturable minibatch step of online dictionary
learning.
"""
from ._lib import (SC_KERNEL_AUTO, SC_KERNEL_CTA, SC_KERNEL_WARP,  # noqa: F401
                   SC_L1COEFFS, SC_L2ERROR, SC_PENALTY, SC_PREC_BF16X3, SC_PREC_FP32,
                   ScError, device_count, last_error, last_profile, lib)
from .api import (corr_device, lasso, lasso_device, lassoMask, omp, omp_device,  # noqa: F401
                  ompMask)
from .serve import Server, request  # noqa: F401
from .dictlearn import MinibatchStep  # noqa: F401

L1COEFFS, L2ERROR, PENALTY = SC_L1COEFFS, SC_L2ERROR, SC_PENALTY
