"""The minibatch step of online dictionary learning (Trainer::train,
dictLearn/dicts.h:526-603) on CUDA tensors.

    step = spams_b200.MinibatchStep(m=144, K=1024, batch=1024, lambda1=0.1)
    it = torch.zeros(1, dtype=torch.int64, device="cuda")
    step(D, X, it, perm=perm, A=A, B=B)      # one minibatch; it += 1 on the device

D (m x K), X (m x M), A (K x K) and B (m x K) are column-major float32 CUDA
tensors (the .t() views of row-major K x m, M x m, K x K, K x m tensors).  A
step enqueues everything on the current stream without synchronising, so a
step (after a first eager one) can be captured in a CUDA graph and replayed
for every minibatch: the minibatch index comes from the device counter `it`.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

from . import _lib

# constraint_type, decomp/decomp.h:95
L1COEFFS, L2ERROR, PENALTY, SPARSITY, L2ERROR2, PENALTY2 = 0, 1, 2, 3, 4, 5


def _colmajor(t, rows: int, cols: int, name: str) -> None:
    import torch
    if not (t.is_cuda and t.dtype == torch.float32 and tuple(t.shape) == (rows, cols)
            and t.stride(0) == 1 and t.stride(1) == rows):
        raise ValueError(f"dictionary learning: {name} must be a column-major float32 CUDA "
                         f"tensor of shape ({rows}, {cols})")


class _DevArray:
    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 2}


class MinibatchStep:
    """One minibatch step of the online dictionary-learning loop (see the
    module docstring).  mode / lambda1 / lambda2 / posAlpha follow
    ParamDictLearn: modes 0-2 code with LARS-Lasso, 3-5 with OMP."""

    def __init__(self, m: int, K: int, batch: int, mode: int = PENALTY, lambda1: float = 0.1,
                 lambda2: float = 0.0, posAlpha: bool = False, precision: Optional[int] = None,
                 device: int = 0):
        h = C.c_void_p()
        prec = _lib.SC_PREC_FP32 if precision is None else int(precision)
        _lib.check(_lib.lib().sc_dl_create(int(device), int(m), int(K), int(batch), int(mode),
                                           float(lambda1), float(lambda2), int(bool(posAlpha)),
                                           prec, C.byref(h)))
        self._h = h
        self.m, self.K, self.batch = int(m), int(K), int(batch)

    def close(self) -> None:
        if self._h:
            _lib.check(_lib.lib().sc_dl_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __call__(self, D, X, it, perm=None, A=None, B=None, beta: float = 1.0,
                 gamma: float = 1.0, stream=None) -> None:
        import torch
        _colmajor(D, self.m, self.K, "D")
        _colmajor(X, self.m, X.shape[1], "X")
        if not (it.is_cuda and it.dtype == torch.int64 and it.numel() >= 1):
            raise ValueError("dictionary learning: it must be an int64 CUDA tensor")
        if perm is not None and not (perm.is_cuda and perm.dtype == torch.int32
                                     and perm.numel() == X.shape[1]):
            raise ValueError("dictionary learning: perm must be an int32 CUDA tensor of M entries")
        if A is not None:
            _colmajor(A, self.K, self.K, "A")
        if B is not None:
            _colmajor(B, self.m, self.K, "B")
        s = stream if stream is not None else torch.cuda.current_stream(D.device)

        def vp(t):
            return C.c_void_p(t.data_ptr()) if t is not None else None

        _lib.check(_lib.lib().sc_dl_step_f32(
            self._h, vp(D), vp(X), int(X.shape[1]), vp(perm), vp(it), vp(A), vp(B),
            float(beta), float(gamma), C.c_void_p(s.cuda_stream)))

    def profile(self, on: bool = True) -> None:
        """Record the coding stages' device times of later (eager) steps, read
        with spams_b200.last_profile()."""
        _lib.check(_lib.lib().sc_dl_profile(self._h, int(bool(on))))

    def codes(self):
        """Copies of the last step's codes as CUDA tensors (colptr, rows, vals)."""
        import torch
        cp, r, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _lib.check(_lib.lib().sc_dl_codes(self._h, C.byref(cp), C.byref(r), C.byref(v)))
        colptr = torch.as_tensor(_DevArray(cp.value, self.batch + 1, "<i8"), device="cuda").clone()
        nnz = int(colptr[-1].item())
        rows = torch.as_tensor(_DevArray(r.value, max(nnz, 1), "<i4"), device="cuda")[:nnz].clone()
        vals = torch.as_tensor(_DevArray(v.value, max(nnz, 1), "<f4"), device="cuda")[:nnz].clone()
        return colptr, rows, vals
