"""Column sharding of a coding job over several GPUs (one process per GPU).

Signals are independent (the reference codes them in an OpenMP loop over
columns, decomp/decomp.h:367 and :1611), so a job splits into contiguous
column blocks with no communication on the data path: every rank codes its
block against the same dictionary on its own GPU, and the per-block CSC
results are joined by offsetting their column pointers.  The only collective
is the final gather of the results to one rank (or to all).
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np
import scipy.sparse as ssp


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, end) of rank's contiguous block when n columns are split over
    `world` ranks as evenly as possible (the first n % world get one more)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("shard_bounds: bad world / rank")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def concat_csc(parts: Sequence[ssp.csc_matrix], n_rows: Optional[int] = None) -> ssp.csc_matrix:
    """Join column blocks (in rank order) into one CSC matrix: rows and values
    are concatenated, each block's column pointers are shifted by the nonzeros
    before it.  Empty 0 x 0 blocks (the reference's cleared output) count as
    blocks of zero columns."""
    parts = [p.tocsc() for p in parts]
    m = n_rows if n_rows is not None else max((p.shape[0] for p in parts), default=0)
    n = sum(p.shape[1] for p in parts)
    indptr = np.zeros(n + 1, dtype=np.int64)
    indices, data = [], []
    col, off = 0, 0
    for p in parts:
        k = p.shape[1]
        indptr[col + 1:col + k + 1] = off + p.indptr[1:].astype(np.int64)
        indices.append(p.indices)
        data.append(p.data)
        col += k
        off += p.nnz
    dtype = parts[0].dtype if parts else np.float64
    return ssp.csc_matrix((np.concatenate(data) if data else np.zeros(0, dtype),
                           np.concatenate(indices) if indices else np.zeros(0, np.int32), indptr),
                          shape=(m, n))


def _gather_csc(part: ssp.csc_matrix, group, dst: Optional[int]):
    """Gather every rank's CSC block as flat arrays (tensor collectives; no
    pickling): column counts, row indices and values, each padded to the
    largest block.  Returns the blocks in rank order on `dst` (every rank
    when dst is None), else None."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = (torch.device("cuda", torch.cuda.current_device())
           if dist.get_backend(group) == "nccl" else torch.device("cpu"))
    p = part.tocsc()
    meta = torch.tensor([p.shape[0], p.shape[1], p.nnz], dtype=torch.int64, device=dev)
    metas = [torch.zeros_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    metas = [[int(v) for v in m.cpu()] for m in metas]
    maxc = max(1, max(m[1] for m in metas))
    maxz = max(1, max(m[2] for m in metas))
    vdt = torch.float64 if p.dtype == np.float64 else torch.float32
    counts = torch.zeros(maxc, dtype=torch.int64, device=dev)
    rows = torch.zeros(maxz, dtype=torch.int32, device=dev)
    vals = torch.zeros(maxz, dtype=vdt, device=dev)
    if p.shape[1]:
        counts[:p.shape[1]] = torch.from_numpy(np.diff(p.indptr).astype(np.int64))
    if p.nnz:
        rows[:p.nnz] = torch.from_numpy(p.indices.astype(np.int32))
        vals[:p.nnz] = torch.from_numpy(np.ascontiguousarray(p.data))
    mine = dst is None or rank == dst
    out = []
    for t in (counts, rows, vals):
        bufs = [torch.zeros_like(t) for _ in range(world)] if mine else None
        if dst is None:
            dist.all_gather(bufs, t, group=group)
        else:
            dist.gather(t, bufs, dst=dst, group=group)
        out.append(bufs)
    if not mine:
        return None
    parts = []
    for r, (m, nc, nz) in enumerate(metas):
        indptr = np.zeros(nc + 1, np.int64)
        indptr[1:] = np.cumsum(out[0][r][:nc].cpu().numpy())
        parts.append(ssp.csc_matrix((out[2][r][:nz].cpu().numpy(), out[1][r][:nz].cpu().numpy(),
                                     indptr), shape=(m, nc)))
    return parts


def code_sharded(code: Callable, X: np.ndarray, *args, group=None, dst: Optional[int] = 0,
                 **kwargs) -> Optional[ssp.csc_matrix]:
    """Code the columns of X over the ranks of a torch.distributed group.

    Every rank passes the same X (m x n) and dictionary arguments; rank r
    codes columns shard_bounds(n, world, r) with `code(X_block, *args,
    **kwargs)` (spams_b200.omp or spams_b200.lasso on the rank's GPU).  The
    blocks are gathered to `dst` (None: to every rank) as flat CSC arrays,
    and that rank returns the joined K x n matrix; the other ranks return
    None.  Per-signal arrays in kwargs (L / eps / lambda1 with n entries) are
    sliced to the block."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = X.shape[1]
    s, e = shard_bounds(n, world, rank)
    kw = {}
    for k, v in kwargs.items():
        if isinstance(v, np.ndarray) and v.ndim == 1 and v.size == n and n > 1:
            v = v[s:e]
        kw[k] = v
    part = code(np.asfortranarray(X[:, s:e]), *args, **kw)
    parts = _gather_csc(part, group, dst)
    if parts is None:
        return None
    K = max(p.shape[0] for p in parts)
    return concat_csc(parts, K)
