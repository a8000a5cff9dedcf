"""Row-sharded SpMV over several processes (one per GPU), the multi-GPU form
of the CRS path; the reference is single-node OpenMP only.

The rows of a square CRS matrix are cut into ``world`` contiguous ranges
balanced by nonzeros (``row_bounds``); rank k keeps rows [b_k, b_{k+1}) with
their global column indices and owns the same range of x and y.  One product
is a single exchange and a local product: every rank's x slice is gathered
into the full x (one ``torch.distributed.all_gather`` of slices padded to the
longest range), then the rank multiplies its rows locally —
on the GPU through the CRS kernels (the default), or through any callable
``local_spmv(alpha, x_full, beta, y_local)`` given at construction.

Every rank must call ``spmv`` the same number of times in the same order
(the gather is a collective).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import formats as F


def row_bounds(Rst, world: int) -> np.ndarray:
    """world + 1 row bounds: range k holds about nnz / world nonzeros (whole
    rows; a rank may get an empty range when rows are few and long)."""
    Rst = np.asarray(Rst, dtype=np.int64)
    m = len(Rst) - 1
    if world < 1:
        raise ValueError("row_bounds: world must be >= 1")
    nz = int(Rst[-1])
    targets = (np.arange(1, world, dtype=np.int64) * nz) // world
    inner = np.searchsorted(Rst, targets, side="right") - 1  # last row starting at or before the target
    b = np.concatenate([[0], np.clip(inner, 0, m), [m]]).astype(np.int64)
    return np.maximum.accumulate(b)


class RowShardedCRS:
    """This rank's rows of a square CRS matrix (host arrays of the whole
    matrix, or at least its row pointer and this rank's rows)."""

    def __init__(self, m: int, n: int, Rst, Col, Val, rank: int | None = None, world: int | None = None,
                 device="cuda", dtype=torch.float64, local_spmv=None, group=None):
        if m != n:
            raise ValueError("RowShardedCRS: the matrix must be square (x and y share the row ranges)")
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else rank
        self.world = dist.get_world_size(group) if world is None else world
        self.m, self.n = m, n
        self.bounds = row_bounds(Rst, self.world)
        self.r0, self.r1 = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
        self.maxlen = int(np.max(np.diff(self.bounds))) if self.world else 0
        Rst = np.asarray(Rst, dtype=np.int64)
        k0, k1 = int(Rst[self.r0]), int(Rst[self.r1])
        self.Rst_l = (Rst[self.r0:self.r1 + 1] - k0).astype(np.int32)
        self.Col_l = np.asarray(Col[k0:k1], dtype=np.int32)
        self.Val_l = np.asarray(Val[k0:k1])
        self.device, self.dtype = torch.device(device), dtype
        self._local = local_spmv
        if local_spmv is None:
            self.A_l = F.spMtxCRS.from_host(self.r1 - self.r0, n, self.Rst_l, self.Col_l, self.Val_l, dtype=dtype,
                                            device=device)
        self._pad = torch.zeros(self.maxlen, dtype=dtype, device=self.device)
        self._full = torch.zeros(self.world * self.maxlen, dtype=dtype, device=self.device)

    @property
    def local_rows(self) -> int:
        return self.r1 - self.r0

    def gather_x(self, x_local: torch.Tensor) -> torch.Tensor:
        """The full x from every rank's slice (one all-gather)."""
        if x_local.numel() != self.local_rows:
            raise ValueError("gather_x: x_local must hold this rank's rows of x")
        self._pad[:self.local_rows].copy_(x_local)
        dist.all_gather(list(self._full.view(self.world, self.maxlen).unbind(0)), self._pad, group=self.group)
        parts = [self._full[k * self.maxlen:k * self.maxlen + int(self.bounds[k + 1] - self.bounds[k])]
                 for k in range(self.world)]
        return torch.cat(parts)

    def spmv(self, x_local: torch.Tensor, alpha: float = 1.0, beta: float = 0.0,
             y_local: torch.Tensor | None = None) -> torch.Tensor:
        """y_local = alpha * (A x)[rows of this rank] + beta * y_local."""
        x_full = self.gather_x(x_local)
        if y_local is None:
            y_local = torch.zeros(self.local_rows, dtype=self.dtype, device=self.device)
        if self.local_rows == 0:
            return y_local
        if self._local is not None:
            self._local(alpha, x_full, beta, y_local)
        else:
            st = F.sparse_mv(F.SPARSE_OPERATION_NON_TRANSPOSE, alpha, self.A_l, F.sparse_matrix_descr(), x_full, beta,
                             y_local)
            if st.code != 0:
                raise RuntimeError(f"RowShardedCRS.spmv: status {st.code}")
        return y_local
