"""Row-sharded SpMV over several processes (one per GPU), the multi-GPU form
of the CRS path; the reference is single-node OpenMP only.

The rows of a square CRS matrix are cut into ``world`` contiguous ranges
balanced by nonzeros (``row_bounds``); rank k keeps rows [b_k, b_{k+1}) and
owns the same range of x and y.  Its rows are split by column into

* the diagonal block (columns in [b_k, b_{k+1})), which needs only the
  rank's own x slice, and
* the off-diagonal block, whose columns are renumbered over the list of
  remote columns the rows actually reference (the rank's "ghost" columns).

One product: the exchange of x starts asynchronously, the diagonal block's
product runs while it is in flight (y = alpha*A_diag*x_own + beta*y), then
y += alpha*A_off*x_ghost once the ghosts have arrived.  Two exchanges:

* ``"allgather"``: every rank's slice (padded to the longest range) is
  all-gathered into one reusable buffer; the off-diagonal columns index that
  padded buffer directly, so nothing is concatenated;
* ``"halo"``: each rank sends every other rank exactly the x entries that
  rank's off-diagonal block references (one ``all_to_all_single`` with
  per-rank sizes fixed at construction); for banded and stencil matrices
  only neighbouring ranks exchange, and only the band's width of entries.

With NCCL the collectives run over NVLink on NCCL's own stream (no
multicast loads); ``work.wait()`` orders the off-diagonal product after
them on the current stream.  The local products run on the GPU through the
CRS kernels (the default), or through ``local_spmv(which, alpha, x, beta,
y)`` given at construction (``which`` is ``"diag"`` or ``"off"``).

Every rank must call ``spmv`` the same number of times in the same order
(the exchange is a collective).
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


def _split_rows(Rst_l, Col_l, Val_l, r0, r1):
    """The local rows split by column: (diagonal CRS with columns - r0,
    off-diagonal CRS with global columns).  Row order and the order of the
    entries inside a row are kept."""
    nrows = len(Rst_l) - 1
    own = (Col_l >= r0) & (Col_l < r1)
    row_of = np.repeat(np.arange(nrows, dtype=np.int64), np.diff(Rst_l))
    d_cnt = np.bincount(row_of[own], minlength=nrows)
    o_cnt = np.bincount(row_of[~own], minlength=nrows)
    d_Rst = np.concatenate([[0], np.cumsum(d_cnt)]).astype(np.int32)
    o_Rst = np.concatenate([[0], np.cumsum(o_cnt)]).astype(np.int32)
    return ((d_Rst, (Col_l[own] - r0).astype(np.int32), Val_l[own]),
            (o_Rst, Col_l[~own].astype(np.int64), Val_l[~own]))


class RowShardedCRS:
    """This rank's rows of a square CRS matrix (host arrays of the whole
    matrix, or at least its row pointer and this rank's rows)."""

    def __init__(self, m: int, n: int, Rst, Col, Val, rank: int | None = None, world: int | None = None,
                 device="cuda", dtype=torch.float64, local_spmv=None, group=None, exchange: str = "halo",
                 overlap: bool = True):
        if m != n:
            raise ValueError("RowShardedCRS: the matrix must be square (x and y share the row ranges)")
        if exchange not in ("halo", "allgather"):
            raise ValueError("RowShardedCRS: exchange must be 'halo' or 'allgather'")
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else rank
        self.world = dist.get_world_size(group) if world is None else world
        self.m, self.n = m, n
        self.exchange, self.overlap = exchange, overlap
        self.bounds = row_bounds(Rst, self.world)
        self.r0, self.r1 = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
        self.maxlen = max(1, int(np.max(np.diff(self.bounds)))) if self.world else 1
        Rst = np.asarray(Rst, dtype=np.int64)
        k0, k1 = int(Rst[self.r0]), int(Rst[self.r1])
        self.Rst_l = (Rst[self.r0:self.r1 + 1] - k0).astype(np.int32)
        self.Col_l = np.asarray(Col[k0:k1], dtype=np.int32)
        self.Val_l = np.asarray(Val[k0:k1])
        self.device, self.dtype = torch.device(device), dtype
        self._local = local_spmv
        (dR, dC, dV), (oR, oC, oV) = _split_rows(self.Rst_l, self.Col_l, self.Val_l, self.r0, self.r1)
        self.diag = (dR, dC, dV)
        owner = np.searchsorted(self.bounds, oC, side="right") - 1  # rank owning each remote column
        if exchange == "allgather":
            # position of a global column in the padded gathered buffer
            pos = owner * self.maxlen + (oC - self.bounds[owner])
            self.off = (oR, pos.astype(np.int32), oV)
            self.n_ghost = self.world * self.maxlen
            self._pad = torch.zeros(self.maxlen, dtype=dtype, device=self.device)
            self._ghost = torch.zeros(self.n_ghost, dtype=dtype, device=self.device)
        else:
            # the distinct remote columns, ascending (so grouped by owner rank)
            ghosts, inv = np.unique(oC, return_inverse=True)
            self.off = (oR, inv.astype(np.int32), oV)
            self.n_ghost = len(ghosts)
            g_owner = np.searchsorted(self.bounds, ghosts, side="right") - 1
            self.recv_counts = np.bincount(g_owner, minlength=self.world).astype(np.int64)
            # tell every rank which of its entries this rank needs
            # (on the rank's device: NCCL moves device tensors only)
            need = np.concatenate([ghosts[g_owner == k] - self.bounds[k] for k in range(self.world)])
            if self.world > 1:
                counts = torch.as_tensor(self.recv_counts, dtype=torch.int64, device=self.device)
                send_counts = torch.empty_like(counts)
                dist.all_to_all_single(send_counts, counts, group=group)
                self.send_counts = send_counts.cpu().numpy().astype(np.int64)
                send_idx = torch.empty(int(self.send_counts.sum()), dtype=torch.int64, device=self.device)
                dist.all_to_all_single(send_idx, torch.as_tensor(need, dtype=torch.int64, device=self.device),
                                       output_split_sizes=self.send_counts.tolist(),
                                       input_split_sizes=self.recv_counts.tolist(), group=group)
            else:
                self.send_counts = np.zeros(1, np.int64)
                send_idx = torch.empty(0, dtype=torch.int64, device=self.device)
            self._send_idx = send_idx
            self._send = torch.zeros(int(self.send_counts.sum()), dtype=dtype, device=self.device)
            self._ghost = torch.zeros(max(self.n_ghost, 1), dtype=dtype, device=self.device)
        self.exchanged_per_spmv = (int(self.send_counts.sum()) if exchange == "halo"
                                   else self.maxlen * (self.world - 1))
        if local_spmv is None:
            nl = self.r1 - self.r0
            self.A_diag = F.spMtxCRS.from_host(nl, max(nl, 1), dR, dC, dV, dtype=dtype, device=device)
            self.A_off = F.spMtxCRS.from_host(nl, max(self.n_ghost, 1), oR, self.off[1], oV, dtype=dtype,
                                              device=device)

    @property
    def local_rows(self) -> int:
        return self.r1 - self.r0

    def _start_exchange(self, x_local: torch.Tensor):
        """Starts the x exchange; returns the pending work (or None when it
        ran synchronously, or there is nothing to exchange)."""
        if self.world == 1:
            return None
        if self.exchange == "allgather":
            self._pad[:self.local_rows].copy_(x_local)
            return dist.all_gather_into_tensor(self._ghost, self._pad, group=self.group, async_op=self.overlap)
        if self._send.numel():
            torch.index_select(x_local, 0, self._send_idx, out=self._send)
        return dist.all_to_all_single(self._ghost[:self.n_ghost], self._send,
                                      output_split_sizes=self.recv_counts.tolist(),
                                      input_split_sizes=self.send_counts.tolist(), group=self.group,
                                      async_op=self.overlap)

    def gather_x(self, x_local: torch.Tensor) -> torch.Tensor:
        """The ghost values this rank's off-diagonal block reads (after one
        exchange), in its column numbering."""
        if x_local.numel() != self.local_rows:
            raise ValueError("gather_x: x_local must hold this rank's rows of x")
        work = self._start_exchange(x_local)
        if work is not None:
            work.wait()
        return self._ghost[:self.n_ghost]

    def _product(self, which: str, alpha: float, x: torch.Tensor, beta: float, y: torch.Tensor):
        if self._local is not None:
            self._local(which, alpha, x, beta, y)
            return
        A = self.A_diag if which == "diag" else self.A_off
        st = F.sparse_mv(F.SPARSE_OPERATION_NON_TRANSPOSE, alpha, A, F.sparse_matrix_descr(), x, beta, y)
        if st.code != 0:
            raise RuntimeError(f"RowShardedCRS.spmv ({which}): status {st.code}")

    def spmv(self, x_local: torch.Tensor, alpha: float = 1.0, beta: float = 0.0,
             y_local: torch.Tensor | None = None) -> torch.Tensor:
        """y_local = alpha * (A x)[rows of this rank] + beta * y_local."""
        if x_local.numel() != self.local_rows:
            raise ValueError("spmv: x_local must hold this rank's rows of x")
        if y_local is None:
            y_local = torch.zeros(self.local_rows, dtype=self.dtype, device=self.device)
        work = self._start_exchange(x_local)  # in flight during the diagonal product
        if self.local_rows:
            self._product("diag", alpha, x_local, beta, y_local)
        if work is not None:
            work.wait()
        if self.local_rows and self.n_ghost:
            self._product("off", alpha, self._ghost[:self.n_ghost], 1.0, y_local)
        return y_local
