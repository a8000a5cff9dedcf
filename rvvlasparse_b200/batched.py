"""Batched SpMV over many CRS matrices with k right-hand sides, in one
persistent launch (optionally captured in a CUDA graph), through the C ABI
(``rvvla_batched_*``).  No reference counterpart.

X holds every matrix's n_i x k block and Y every m_i x k block, row-major,
packed in matrix order; ``x_off``/``y_off`` give the first element of each.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import check, load
from .formats import _ptr, _stream, spMtxCRS


class SpMVBatch:
    """A plan for Y_i = alpha * A_i X_i + beta * Y_i over ``mats``.

    ``mode``/``param`` choose per matrix CSR (0, threads per row) or
    SELL-C-sigma (1, sigma); ``tune=True`` lets the library's autotuner
    measure the candidates and choose."""

    def __init__(self, mats: list[spMtxCRS], k: int = 1, tune: bool = False, mode=None, param=None):
        if not mats:
            raise ValueError("SpMVBatch: no matrices")
        dt = mats[0].dtype
        if any(m.dtype != dt for m in mats) or dt not in (torch.float64, torch.float32):
            raise ValueError("SpMVBatch: all matrices must share a float32 or float64 value type")
        self.mats, self.k, self.dtype = list(mats), int(k), dt
        self._descs = (_capi.rvvla_crs * len(mats))(*[m.desc() for m in mats])
        lib = load()
        vb = 8 if dt == torch.float64 else 4
        n = len(mats)
        self.mode = np.zeros(n, np.int32) if mode is None else np.ascontiguousarray(mode, np.int32)
        self.param = np.zeros(n, np.int32) if param is None else np.ascontiguousarray(param, np.int32)
        self.tuned_ms = None
        if tune:
            ms = C.c_double(0.0)
            check(lib.rvvla_batched_autotune(self._descs, n, vb, self.k, self.mode.ctypes.data, self.param.ctypes.data,
                                             C.byref(ms), _stream()), "rvvla_batched_autotune")
            self.tuned_ms = ms.value
        self._plan = _capi.rvvla_batch_owned()
        st = lib.rvvla_batched_plan(self._descs, n, vb, self.k, self.mode.ctypes.data, self.param.ctypes.data,
                                    C.byref(self._plan), _stream())
        if st != 0:
            raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(lib.rvvla_last_error().decode())
        self.x_off = np.ctypeslib.as_array(self._plan.x_off, shape=(n + 1,)).copy()
        self.y_off = np.ctypeslib.as_array(self._plan.y_off, shape=(n + 1,)).copy()
        self.x_len, self.y_len = int(self.x_off[-1]), int(self.y_off[-1])
        self.ntiles, self.grid = int(self._plan.h.ntiles), int(self._plan.h.grid)

    def __del__(self):
        try:
            load().rvvla_batched_free(C.byref(self._plan))
        except Exception:
            pass

    def spmv(self, alpha: float, X: torch.Tensor, beta: float, Y: torch.Tensor) -> int:
        if X.numel() < self.x_len or Y.numel() < self.y_len or X.dtype != self.dtype or Y.dtype != self.dtype:
            return _capi.RVVLA_ERR_INVALID_ARG
        lib = load()
        fn = lib.rvvla_batched_spmv_f64 if self.dtype == torch.float64 else lib.rvvla_batched_spmv_f32
        return fn(C.byref(self._plan.h), float(alpha), _ptr(X), float(beta), _ptr(Y), _stream())

    def graph(self, alpha: float, X: torch.Tensor, beta: float, Y: torch.Tensor) -> "BatchGraph":
        """Captures one launch (these alpha, X, beta, Y) into a CUDA graph on
        the current stream, which must not be the legacy default stream."""
        return BatchGraph(self, alpha, X, beta, Y)


class BatchGraph:
    def __init__(self, batch: SpMVBatch, alpha, X, beta, Y):
        self._keep = (batch, X, Y)
        lib = load()
        h = C.c_void_p()
        check(lib.rvvla_batched_graph(C.byref(batch._plan.h), float(alpha), _ptr(X), float(beta), _ptr(Y),
                                      _stream(), C.byref(h)), "rvvla_batched_graph")
        self._h = h

    def launch(self) -> None:
        check(load().rvvla_batched_graph_launch(self._h, _stream()), "rvvla_batched_graph_launch")

    def __del__(self):
        try:
            load().rvvla_batched_graph_free(self._h)
        except Exception:
            pass
