"""torch.autograd binding of the adjoint kernels (a thin test binding).

``spmv(pattern, values, x, alpha)`` computes y = alpha * A(values) @ x for a
CRS sparsity pattern fixed in a :class:`CrsPattern`; its backward runs the
library's adjoint kernels through the C ABI:

* dx = alpha * A^T g — ``rvvla_spmv_adjoint_x_values_*`` on the transposed
  CRS built once per pattern by ``rvvla_csr_transpose``, reading the current
  ``values`` through the stored permutation inside the kernel
  (``adjoint_x_refreshed`` goes through ``rvvla_csr_transpose_values`` and
  ``rvvla_spmv_adjoint_x_*`` instead);
* dvalues[k] = alpha * g[row(k)] * x[Col[k]] — ``rvvla_sddmm_values_*``.

The reference has no adjoint (it declares SPARSE_OPERATION_TRANSPOSE in
include/types.h:24-27 and ignores it).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi
from ._capi import check, load
from .formats import _ptr, _stream, spMtxCRS


class CrsPattern:
    """Sparsity pattern of an m x n CRS matrix on the GPU, with its transpose."""

    def __init__(self, m: int, n: int, Rst: torch.Tensor, Col: torch.Tensor, dtype: torch.dtype):
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("CrsPattern: dtype must be float64 or float32")
        self.m, self.n, self.nz = int(m), int(n), int(Col.numel())
        self.dtype = dtype
        self.Rst, self.Col = Rst, Col
        self._crs = spMtxCRS(self.m, self.n, self.nz, Rst, Col, None)
        self._code = _capi.RVVLA_F64 if dtype == torch.float64 else _capi.RVVLA_F32
        self._tr = _capi.rvvla_transpose_owned()
        lib = load()
        d = _capi.rvvla_crs(self.m, self.n, self.nz, _ptr(Rst), _ptr(Col), None, None, 0, 0)
        vb = 8 if dtype == torch.float64 else 4
        st = lib.rvvla_csr_transpose(C.byref(d), vb, C.byref(self._tr), _stream())
        if st != 0:
            raise RuntimeError(lib.rvvla_last_error().decode())

    def __del__(self):
        try:
            load().rvvla_csr_transpose_free(C.byref(self._tr))
        except Exception:
            pass

    def desc(self, values: torch.Tensor) -> _capi.rvvla_crs:
        d = self._crs.desc(self._code)
        d.Val = _ptr(values)
        return d

    def transposed(self) -> dict:
        """A^T's arrays (copied to torch tensors): Rst, Col, perm, Val."""
        from .formats import _owned_to_tensor

        dev = self.Rst.device
        return {"Rst": _owned_to_tensor(self._tr.Rst, self.n + 1, torch.int32, dev),
                "Col": _owned_to_tensor(self._tr.Col, self.nz, torch.int32, dev),
                "perm": _owned_to_tensor(self._tr.perm, self.nz, torch.int32, dev),
                "Val": _owned_to_tensor(self._tr.Val, self.nz, self.dtype, dev)}

    # ---- the three products, on the current stream
    def forward(self, values: torch.Tensor, x: torch.Tensor, alpha: float) -> torch.Tensor:
        lib = load()
        y = torch.empty(self.m, dtype=self.dtype, device=x.device)
        fn = lib.rvvla_crs_spmv_f64 if self.dtype == torch.float64 else lib.rvvla_crs_spmv_f32
        check(fn(C.byref(self.desc(values)), float(alpha), _ptr(x), 0.0, _ptr(y), _stream()), "crs_spmv")
        return y

    def adjoint_x(self, values: torch.Tensor, g: torch.Tensor, alpha: float) -> torch.Tensor:
        """dx = alpha * A(values)^T g; the values are read through the
        transpose's permutation inside the kernel."""
        lib = load()
        dx = torch.empty(self.n, dtype=self.dtype, device=g.device)
        fn = (lib.rvvla_spmv_adjoint_x_values_f64 if self.dtype == torch.float64
              else lib.rvvla_spmv_adjoint_x_values_f32)
        check(fn(C.byref(self._tr.h), _ptr(values), float(alpha), _ptr(g), 0.0, _ptr(dx), _stream()),
              "spmv_adjoint_x_values")
        return dx

    def adjoint_x_refreshed(self, values: torch.Tensor, g: torch.Tensor, alpha: float) -> torch.Tensor:
        """The same product through rvvla_csr_transpose_values (A^T's own
        value array re-gathered first) and rvvla_spmv_adjoint_x."""
        lib = load()
        check(lib.rvvla_csr_transpose_values(C.byref(self._tr.h), _ptr(values), self._tr.Val, _stream()),
              "csr_transpose_values")
        dx = torch.empty(self.n, dtype=self.dtype, device=g.device)
        fn = lib.rvvla_spmv_adjoint_x_f64 if self.dtype == torch.float64 else lib.rvvla_spmv_adjoint_x_f32
        check(fn(C.byref(self._tr.h), float(alpha), _ptr(g), 0.0, _ptr(dx), _stream()), "spmv_adjoint_x")
        return dx

    def sddmm(self, g: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
        lib = load()
        dv = torch.empty(self.nz, dtype=self.dtype, device=g.device)
        fn = lib.rvvla_sddmm_values_f64 if self.dtype == torch.float64 else lib.rvvla_sddmm_values_f32
        check(fn(C.byref(self._crs.desc()), _ptr(g), _ptr(x), _ptr(dv), _stream()), "sddmm_values")
        return dv


class SpMVFunction(torch.autograd.Function):
    """y = alpha * A(values) @ x with the pattern held by a CrsPattern."""

    @staticmethod
    def forward(ctx, values, x, pattern: CrsPattern, alpha: float = 1.0):
        values = values.contiguous()
        x = x.contiguous()
        ctx.save_for_backward(values, x)
        ctx.pattern, ctx.alpha = pattern, float(alpha)
        return pattern.forward(values, x, alpha)

    @staticmethod
    def backward(ctx, g):
        values, x = ctx.saved_tensors
        p, alpha = ctx.pattern, ctx.alpha
        g = g.contiguous()
        dvalues = dx = None
        if ctx.needs_input_grad[0]:
            gs = g if alpha == 1.0 else g * alpha
            dvalues = p.sddmm(gs, x)
        if ctx.needs_input_grad[1]:
            dx = p.adjoint_x(values, g, alpha)
        return dvalues, dx, None, None


def spmv(pattern: CrsPattern, values: torch.Tensor, x: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
    return SpMVFunction.apply(values, x, pattern, alpha)
