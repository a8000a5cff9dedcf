"""Krylov solvers on the GPU, callers of the CRS path; the reference has no
solver.  ``cg`` (``rvvla_cg_*``) for symmetric positive definite matrices,
``bicgstab`` (``rvvla_bicgstab_*``) for general square ones.

Each iteration runs q = A p with p.q fused into the SpMV (the CRS lane-run
kernel dots every row piece with p as it leaves the kernel), then the x / r
update with the new r.r fused into the same pass; the host reads r.r every
``check_every`` iterations.  ``spmv_dot`` exposes the fused product alone.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi
from . import formats as F


def cg(A: F.spMtxCRS, b: torch.Tensor, x0: torch.Tensor | None = None, rtol: float = 1e-8,
       max_iter: int = 1000, check_every: int = 10):
    """Solves A x = b; returns (x, iterations, ||r|| / ||b||).  A is an
    spMtxCRS (fp64 or fp32, square, symmetric positive definite), b a CUDA
    vector of A's value type."""
    if A.dtype not in (torch.float64, torch.float32):
        raise TypeError("cg: A must hold fp64 or fp32 values")
    if b.dtype != A.dtype or not b.is_cuda or b.numel() != A.m:
        raise ValueError("cg: b must be a CUDA vector of A's type with m entries")
    lib = _capi.load()
    x = torch.zeros_like(b) if x0 is None else x0.detach().clone().contiguous()
    b = b.contiguous()
    code = _capi.RVVLA_F64 if A.dtype == torch.float64 else _capi.RVVLA_F32
    d = A.desc(code)
    it, rr = C.c_int64(0), C.c_double(0.0)
    fn = lib.rvvla_cg_f64 if A.dtype == torch.float64 else lib.rvvla_cg_f32
    st = fn(C.byref(d), b.data_ptr(), x.data_ptr(), int(max_iter), float(rtol), int(check_every), C.byref(it),
            C.byref(rr), torch.cuda.current_stream().cuda_stream)
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(msg)
    return x, it.value, rr.value


def bicgstab(A: F.spMtxCRS, b: torch.Tensor, x0: torch.Tensor | None = None, rtol: float = 1e-8,
             max_iter: int = 1000, check_every: int = 10):
    """Solves A x = b by BiCGStab (unpreconditioned); returns (x,
    iterations, ||r|| / ||b||, breakdown).  A is an spMtxCRS (fp64 or fp32,
    square), b a CUDA vector of A's value type.  breakdown is True when the
    iteration stopped unconverged on an exactly zero r^.r, r^.v or t.t."""
    if A.dtype not in (torch.float64, torch.float32):
        raise TypeError("bicgstab: A must hold fp64 or fp32 values")
    if b.dtype != A.dtype or not b.is_cuda or b.numel() != A.m:
        raise ValueError("bicgstab: b must be a CUDA vector of A's type with m entries")
    lib = _capi.load()
    x = torch.zeros_like(b) if x0 is None else x0.detach().clone().contiguous()
    b = b.contiguous()
    code = _capi.RVVLA_F64 if A.dtype == torch.float64 else _capi.RVVLA_F32
    d = A.desc(code)
    it, rr, bd = C.c_int64(0), C.c_double(0.0), C.c_int(0)
    fn = lib.rvvla_bicgstab_f64 if A.dtype == torch.float64 else lib.rvvla_bicgstab_f32
    st = fn(C.byref(d), b.data_ptr(), x.data_ptr(), int(max_iter), float(rtol), int(check_every), C.byref(it),
            C.byref(rr), C.byref(bd), torch.cuda.current_stream().cuda_stream)
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(msg)
    return x, it.value, rr.value, bool(bd.value)


def spmv_dot(A: F.spMtxCRS, x: torch.Tensor):
    """(y, d) with y = A x and d = x^T A x (a one-element CUDA tensor), in one
    pass over A (square, fp64 or fp32)."""
    if x.dtype != A.dtype or not x.is_cuda or x.numel() != A.n:
        raise ValueError("spmv_dot: x must be a CUDA vector of A's type with n entries")
    lib = _capi.load()
    code = _capi.RVVLA_F64 if A.dtype == torch.float64 else _capi.RVVLA_F32
    d = A.desc(code)
    y = torch.empty(A.m, dtype=A.dtype, device=x.device)
    dot = torch.empty(1, dtype=A.dtype, device=x.device)
    fn = lib.rvvla_crs_spmv_dot_f64 if A.dtype == torch.float64 else lib.rvvla_crs_spmv_dot_f32
    st = fn(C.byref(d), x.contiguous().data_ptr(), y.data_ptr(), dot.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(msg)
    return y, dot
