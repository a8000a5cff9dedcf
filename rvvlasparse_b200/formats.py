"""Python mirror of RVVLASparse's SpMV API over the C ABI (GPU only).

Names, fields and argument meaning follow the reference:

* ``sparse_mv(op, alpha, mat, descr, b, beta, y, stage=ALL)`` mirrors
  ``sparse_mv<T, Mtx, simd, stage>`` (include/spmv_mtx.h:21-29) and returns a
  ``sparse_matrix_status`` whose ``code`` is 0 on success (the C-ABI status
  otherwise);
* ``convert(dist, src, params)`` mirrors ``convert<T, MtxDist, simd>``
  (include/convert.h:30-31) and raises like the reference's HCSR builder
  (ValueError for std::invalid_argument, OverflowError for std::length_error,
  RuntimeError for std::logic_error);
* the ``spMtx*`` classes carry the reference classes' public fields, with the
  arrays as CUDA tensors.

Vectors ``b`` and ``y`` are CUDA tensors of the matrix's value type (fp32
for the mixed-precision forms).  Host numpy vectors are accepted too: they are
copied to the device and ``y`` is copied back (the end-to-end path).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum

import numpy as np
import torch

from . import _capi
from ._capi import check, load

# ------------------------------------------------------------------ types.h


class sparse_operation_t(IntEnum):
    SPARSE_OPERATION_NON_TRANSPOSE = 0
    SPARSE_OPERATION_TRANSPOSE = 1


class sparse_matrix_mv_stage(IntEnum):
    SPARSE_MATRIX_MV_PREPARATION = 0
    SPARSE_MATRIX_MV_MULT = 1
    SPARSE_MATRIX_MV_GET_RESULTS = 2
    SPARSE_MATRIX_MV_ALL_STAGES = 3


SPARSE_OPERATION_NON_TRANSPOSE = sparse_operation_t.SPARSE_OPERATION_NON_TRANSPOSE
SPARSE_OPERATION_TRANSPOSE = sparse_operation_t.SPARSE_OPERATION_TRANSPOSE
SPARSE_MATRIX_MV_PREPARATION = sparse_matrix_mv_stage.SPARSE_MATRIX_MV_PREPARATION
SPARSE_MATRIX_MV_MULT = sparse_matrix_mv_stage.SPARSE_MATRIX_MV_MULT
SPARSE_MATRIX_MV_GET_RESULTS = sparse_matrix_mv_stage.SPARSE_MATRIX_MV_GET_RESULTS
SPARSE_MATRIX_MV_ALL_STAGES = sparse_matrix_mv_stage.SPARSE_MATRIX_MV_ALL_STAGES


@dataclass
class sparse_matrix_status:
    code: int = 0


@dataclass
class sparse_matrix_descr:
    pass


@dataclass
class convertParams:
    """``convertParams{std::map<string, convertValue>}`` (include/convert.h:21-28)."""
    param: dict = field(default_factory=dict)

    def __init__(self, param: dict | None = None, **kw):
        self.param = dict(param or {})
        self.param.update(kw)


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _dtype_code(t: torch.dtype) -> int:
    return {torch.float64: _capi.RVVLA_F64, torch.float32: _capi.RVVLA_F32,
            torch.bfloat16: _capi.RVVLA_BF16}[t]


# ------------------------------------------------------------------ CRS


class spMtxCRS:
    """``spMtxCRS<ValT>`` (include/CRS.h:10-20): m, n, nz, Rst[m+1], Col[nz], Val[nz]."""

    def __init__(self, m: int = 0, n: int = 0, nz: int = 0, Rst=None, Col=None, Val=None):
        self.m, self.n, self.nz = int(m), int(n), int(nz)
        self.Rst, self.Col, self.Val = Rst, Col, Val
        self._plans: dict[int, torch.Tensor] = {}

    @classmethod
    def from_host(cls, m, n, Rst, Col, Val, dtype=torch.float64, device="cuda"):
        Rst = torch.as_tensor(np.ascontiguousarray(Rst, dtype=np.int32)).to(device)
        Col = torch.as_tensor(np.ascontiguousarray(Col, dtype=np.int32)).to(device)
        Val = torch.as_tensor(np.ascontiguousarray(Val)).to(device=device, dtype=dtype)
        return cls(m, n, int(Col.numel()), Rst, Col, Val)

    @property
    def dtype(self) -> torch.dtype:
        return self.Val.dtype

    def astype(self, dtype: torch.dtype) -> "spMtxCRS":
        return spMtxCRS(self.m, self.n, self.nz, self.Rst, self.Col, self.Val.to(dtype))

    def desc(self, plan_dtype: int | None = None) -> _capi.rvvla_crs:
        d = _capi.rvvla_crs(self.m, self.n, self.nz, _ptr(self.Rst), _ptr(self.Col), _ptr(self.Val), None, 0, 0)
        if plan_dtype is not None and self.m > 0:
            plan, tiles, kind = self.plan(plan_dtype)
            d.plan = plan.data_ptr()
            d.plan_tiles = tiles
            d.plan_kind = kind
        return d

    def plan(self, dtype_code: int):
        """Row-structure analysis (rvvla_crs_analyze), cached per value type:
        (plan tensor, plan_tiles, plan_kind)."""
        key = _capi.RVVLA_F64 if dtype_code == _capi.RVVLA_F64 else _capi.RVVLA_F32
        if key not in self._plans:
            lib = load()
            n = lib.rvvla_crs_plan_len(self.m, self.nz, key)
            plan = torch.empty(max(int(n), 1), dtype=torch.int32, device=self.Rst.device)
            d = _capi.rvvla_crs(self.m, self.n, self.nz, _ptr(self.Rst), _ptr(self.Col), _ptr(self.Val), None, 0, 0)
            tiles, kind = C.c_int64(0), C.c_int32(0)
            check(lib.rvvla_crs_analyze(C.byref(d), key, plan.data_ptr(), C.byref(tiles), C.byref(kind), _stream()),
                  "rvvla_crs_analyze")
            self._plans[key] = (plan, tiles.value, kind.value)
        return self._plans[key]


# ------------------------------------------------------------------ HCSR


class spMtxHCSR:
    """``spMtxHCSR<ValT>`` (include/HCSR.h:39-53)."""

    def __init__(self):
        self.R = self.C = self.m = self.n = self.nz = self.b_m = self.b_n = 0
        self.block_ptr = self.row_offset = self.row_ptr = self.col_idx = self.values = None

    def desc(self) -> _capi.rvvla_hcsr:
        return _capi.rvvla_hcsr(self.R, self.C, self.m, self.n, self.nz, self.b_m, self.b_n,
                                _ptr(self.block_ptr), _ptr(self.row_offset), _ptr(self.row_ptr),
                                _ptr(self.col_idx), _ptr(self.values),
                                0 if self.row_ptr is None else self.row_ptr.numel())

    @property
    def dtype(self) -> torch.dtype:
        return self.values.dtype

    def astype(self, dtype: torch.dtype) -> "spMtxHCSR":
        h = spMtxHCSR()
        h.__dict__.update(self.__dict__)
        h.values = self.values.to(dtype)
        return h

    def to_host(self) -> dict:
        out = {k: getattr(self, k) for k in ("R", "C", "m", "n", "nz", "b_m", "b_n")}
        for k in ("block_ptr", "row_offset", "row_ptr", "col_idx", "values"):
            out[k] = getattr(self, k).cpu().numpy()
        return out


def _owned_to_tensor(ptr: int, n: int, dtype: torch.dtype, device) -> torch.Tensor:
    """Copy a library-owned device array into a torch tensor."""
    t = torch.empty(max(n, 0), dtype=dtype, device=device)
    if n > 0:
        check(load().rvvla_memcpy(t.data_ptr(), ptr, n * t.element_size(), _stream()), "rvvla_memcpy")
    return t


def _hcsr_convert(dist: spMtxHCSR, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    if src.dtype == torch.float64:
        R, Cc = 2000, 2000  # convert<double, spMtxHCSR, false> defaults (crs_to_hcsr.cpp:140-142)
    else:
        R, Cc = 4000, 4000  # convert<float, spMtxHCSR, false> defaults (crs_to_hcsr.cpp:157-159)
    p = 2.0
    if "R" in params.param:
        R = int(params.param["R"])
    if "C" in params.param:
        Cc = int(params.param["C"])
    if "p" in params.param:
        p = float(params.param["p"])
    if R <= 0 or Cc <= 0:
        raise ValueError("crs_to_HCSR: R and C must be positive")
    owned = _capi.rvvla_hcsr_owned()
    d = src.desc()
    st = lib.rvvla_hcsr_build(C.byref(d), src.Val.element_size(), R, Cc, p, C.byref(owned), _stream())
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        if st == _capi.RVVLA_ERR_INVALID_ARG:
            raise ValueError(msg)
        if st == _capi.RVVLA_ERR_TOO_LARGE:
            raise OverflowError(msg)
        raise RuntimeError(msg)
    try:
        h = owned.h
        dev = src.Val.device
        dist.R, dist.C, dist.m, dist.n, dist.nz, dist.b_m, dist.b_n = h.R, h.C, h.m, h.n, h.nz, h.b_m, h.b_n
        nb1 = h.b_m * h.b_n + 1
        dist.block_ptr = _owned_to_tensor(owned.block_ptr, nb1, torch.int32, dev)
        dist.row_offset = _owned_to_tensor(owned.row_offset, nb1, torch.int32, dev)
        dist.row_ptr = _owned_to_tensor(owned.row_ptr, h.row_ptr_len, torch.int32, dev)
        dist.col_idx = _owned_to_tensor(owned.col_idx, h.nz, torch.int16, dev)
        dist.values = _owned_to_tensor(owned.values, h.nz, src.Val.dtype, dev)
    finally:
        lib.rvvla_hcsr_free(C.byref(owned))


# ------------------------------------------------------------------ generic


class _GpuFormat:
    """Mirror of a reference format class: scalar fields + CUDA arrays.
    Subclasses list SCALARS, ARRAYS (name -> torch dtype, None = value type),
    the ctypes descriptor type and the value array's name."""

    SCALARS: tuple = ()
    ARRAYS: dict = {}
    CDESC = None
    VALUE = ""

    def __init__(self):
        for k in self.SCALARS:
            setattr(self, k, 0)
        for k in self.ARRAYS:
            setattr(self, k, None)

    @property
    def dtype(self) -> torch.dtype:
        return getattr(self, self.VALUE).dtype

    def astype(self, dtype: torch.dtype):
        c = type(self)()
        c.__dict__.update(self.__dict__)
        setattr(c, self.VALUE, getattr(self, self.VALUE).to(dtype))
        return c

    def desc(self):
        d = self.CDESC()
        for k in self.SCALARS:
            if hasattr(d, k):
                setattr(d, k, int(getattr(self, k)))
        for k in self.ARRAYS:
            if hasattr(d, k):
                setattr(d, k, _ptr(getattr(self, k)))
        return d

    def to_host(self) -> dict:
        out = {k: int(getattr(self, k)) for k in self.SCALARS}
        for k in self.ARRAYS:
            a = getattr(self, k)
            if a is not None:
                out[k] = a.cpu().numpy()
        return out

    def _adopt(self, owned, sizes: dict, value_dtype, device) -> None:
        h = owned.h
        for k in self.SCALARS:
            if hasattr(h, k):
                setattr(self, k, int(getattr(h, k)))
        for k, n in sizes.items():
            dt = self.ARRAYS[k] or value_dtype
            setattr(self, k, _owned_to_tensor(getattr(owned, k), int(n), dt, device))


def _build(lib_fn, free_fn, owned, *args):
    st = lib_fn(*args, C.byref(owned), _stream())
    if st != 0:
        msg = load().rvvla_last_error().decode()
        raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(msg)


class spMtxSELL_C_Sigma(_GpuFormat):
    """``spMtxSELL_C_Sigma<ValT>`` (include/SELL_C_Sigma.h:23-40)."""

    SCALARS = ("m", "n", "cnt_b", "nz", "C", "Sigma", "len")
    ARRAYS = {"vCl": torch.int32, "vCs": torch.int32, "vBs": torch.int32, "vSBs": torch.int32,
              "vCol": torch.int32, "vPerm": torch.int32, "vVal": None}
    CDESC = _capi.rvvla_sell
    VALUE = "vVal"


def _sell_convert(dist, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    owned = _capi.rvvla_sell_owned()
    Cc = int(params.param.get("C", 32))
    sigma = int(params.param.get("sigma", params.param.get("Sigma", 256)))
    _build(lib.rvvla_sell_build, lib.rvvla_sell_free, owned, C.byref(src.desc()), src.Val.element_size(), Cc, sigma)
    try:
        h = owned.h
        sizes = {"vCl": h.cnt_b, "vCs": h.cnt_b, "vBs": h.cnt_b, "vSBs": h.cnt_b, "vCol": h.len, "vPerm": h.m,
                 "vVal": h.len}
        dist._adopt(owned, sizes, src.Val.dtype, src.Val.device)
    finally:
        lib.rvvla_sell_free(C.byref(owned))


class spMtxVNEC(_GpuFormat):
    """``spMtxVNEC<ValT>`` (include/VNEC.h:35-76).  Unlike the reference (which
    keeps a pointer to the source CRS), the source arrays are copied in."""

    SCALARS = ("m", "n", "nz", "NUM_THREADS_VNEC", "nLanes", "vnec_t", "max_nec", "ngroups", "ntasks", "nreorder",
               "plan_tiles", "plan_kind")
    ARRAYS = {k: (None if k in ("val", "val_align", "reorder_nnz") else torch.int32) for k in _capi.VNEC_ARRAYS}
    CDESC = _capi.rvvla_vnec
    VALUE = "val"

    def astype(self, dtype):
        c = super().astype(dtype)
        for k in ("val_align", "reorder_nnz"):
            if getattr(self, k) is not None:
                setattr(c, k, getattr(self, k).to(dtype))
        return c


def _vnec_convert(dist, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    owned = _capi.rvvla_vnec_owned()
    nt = int(params.param.get("NUM_THREADS_VNEC", params.param.get("threads", 0)))
    variant = int(params.param.get("variant", -1))
    _build(lib.rvvla_vnec_build, lib.rvvla_vnec_free, owned, C.byref(src.desc()), src.Val.element_size(), nt, variant)
    try:
        h = owned.h
        NT = h.NUM_THREADS_VNEC
        sizes = {"ptr": h.m + 1, "indices": h.nz, "val": h.nz, "thread_coord_start": 2 * NT,
                 "thread_coord_end": 2 * NT}
        if h.vnec_t == 0:
            sizes.update({"ecr_indices": h.nz, "NEC_NUM": NT, "use_x_ptr": NT + 1, "v_row_ptr": h.m + 1,
                          "col_start": h.ngroups, "val_align": h.ngroups * h.nLanes})
        elif h.vnec_t == 1:
            sizes.update({"NEC_NUM": NT, "use_x_ptr": NT + 1, "tasks": h.ntasks, "task_start": NT, "task_end": NT,
                          "spvv_len": NT, "row_begin": h.ntasks, "row_end": h.ntasks, "reorder_col": h.nreorder,
                          "reorder_nnz": h.nreorder})
        if owned.plan:  # L variant: the analysed plan of the source CRS
            sizes["plan"] = lib.rvvla_crs_plan_len(h.m, h.nz, _capi.RVVLA_F64 if src.dtype == torch.float64
                                                    else _capi.RVVLA_F32)
        if h.vnec_t in (0, 1):
            # use_x_indices length = use_x_ptr[NT]: read it back
            tmp = _owned_to_tensor(owned.use_x_ptr, NT + 1, torch.int32, src.Val.device)
            sizes["use_x_indices"] = int(tmp[-1].item())
        dist._adopt(owned, sizes, src.Val.dtype, src.Val.device)
        dist.IRD_mat = float(h.IRD_mat)
    finally:
        lib.rvvla_vnec_free(C.byref(owned))


class spMtxLAV(_GpuFormat):
    """``spMtxLAV<ValT>`` (include/LAV.h:11-31); ``sparse_part`` is an
    :class:`spMtxCRS` on the same device."""

    SCALARS = ("SIMD_Lanes", "m", "n", "nz", "segment_count", "chunk_count", "segment_len", "n_steps",
               "long_chunks")
    ARRAYS = {"chunk_offsets": torch.int32, "chunk_offsets_full_mask": torch.int32, "segment_ptr": torch.int64,
              "out_order": torch.int32, "mask": torch.int16, "val": None, "col_id": torch.int32,
              "row_order": torch.int32, "lane_of_slot": torch.uint8}
    CDESC = _capi.rvvla_lav
    VALUE = "val"

    def __init__(self):
        super().__init__()
        self.T = 0.2
        self.sparse_part = None

    def astype(self, dtype: torch.dtype):
        c = super().astype(dtype)
        c.sparse_part = self.sparse_part.astype(dtype)
        return c

    def desc(self):
        d = super().desc()
        d.T = float(self.T)
        d.sparse_part = self.sparse_part.desc(
            _capi.RVVLA_F64 if self.sparse_part.dtype == torch.float64 else _capi.RVVLA_F32)
        return d

    def to_host(self) -> dict:
        out = super().to_host()
        out["T"] = float(self.T)
        out["mask"] = out["mask"].view(np.uint16)
        out["segment_ptr"] = out["segment_ptr"].view(np.uint64)
        sp = self.sparse_part
        out.update(sparse_nz=sp.nz, sp_Rst=sp.Rst.cpu().numpy(), sp_Col=sp.Col.cpu().numpy(),
                   sp_Val=sp.Val.cpu().numpy())
        return out


def _lav_convert(dist, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    owned = _capi.rvvla_lav_owned()
    lanes = int(params.param.get("SIMD_Lanes", 8))
    T = float(params.param.get("T", 0.2))
    seglen = int(params.param.get("segment_len", 40000))
    _build(lib.rvvla_lav_build, lib.rvvla_lav_free, owned, C.byref(src.desc()), src.Val.element_size(), lanes, T,
           seglen)
    try:
        h = owned.h
        L, cc, ns = h.SIMD_Lanes, h.chunk_count, h.segment_count
        sizes = {"chunk_offsets": (cc + 1) * ns, "chunk_offsets_full_mask": cc * ns, "segment_ptr": ns + 1,
                 "out_order": ns * cc * L, "mask": h.n_steps, "val": h.n_steps * L, "col_id": h.n_steps * L,
                 "row_order": h.m}
        if owned.lane_of_slot:  # derived slot -> lane map (SIMD_Lanes <= 256)
            sizes["lane_of_slot"] = ns * cc * L
        dist._adopt(owned, sizes, src.Val.dtype, src.Val.device)
        dist.T = float(h.T)
        dev = src.Val.device
        snz = int(h.sparse_part.nz)
        dist.sparse_part = spMtxCRS(h.m, h.n, snz, _owned_to_tensor(owned.sp_Rst, h.m + 1, torch.int32, dev),
                                    _owned_to_tensor(owned.sp_Col, snz, torch.int32, dev),
                                    _owned_to_tensor(owned.sp_Val, snz, src.Val.dtype, dev))
    finally:
        lib.rvvla_lav_free(C.byref(owned))


class spMtxVHCC(_GpuFormat):
    """``spMtxVHCC<ValT>`` (include/VHCC.h:43-62): the underscore fields of
    the reference without the underscore, vhcc_params flattened.

    ``num_panels`` > 1 (vhcc_params, include/VHCC.h:15-26; the reference
    stores it, but its only kernel, vhcc_spmv_1panel_riscv in
    src/rvv/spmv_vhcc.cpp:73, runs one panel): the columns are cut into
    contiguous ranges of about nz / num_panels nonzeros, ``panels`` holds one
    single-panel spMtxVHCC per non-empty range (global column indices kept),
    and a product runs them in order — β on the first, 1 after — so row i
    sums its panels' partial sums in column-range order.  The object itself
    then holds only the scalars."""

    SCALARS = ("num_rows", "num_cols", "num_entries", "num_vectors", "pad_entries", "pad_rows", "num_threads",
               "num_panels", "tile_row", "tile_col", "vec_size", "n_masks", "n_eor", "scan_mask_bytes", "n_rowarr")
    ARRAYS = {"thr_info": torch.int32, "veceor_ptr": torch.int32, "scan_mask": torch.uint8, "row_arr": torch.int32,
              "col_arr": torch.int32, "vals_arr": None}
    CDESC = _capi.rvvla_vhcc
    VALUE = "vals_arr"

    def __init__(self):
        super().__init__()
        self.panels: list[spMtxVHCC] = []

    @property
    def dtype(self) -> torch.dtype:
        return self.panels[0].dtype if self.panels else super().dtype

    def astype(self, dtype: torch.dtype):
        if not self.panels:
            return super().astype(dtype)
        c = type(self)()
        c.__dict__.update(self.__dict__)
        c.panels = [p.astype(dtype) for p in self.panels]
        return c

    def desc(self):
        if self.panels:
            raise ValueError("spMtxVHCC: a multi-panel matrix has one descriptor per panel (.panels[k].desc())")
        return super().desc()

    def to_host(self) -> dict:
        if not self.panels:
            return super().to_host()
        out = {k: int(getattr(self, k)) for k in self.SCALARS}
        out["panels"] = [p.to_host() for p in self.panels]
        return out


def column_panels(src: spMtxCRS, num_panels: int) -> list[tuple[int, int, spMtxCRS]]:
    """Cuts ``src`` by columns into ``num_panels`` contiguous ranges [c0, c1)
    holding about nz / num_panels nonzeros each (whole columns, so a range
    may hold more, or nothing), as (c0, c1, CRS of the same shape with only
    that range's nonzeros, global column indices, row-major order kept).
    Torch operations on the arrays' own device; the multi-panel VHCC
    builder's split."""
    P = int(num_panels)
    if P < 1:
        raise ValueError("column_panels: num_panels must be >= 1")
    m, n, nz = src.m, src.n, src.nz
    dev = src.Col.device
    col = src.Col[:nz].long()
    prefix = torch.zeros(n + 1, dtype=torch.int64, device=dev)  # nonzeros in columns < c
    if nz:
        prefix[1:] = torch.cumsum(torch.bincount(col, minlength=n)[:n], 0)
    targets = (torch.arange(1, P, dtype=torch.int64, device=dev) * nz) // P
    inner = torch.searchsorted(prefix, targets, side="left").clamp(0, n)
    bounds = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), inner,
                        torch.full((1,), n, dtype=torch.int64, device=dev)])
    bounds = torch.cummax(bounds, 0).values.tolist()
    row_of = torch.repeat_interleave(torch.arange(m, device=dev), torch.diff(src.Rst.long()), output_size=nz)
    out = []
    for k in range(P):
        c0, c1 = int(bounds[k]), int(bounds[k + 1])
        keep = (col >= c0) & (col < c1)
        cnt = torch.bincount(row_of[keep], minlength=m)[:m]
        Rst = torch.zeros(m + 1, dtype=torch.int32, device=dev)
        Rst[1:] = torch.cumsum(cnt, 0).to(torch.int32)
        Col, Val = src.Col[:nz][keep].contiguous(), src.Val[:nz][keep].contiguous()
        out.append((c0, c1, spMtxCRS(m, n, int(Col.numel()), Rst, Col, Val)))
    return out


def _vhcc_convert(dist, src: spMtxCRS, params: convertParams) -> None:
    P = int(params.param.get("num_panels", 1))
    if P < 1:
        raise ValueError("convert<spMtxVHCC>: num_panels must be >= 1")
    if P > 1 and src.nz > 0:
        one = convertParams({k: v for k, v in params.param.items() if k != "num_panels"})
        parts = []
        for _, _, sub in column_panels(src, P):
            if sub.nz:
                parts.append(spMtxVHCC())
                _vhcc_convert(parts[-1], sub, one)
        head = parts[0]
        for k in spMtxVHCC.SCALARS:
            setattr(dist, k, getattr(head, k))
        for k in spMtxVHCC.ARRAYS:
            setattr(dist, k, None)
        dist.num_panels = len(parts)
        dist.num_entries = src.nz
        for k in ("num_vectors", "pad_entries", "n_eor", "scan_mask_bytes", "n_rowarr", "num_threads"):
            setattr(dist, k, sum(int(getattr(q, k)) for q in parts))
        dist.pad_rows = max(int(q.pad_rows) for q in parts)
        dist.panels = parts
        return
    dist.panels = []
    lib = load()
    owned = _capi.rvvla_vhcc_owned()
    nt = int(params.param.get("num_threads", 0))
    _build(lib.rvvla_vhcc_build, lib.rvvla_vhcc_free, owned, C.byref(src.desc()), src.Val.element_size(), nt)
    try:
        h = owned.h
        sizes = {"thr_info": h.num_threads * 10, "veceor_ptr": h.n_eor, "scan_mask": h.scan_mask_bytes,
                 "row_arr": h.n_rowarr, "col_arr": h.num_vectors * h.vec_size, "vals_arr": h.num_vectors * h.vec_size}
        dist._adopt(owned, sizes, src.Val.dtype, src.Val.device)
    finally:
        lib.rvvla_vhcc_free(C.byref(owned))


class spMtxCVR(_GpuFormat):
    """``spMtxCVR<ValT>`` (include/CVR.h:22-37)."""

    SCALARS = ("nItems", "numRows", "numCols", "SIMD_LEN", "Nthreads", "Nthreads_avail", "no_empty_rows",
               "n_record", "n_writeback")
    ARRAYS = {"vPack_vec_vals": None, "vPack_vec_cols": torch.int32, "vPack_vec_record": torch.int32,
              "writeback_pos_record": torch.int32}
    CDESC = _capi.rvvla_cvr
    VALUE = "vPack_vec_vals"


def _cvr_convert(dist, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    owned = _capi.rvvla_cvr_owned()
    nt = int(params.param.get("Nthreads", 0))
    _build(lib.rvvla_cvr_build, lib.rvvla_cvr_free, owned, C.byref(src.desc()), src.Val.element_size(), nt)
    try:
        h = owned.h
        sizes = {"vPack_vec_vals": h.nItems, "vPack_vec_cols": h.nItems, "vPack_vec_record": h.n_record,
                 "writeback_pos_record": h.n_writeback}
        dist._adopt(owned, sizes, src.Val.dtype, src.Val.device)
    finally:
        lib.rvvla_cvr_free(C.byref(owned))


# ------------------------------------------------------------------ CSR5


class spMtxCSR5:
    """``spMtxCSR5<ValT>`` (include/CSR5.h:57-88): the underscore fields of the
    reference without the underscore, arrays on the GPU."""

    SCALARS = ("m", "n", "nnz", "bit_y_offset", "bit_seg_offset", "tile_desc_len", "tail_tile_start", "p",
               "omega", "sigma", "num_offsets", "no_empty_rows")
    ARRAYS = ("csr_row_pointer", "csr_column_index", "csr_value", "tile_pointer", "tile_descriptor",
              "tile_empty_offset_pointer", "tile_empty_offset")

    def __init__(self):
        for k in self.SCALARS:
            setattr(self, k, 0)
        for k in self.ARRAYS:
            setattr(self, k, None)

    @property
    def dtype(self) -> torch.dtype:
        return self.csr_value.dtype

    def astype(self, dtype: torch.dtype) -> "spMtxCSR5":
        c = spMtxCSR5()
        c.__dict__.update(self.__dict__)
        c.csr_value = self.csr_value.to(dtype)
        return c

    def desc(self) -> _capi.rvvla_csr5:
        d = _capi.rvvla_csr5()
        for k in self.SCALARS:
            setattr(d, k, int(getattr(self, k)))
        for k in self.ARRAYS:
            setattr(d, k, _ptr(getattr(self, k)))
        return d

    def to_host(self) -> dict:
        out = {k: int(getattr(self, k)) for k in self.SCALARS}
        for k in self.ARRAYS:
            out[k] = getattr(self, k).cpu().numpy()
        return out


def _csr5_convert(dist: spMtxCSR5, src: spMtxCRS, params: convertParams) -> None:
    lib = load()
    omega = int(params.param.get("omega", 32))
    sigma = int(params.param.get("sigma", 16))
    owned = _capi.rvvla_csr5_owned()
    d = src.desc()
    st = lib.rvvla_csr5_build(C.byref(d), src.Val.element_size(), omega, sigma, C.byref(owned), _stream())
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        raise (ValueError if st == _capi.RVVLA_ERR_INVALID_ARG else RuntimeError)(msg)
    try:
        h = owned.h
        dev = src.Val.device
        for k in spMtxCSR5.SCALARS:
            setattr(dist, k, int(getattr(h, k)))
        nfull = max(h.p - 1, 0)
        sizes = {"csr_row_pointer": (h.m + 1, torch.int32), "csr_column_index": (h.nnz, torch.int32),
                 "csr_value": (h.nnz, src.Val.dtype), "tile_pointer": (h.p + 1, torch.int32),
                 "tile_descriptor": (nfull * h.omega * h.tile_desc_len, torch.int32),
                 "tile_empty_offset_pointer": (h.p, torch.int32),
                 "tile_empty_offset": (h.num_offsets, torch.int32)}
        for k, (n, dt) in sizes.items():
            setattr(dist, k, _owned_to_tensor(getattr(owned, k), n, dt, dev))
    finally:
        lib.rvvla_csr5_free(C.byref(owned))


# ------------------------------------------------------------------ dispatch


def convert(dist, src: spMtxCRS, params: convertParams | None = None):
    """``convert<T, MtxDist, simd>(dist, src, params)`` run on the GPU."""
    params = params or convertParams()
    builders = _builders()
    for cls, fn in builders.items():
        if isinstance(dist, cls):
            fn(dist, src, params)
            return dist
    raise TypeError(f"convert: unsupported destination {type(dist).__name__}")


def _builders():
    return {spMtxHCSR: _hcsr_convert, spMtxCSR5: _csr5_convert, spMtxSELL_C_Sigma: _sell_convert,
            spMtxVNEC: _vnec_convert, spMtxVHCC: _vhcc_convert, spMtxCVR: _cvr_convert, spMtxLAV: _lav_convert}


def _call_spmv(mat, alpha, b: torch.Tensor, beta, y: torch.Tensor, mixed: bool,
               stage=SPARSE_MATRIX_MV_ALL_STAGES) -> int:
    lib = load()
    st = _stream()
    vt = mat.dtype
    if isinstance(mat, spMtxCVR):
        if mixed:
            return _capi.RVVLA_ERR_UNSUPPORTED
        fn = lib.rvvla_cvr_spmv_f64 if vt == torch.float64 else lib.rvvla_cvr_spmv_f32
        return fn(C.byref(mat.desc()), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxLAV):
        if mixed:
            return _capi.RVVLA_ERR_UNSUPPORTED
        fn = lib.rvvla_lav_spmv_f64 if vt == torch.float64 else lib.rvvla_lav_spmv_f32
        return fn(C.byref(mat.desc()), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxVHCC):
        if mixed:
            return _capi.RVVLA_ERR_UNSUPPORTED
        fn = lib.rvvla_vhcc_spmv_f64 if vt == torch.float64 else lib.rvvla_vhcc_spmv_f32
        if not mat.panels:
            return fn(C.byref(mat.desc()), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        for k, p in enumerate(mat.panels):  # y = alpha * A_k b + (beta, then 1) * y, panel after panel
            rc = fn(C.byref(p.desc()), float(alpha), _ptr(b), float(beta) if k == 0 else 1.0, _ptr(y), st)
            if rc:
                return rc
        return 0
    if isinstance(mat, spMtxVNEC):
        if mixed:
            return _capi.RVVLA_ERR_UNSUPPORTED
        d = mat.desc()
        d.IRD_mat = float(getattr(mat, "IRD_mat", 0.0))
        fn = lib.rvvla_vnec_spmv_f64 if vt == torch.float64 else lib.rvvla_vnec_spmv_f32
        return fn(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxSELL_C_Sigma):
        d = mat.desc()
        if mixed:
            return lib.rvvla_sell_spmv_mixed(C.byref(d), _dtype_code(vt), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        fn = lib.rvvla_sell_spmv_f64 if vt == torch.float64 else lib.rvvla_sell_spmv_f32
        return fn(C.byref(d), int(stage), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxCRS):
        if mixed:
            d = mat.desc(_capi.RVVLA_F32)
            return lib.rvvla_crs_spmv_mixed(C.byref(d), _dtype_code(vt), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        if vt == torch.float64:
            d = mat.desc(_capi.RVVLA_F64)
            return lib.rvvla_crs_spmv_f64(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        d = mat.desc(_capi.RVVLA_F32)
        return lib.rvvla_crs_spmv_f32(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxHCSR):
        d = mat.desc()
        if mixed:
            return lib.rvvla_hcsr_spmv_mixed(C.byref(d), _dtype_code(vt), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        if vt == torch.float64:
            return lib.rvvla_hcsr_spmv_f64(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        return lib.rvvla_hcsr_spmv_f32(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    if isinstance(mat, spMtxCSR5):
        d = mat.desc()
        if mixed:
            return lib.rvvla_csr5_spmv_mixed(C.byref(d), _dtype_code(vt), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        if vt == torch.float64:
            return lib.rvvla_csr5_spmv_f64(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
        return lib.rvvla_csr5_spmv_f32(C.byref(d), float(alpha), _ptr(b), float(beta), _ptr(y), st)
    raise TypeError(f"sparse_mv: unsupported matrix {type(mat).__name__}")


def _vec_type(mat, mixed: bool) -> torch.dtype:
    return torch.float32 if mixed else mat.dtype


def _spmv(op, alpha, mat, descr, b, beta, y, mixed: bool, stage=SPARSE_MATRIX_MV_ALL_STAGES):
    status = sparse_matrix_status()
    transpose = int(op) == int(SPARSE_OPERATION_TRANSPOSE)
    if transpose and (mixed or not isinstance(mat, spMtxCRS) or mat.dtype not in (torch.float64, torch.float32)):
        # A^T b exists for CRS (through the adjoint's transposed layout) only
        status.code = _capi.RVVLA_ERR_UNSUPPORTED
        return status
    vt = _vec_type(mat, mixed)
    host_y = None
    if isinstance(b, np.ndarray):
        b = torch.as_tensor(b).to("cuda", dtype=vt)
    if isinstance(y, np.ndarray):
        host_y = y
        y = torch.as_tensor(y).to("cuda", dtype=vt)
    if b.dtype != vt or y.dtype != vt or not b.is_cuda or not y.is_cuda:
        status.code = _capi.RVVLA_ERR_INVALID_ARG
        return status
    if transpose:
        status.code = _call_transpose(mat, alpha, b, beta, y) if stage in (SPARSE_MATRIX_MV_ALL_STAGES,
                                                                          SPARSE_MATRIX_MV_MULT) else 0
    else:
        status.code = _call_spmv(mat, alpha, b, beta, y, mixed) if stage == SPARSE_MATRIX_MV_ALL_STAGES \
            else _call_stage(mat, alpha, b, beta, y, stage)
    if host_y is not None and status.code == 0:
        host_y[...] = y.cpu().numpy()
    return status


def _call_transpose(mat: "spMtxCRS", alpha, b, beta, y) -> int:
    """y <- alpha*A^T*b + beta*y: the transposed CRS is built on the GPU once
    per matrix (rvvla_csr_transpose) and multiplied by the CRS kernels."""
    if b.numel() < mat.m or y.numel() < mat.n:
        return _capi.RVVLA_ERR_INVALID_ARG
    lib = load()
    key = (mat.Rst.data_ptr(), mat.Col.data_ptr(), mat.Val.dtype)
    tr = getattr(mat, "_transpose", None)
    if tr is None or tr[1] != key:
        owned = _capi.rvvla_transpose_owned()
        st = lib.rvvla_csr_transpose(C.byref(mat.desc()), mat.Val.element_size(), C.byref(owned), _stream())
        if st != 0:
            return st
        tr = (_TransposeHandle(owned), key)
        mat._transpose = tr
    # the current values (they may have changed in place) are read through
    # the transpose's permutation
    fn = (lib.rvvla_spmv_adjoint_x_values_f64 if mat.dtype == torch.float64
          else lib.rvvla_spmv_adjoint_x_values_f32)
    return fn(C.byref(tr[0].owned.h), _ptr(mat.Val), float(alpha), _ptr(b), float(beta), _ptr(y), _stream())


class _TransposeHandle:
    """Owns a library-built transposed CRS (freed with the matrix)."""

    def __init__(self, owned):
        self.owned = owned

    def __del__(self):
        try:
            load().rvvla_csr_transpose_free(C.byref(self.owned))
        except Exception:
            pass


def _call_stage(mat, alpha, b, beta, y, stage):
    # Formats other than SELL-C-sigma have no staged form: PREPARATION and
    # GET_RESULTS are no-ops and MULT is the whole product.
    if isinstance(mat, spMtxSELL_C_Sigma):
        return _call_spmv(mat, alpha, b, beta, y, False, stage)
    if stage == SPARSE_MATRIX_MV_MULT:
        return _call_spmv(mat, alpha, b, beta, y, False)
    return 0


def sparse_mv(op, alpha, mat, descr, b, beta, y, stage=SPARSE_MATRIX_MV_ALL_STAGES):
    """y <- alpha*A*b + beta*y on the GPU (``sparse_mv<T, Mtx, simd, stage>``)."""
    return _spmv(op, alpha, mat, descr, b, beta, y, False, stage)


def sparse_mv_mixed(op, alpha, mat, descr, b, beta, y):
    """Mixed precision form: values fp32/bf16, b and y fp32, compensated fp32
    row sums, fp64 cross-tile merges (no reference counterpart)."""
    return _spmv(op, alpha, mat, descr, b, beta, y, True)
