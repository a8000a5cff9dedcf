"""Sparse matrices on disk.

* Matrix Market coordinate files (``read_matrix_market`` /
  ``write_matrix_market``) through the library's native reader and writer;
* the binary CRS container (``save_crs`` / ``load_crs``; ``mtx_to_bin``
  converts a Matrix Market file), a raw dump of Rst / Col / Val behind a
  48-byte header;
* built formats (``save_format`` / ``load_format``): every public field of a
  format object (the reference class's fields; device arrays copied to the
  host) in one ``torch.save`` file, so an expensive GPU build can be cached
  and reloaded onto a device without rebuilding.

The reference's spMtxCRS carries a Matrix Market type code
(include/CRS.h:8,17) but ships no reader, and its test environment names an
"mtx to bin" converter (cmake/TestEnvironment.cmake:62).

Command line: ``python -m rvvlasparse_b200.io mtx2bin in.mtx out.crs [--fp32]``.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np
import torch

from . import _capi
from . import formats as F

_VALUE_ERRORS = (_capi.RVVLA_ERR_INVALID_ARG, _capi.RVVLA_ERR_FORMAT, _capi.RVVLA_ERR_UNSUPPORTED,
                 _capi.RVVLA_ERR_TOO_LARGE)


def _check(lib, st: int) -> None:
    if st != 0:
        msg = lib.rvvla_last_error().decode()
        raise (ValueError if st in _VALUE_ERRORS else OSError)(msg)


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def read_matrix_market(path):
    """(m, n, Rst int32, Col int32, Val float64) of a Matrix Market
    coordinate file; columns ascending in every row, duplicates summed."""
    lib = _capi.load()
    h = _capi.rvvla_host_crs()
    _check(lib, lib.rvvla_mm_read(_path(path), C.byref(h)))
    try:
        m, n, nz = int(h.m), int(h.n), int(h.nz)
        Rst = np.ctypeslib.as_array(C.cast(h.Rst, C.POINTER(C.c_int32)), shape=(m + 1,)).copy()
        Col = (np.ctypeslib.as_array(C.cast(h.Col, C.POINTER(C.c_int32)), shape=(nz,)).copy() if nz
               else np.zeros(0, np.int32))
        Val = (np.ctypeslib.as_array(C.cast(h.Val, C.POINTER(C.c_double)), shape=(nz,)).copy() if nz
               else np.zeros(0, np.float64))
    finally:
        lib.rvvla_host_crs_free(C.byref(h))
    return m, n, Rst, Col, Val


def write_matrix_market(path, m: int, n: int, Rst, Col, Val) -> None:
    """Writes "matrix coordinate real general" with 17 significant digits."""
    lib = _capi.load()
    Rst = np.ascontiguousarray(Rst, dtype=np.int32)
    Col = np.ascontiguousarray(Col, dtype=np.int32)
    Val = np.ascontiguousarray(Val, dtype=np.float64)
    if len(Rst) != m + 1:
        raise ValueError("write_matrix_market: Rst must have m + 1 entries")
    _check(lib, lib.rvvla_mm_write(_path(path), m, n, Rst.ctypes.data, Col.ctypes.data, Val.ctypes.data))


def save_crs(path, m: int, n: int, Rst, Col, Val) -> None:
    """Binary CRS container; Val is stored as fp64 or fp32 as given."""
    lib = _capi.load()
    Rst = np.ascontiguousarray(Rst, dtype=np.int32)
    Col = np.ascontiguousarray(Col, dtype=np.int32)
    Val = np.ascontiguousarray(Val)
    if Val.dtype not in (np.float64, np.float32):
        raise ValueError("save_crs: values must be float64 or float32")
    if len(Rst) != m + 1 or len(Col) != len(Val):
        raise ValueError("save_crs: array lengths do not match m and each other")
    _check(lib, lib.rvvla_crs_save(_path(path), m, n, len(Col), Rst.ctypes.data, Col.ctypes.data, Val.ctypes.data,
                                   Val.itemsize))


def load_crs(path):
    """(m, n, Rst, Col, Val) of a binary CRS file (Val fp64 or fp32 as stored)."""
    lib = _capi.load()
    m, n, nz, vb = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
    p = _path(path)
    _check(lib, lib.rvvla_crs_load_info(p, C.byref(m), C.byref(n), C.byref(nz), C.byref(vb)))
    Rst = np.empty(m.value + 1, np.int32)
    Col = np.empty(nz.value, np.int32)
    Val = np.empty(nz.value, np.float64 if vb.value == 8 else np.float32)
    _check(lib, lib.rvvla_crs_load(p, Rst.ctypes.data, Col.ctypes.data, Val.ctypes.data))
    return m.value, n.value, Rst, Col, Val


def mtx_to_bin(src, dst, dtype=np.float64) -> tuple[int, int, int]:
    """Converts a Matrix Market file into the binary CRS container;
    returns (m, n, nz)."""
    m, n, Rst, Col, Val = read_matrix_market(src)
    save_crs(dst, m, n, Rst, Col, Val.astype(dtype))
    return m, n, len(Col)


_CLASSES = {c.__name__: c for c in (F.spMtxCRS, F.spMtxHCSR, F.spMtxSELL_C_Sigma, F.spMtxCSR5, F.spMtxLAV,
                                    F.spMtxVNEC, F.spMtxVHCC, F.spMtxCVR)}


def _state(obj) -> dict:
    fields = {}
    for k, v in vars(obj).items():
        if k.startswith("_"):  # caches (analysis plans, transposes) are rebuilt on demand
            continue
        if isinstance(v, torch.Tensor):
            fields[k] = ("tensor", v.detach().cpu())
        elif v is None or isinstance(v, (bool, int, float, str)):
            fields[k] = ("value", v)
        elif type(v).__name__ in _CLASSES:
            fields[k] = ("format", _state(v))
        elif isinstance(v, list) and all(type(e).__name__ in _CLASSES for e in v):  # multi-panel VHCC
            fields[k] = ("formats", [_state(e) for e in v])
        else:
            raise TypeError(f"save_format: field {k} of {type(obj).__name__} cannot be stored ({type(v).__name__})")
    return {"class": type(obj).__name__, "fields": fields}


def _restore(state: dict, device):
    cls = _CLASSES.get(state.get("class"))
    if cls is None:
        raise ValueError(f"load_format: unknown format class {state.get('class')!r}")
    obj = cls()
    for k, (kind, v) in state["fields"].items():
        if kind == "tensor":
            v = v.to(device)
        elif kind == "format":
            v = _restore(v, device)
        elif kind == "formats":
            v = [_restore(e, device) for e in v]
        setattr(obj, k, v)
    return obj


def save_format(mat, path) -> None:
    """Stores a built format object (any of the eight classes) in one file."""
    if type(mat).__name__ not in _CLASSES:
        raise TypeError(f"save_format: not a format object: {type(mat).__name__}")
    torch.save({"rvvlasparse_b200_format": 1, "state": _state(mat)}, os.fspath(path))


def load_format(path, device="cuda"):
    """The format object stored by save_format, its arrays on `device`."""
    blob = torch.load(os.fspath(path), map_location="cpu", weights_only=True)
    if not isinstance(blob, dict) or blob.get("rvvlasparse_b200_format") != 1:
        raise ValueError("load_format: not a saved format file")
    return _restore(blob["state"], device)


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if len(argv) >= 3 and argv[0] == "mtx2bin":
        dt = np.float32 if "--fp32" in argv[3:] else np.float64
        m, n, nz = mtx_to_bin(argv[1], argv[2], dt)
        print(f"{argv[2]}: {m} x {n}, {nz} nonzeros, {'fp32' if dt == np.float32 else 'fp64'} values")
        return 0
    print("usage: python -m rvvlasparse_b200.io mtx2bin in.mtx out.crs [--fp32]", file=sys.stderr)
    return 2


if __name__ == "__main__":
    sys.exit(main())
