"""The C++ drop-in: a program written against the reference's C++ API
(sparse_matrix.h, convert, sparse_mv, the spMtx* classes) linked with
librvvla_dropin.so.  CPU: the library exports an overload per format and
value type.  GPU: the program's own checks pass for all eight formats, the
SELL stages and the CRS transpose, and its HCSR arrays (reference default R,
C, p) equal the reference's convert<double, spMtxHCSR, false>."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from rvvlasparse_b200 import build as B

FORMATS = ("spMtxCRS", "spMtxHCSR", "spMtxSELL_C_Sigma", "spMtxCSR5", "spMtxLAV", "spMtxVNEC", "spMtxVHCC",
           "spMtxCVR")


def _exports():
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", B.DROPIN_LIB], capture_output=True, text=True,
                         check=True).stdout
    return out


def test_dropin_library_exports_every_format():
    syms = _exports()
    for f in FORMATS:
        for t in ("double", "float"):
            assert f"SparseMatrixLib::rvvla_sparse_mv(SparseMatrixLib::sparse_operation_t, {t}, " \
                   f"SparseMatrixLib::{f}<{t}> const&" in syms, (f, t)
            if f not in ("spMtxCRS", "spMtxVNEC"):
                assert f"SparseMatrixLib::rvvla_convert(SparseMatrixLib::{f}<{t}>&" in syms, (f, t)
    assert "SparseMatrixLib::spMtxCSR5<double>::asCSR5" in syms
    assert os.path.exists(B.DROPIN_TEST)


def _laplace_crs(g):
    Rst, Col, Val = [0], [], []
    for i in range(g):
        for j in range(g):
            r = i * g + j
            ent = []
            if i > 0:
                ent.append((r - g, -1.0))
            if j > 0:
                ent.append((r - 1, -1.0))
            ent.append((r, 4.0))
            if j < g - 1:
                ent.append((r + 1, -1.0))
            if i < g - 1:
                ent.append((r + g, -1.0))
            for c, v in ent:
                Col.append(c)
                Val.append(v)
            Rst.append(len(Col))
    m = g * g
    return O.crs(m, m, np.array(Rst, np.int32), np.array(Col, np.int32), np.array(Val, np.float64))


def _read_dump(path):
    with open(path, "rb") as f:
        sc = np.frombuffer(f.read(7 * 8), np.uint64)
        arrs = []
        for dt in (np.int32, np.uint32, np.uint32, np.uint16, np.float64):
            n = int(np.frombuffer(f.read(8), np.uint64)[0])
            arrs.append(np.frombuffer(f.read(n * np.dtype(dt).itemsize), dt))
    keys = ("block_ptr", "row_offset", "row_ptr", "col_idx", "values")
    return dict(zip(("R", "C", "m", "n", "nz", "b_m", "b_n"), (int(v) for v in sc)), **dict(zip(keys, arrs)))


@pytest.mark.gpu
def test_dropin_program_on_gpu(tmp_path):
    dump = tmp_path / "hcsr.bin"
    res = subprocess.run([B.DROPIN_TEST, str(dump)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.strip().startswith("OK")
    h = _read_dump(dump)
    A = _laplace_crs(256)
    ref = O.ref_hcsr_convert(A) if O.ref_available() else O.build_hcsr(A, 2000, 2000, 2.0)
    for k in ("R", "C", "m", "n", "nz", "b_m", "b_n"):
        assert h[k] == int(ref[k]), k
    for k in ("block_ptr", "row_offset", "row_ptr", "col_idx", "values"):
        assert np.array_equal(h[k], np.asarray(ref[k]).view(h[k].dtype) if np.asarray(ref[k]).dtype.itemsize ==
                              h[k].dtype.itemsize else ref[k]), k
