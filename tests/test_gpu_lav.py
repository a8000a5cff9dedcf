"""GPU parity: LAV builder (bit-exact with the oracle builder and the golden
layouts, whose outputs came from the reference scalar kernel) and LAV SpMV
(sparse part through the CRS kernels, dense segments per launch)."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import golden_files, golden_id, load_golden, tol_for
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = golden_files()
NT = R.SPARSE_OPERATION_NON_TRANSPOSE
TDT = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}
LAYOUT = ("chunk_offsets", "chunk_offsets_full_mask", "segment_ptr", "out_order", "mask", "val", "col_id",
          "sp_Rst", "sp_Col", "sp_Val")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def build(m, n, Rst, Col, Val, lanes=8, T=0.2, seglen=40000):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=TDT[np.asarray(Val).dtype])
    V = R.spMtxLAV()
    R.convert(V, A, R.convertParams(SIMD_Lanes=lanes, T=T, segment_len=seglen))
    return V


def run(mat, alpha, x, beta, y0):
    y = dev(y0)
    st = R.sparse_mv(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


def same(h, o, k):
    a, b = np.asarray(h[k]), np.asarray(o[k])
    return a.shape == b.shape and np.array_equal(a.view(b.dtype) if a.dtype.itemsize == b.dtype.itemsize else a, b)


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def test_lav_golden_layout_and_spmv(g):
    V = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 8, 0.2, 300)
    h = V.to_host()
    for k in LAYOUT:
        assert same(h, {k: g["lav_" + k]}, k), k
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, g["lav_y"]) < tol_for(g["Val"].dtype)


@pytest.mark.parametrize("lanes,T,seglen", [(8, 0.2, 300), (32, 0.0, 7), (16, 0.5, 40000), (4, 1.0, 13),
                                            (32, 0.05, 1)])
def test_lav_builder_and_spmv(g, lanes, T, seglen):
    V = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], lanes, T, seglen)
    A = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    o = O.build_lav(A, lanes, T, seglen)
    h = V.to_host()
    for k in ("SIMD_Lanes", "segment_count", "chunk_count"):
        assert h[k] == int(o[k]), k
    for k in LAYOUT:
        assert same(h, o, k), k
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    assert O.normwise_relerr(y, O.crs_spmv_ld(A, g["alpha"], g["x"], g["beta"], g["y0"])) < tol
    if O.ref_available():  # the reference scalar kernel on the same layout
        assert O.normwise_relerr(y, O.ref_lav(o).spmv(g["alpha"], g["x"], g["beta"], g["y0"])) < tol


def test_lav_rejects_bad_params():
    g = load_golden(GOLD[0])
    with pytest.raises(ValueError):
        build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 0)
    with pytest.raises(ValueError):
        build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 8, 0.2, 0)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_lav_large(dt):
    # a power-law matrix with 2^18 rows: many segments, a non-trivial sparse part
    m, n, Rst, Col, Val = W.powerlaw(1 << 18, seed=3)
    Val = Val.astype(dt)
    V = build(m, n, Rst, Col, Val, 8, 0.2, 4096)
    assert V.segment_count > 1 and V.sparse_part.nz > 0
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(V, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)


@pytest.mark.parametrize("lanes,seglen", [(8, 1 << 18), (8, 4096), (32, 50000), (1, 1 << 18), (4, 9000)])
def test_lav_long_chunks(lanes, seglen):
    # rows of up to 4096 nonzeros: the leading chunks run as one thread block
    # each; the result must not depend on how many chunks take that path
    m, n, Rst, Col, Val = W.powerlaw(1 << 18, seed=11)
    V = build(m, n, Rst, Col, Val, lanes, 0.2, seglen)
    assert 0 < V.long_chunks < V.chunk_count
    x, y0 = W.vector(n, 2), W.vector(m, 3)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.75, x, -0.5, y0)
    for nl in (V.long_chunks, 0, 1, V.chunk_count - 1, V.chunk_count):
        V.long_chunks = nl
        y = run(V, 0.75, x, -0.5, y0)
        assert O.normwise_relerr(y, yref) < tol_for(np.float64), nl


def test_lav_c_abi_builder_carries_sparse_part_plan():
    # the C ABI alone: the builder analyses the sparse part, so a caller that
    # never touches Python plans still gets the CRS lane-run kernel
    import ctypes as C
    from rvvlasparse_b200 import _capi
    m, n, Rst, Col, Val = W.powerlaw(1 << 16, seed=12)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    lib = R.load()
    owned = _capi.rvvla_lav_owned()
    st = torch.cuda.current_stream().cuda_stream
    assert lib.rvvla_lav_build(C.byref(A.desc()), 8, 8, 0.2, 5000, C.byref(owned), st) == 0
    try:
        assert owned.h.sparse_part.nz > 0 and owned.h.sparse_part.plan and owned.h.sparse_part.plan_kind in (1, 2)
        x, y0 = W.vector(n, 1), W.vector(m, 2)
        y = dev(y0)
        assert lib.rvvla_lav_spmv_f64(C.byref(owned.h), 0.5, dev(x).data_ptr(), -1.0, y.data_ptr(), st) == 0
        torch.cuda.synchronize()
        yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, -1.0, y0)
        assert O.normwise_relerr(y.cpu().numpy(), yref) < 1e-12
    finally:
        lib.rvvla_lav_free(C.byref(owned))
