"""GPU parity: VHCC builder (vec_size 32, bit-exact with the oracle builder)
and SpMV against the long-double CSR oracle and the restated RVV kernel."""
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


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def build(m, n, Rst, Col, Val, threads=0):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=TDT[np.asarray(Val).dtype])
    V = R.spMtxVHCC()
    R.convert(V, A, R.convertParams(num_threads=threads))
    return V


def run(mat, alpha, x, beta, y0):
    y = dev(y0)
    st = R.sparse_mv(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


@pytest.mark.parametrize("threads", [1, 7, 64])
def test_vhcc_builder_and_spmv(g, threads):
    V = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], threads)
    o = O.build_vhcc(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), threads, 32)
    h = V.to_host()
    assert np.array_equal(h["thr_info"], o["thr_info"])
    assert np.array_equal(h["veceor_ptr"].view(np.uint32), o["veceor_ptr"])
    assert np.array_equal(h["scan_mask"], o["scan_mask"])
    assert np.array_equal(h["row_arr"].view(np.uint32), o["row_arr"])
    assert np.array_equal(h["col_arr"].view(np.uint32), o["col_arr"])
    assert np.array_equal(h["vals_arr"], o["vals_arr"])
    for k in ("num_vectors", "pad_entries", "pad_rows"):
        assert h[k] == int(o[k]), k
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol
    assert O.normwise_relerr(y, O.spmv(o, g["alpha"], g["x"], g["beta"], g["y0"])) < tol


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vhcc_full_size(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    V = build(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(V, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)


@pytest.mark.parametrize("P", [2, 5])
def test_vhcc_multi_panel(g, P):
    """num_panels > 1: one single-panel structure per column range (each
    bit-exact with the oracle builder on that range), products summed panel
    after panel."""
    A = R.spMtxCRS.from_host(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], dtype=TDT[g["Val"].dtype])
    V = R.spMtxVHCC()
    R.convert(V, A, R.convertParams(num_panels=P, num_threads=7))
    parts = [p for _, _, p in R.formats.column_panels(A, P) if p.nz]
    assert V.num_entries == len(g["Col"])
    if len(g["Col"]):
        assert V.num_panels == len(parts) == len(V.panels)
    for sub, pan in zip(parts, V.panels):
        o = O.build_vhcc(O.crs(sub.m, sub.n, sub.Rst.cpu().numpy(), sub.Col.cpu().numpy(), sub.Val.cpu().numpy()),
                         7, 32)
        h = pan.to_host()
        assert np.array_equal(h["col_arr"].view(np.uint32), o["col_arr"])
        assert np.array_equal(h["vals_arr"], o["vals_arr"])
        assert np.array_equal(h["row_arr"].view(np.uint32), o["row_arr"])
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol_for(g["Val"].dtype)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vhcc_multi_panel_full_size(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=TDT[np.dtype(dt)])
    V = R.spMtxVHCC()
    R.convert(V, A, R.convertParams(num_panels=4))
    assert V.num_panels == 4
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(V, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)
