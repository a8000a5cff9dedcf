"""GPU parity: SELL-C-sigma builder (bit-exact with the oracle builder and the
golden layouts the reference kernel ran on) and the four SpMV stages against
the reference scalar kernel's outputs (golden) and the long-double oracle."""
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


def build(m, n, Rst, Col, Val, C=32, sigma=256, dt=None):
    dt = dt or TDT[np.asarray(Val).dtype]
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=dt)
    S = R.spMtxSELL_C_Sigma()
    R.convert(S, A, R.convertParams(C=C, sigma=sigma))
    return S


def run(mat, alpha, x, beta, y0, stage=R.SPARSE_MATRIX_MV_ALL_STAGES, mixed=False):
    y = dev(y0)
    if mixed:
        st = R.sparse_mv_mixed(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    else:
        st = R.sparse_mv(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y, stage)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def test_sell_builder_matches_golden_layout(g):
    S = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 8, 32).to_host()
    for k in ("vCl", "vCs", "vBs", "vSBs"):
        assert np.array_equal(S[k], g["sell_" + k]), k
    assert np.array_equal(S["vCol"].view(np.uint32), g["sell_vCol"])
    assert np.array_equal(S["vPerm"].view(np.uint32), g["sell_vPerm"])
    assert np.array_equal(S["vVal"], g["sell_vVal"])


@pytest.mark.parametrize("C,sigma", [(32, 256), (4, 1), (64, 100000), (7, 13)])
def test_sell_builder_bitexact_vs_oracle(C, sigma):
    m, n, Rst, Col, Val = W.powerlaw(50000, seed=12)
    S = build(m, n, Rst, Col, Val, C, sigma).to_host()
    o = O.build_sell(O.crs(m, n, Rst, Col, Val), C, sigma)
    for k in ("vCl", "vCs", "vBs", "vSBs"):
        assert np.array_equal(S[k], o[k]), k
    assert np.array_equal(S["vCol"].view(np.uint32), o["vCol"])
    assert np.array_equal(S["vPerm"].view(np.uint32), o["vPerm"])
    assert np.array_equal(S["vVal"], o["vVal"])


def test_sell_spmv_all_stages_vs_reference_golden(g):
    S = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 8, 32)
    y = run(S, g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    assert O.normwise_relerr(y, g["sell_y"]) < tol
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol


def test_sell_separate_stages_equal_all(g):
    S = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 8, 32)
    y_all = run(S, g["alpha"], g["x"], g["beta"], g["y0"])
    y = dev(g["y0"])
    for st in (R.SPARSE_MATRIX_MV_PREPARATION, R.SPARSE_MATRIX_MV_MULT, R.SPARSE_MATRIX_MV_GET_RESULTS):
        assert R.sparse_mv(NT, g["alpha"], S, R.sparse_matrix_descr(), dev(g["x"]), g["beta"], y, st).code == 0
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), y_all)
    # PREPARATION alone permutes y exactly as the reference stage does
    yp = run(S, g["alpha"], g["x"], g["beta"], g["y0"], R.SPARSE_MATRIX_MV_PREPARATION)
    o = O.build_sell(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), 8, 32)
    assert np.array_equal(yp, O.spmv(o, g["alpha"], g["x"], g["beta"], g["y0"], 0))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_sell_full_size_powerlaw(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    S = build(m, n, Rst, Col, Val, 32, 256)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(S, 1.0, x, -1.0, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, -1.0, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)


def test_sell_mixed_within_1e6():
    m, n, Rst, Col, Val = W.stencil27(64, seed=3)
    x = W.vector(n, 0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    S = build(m, n, Rst, Col, Val.astype(np.float32))
    y = run(S, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(y, yref) <= 1e-6


@pytest.mark.parametrize("C,sigma", [(32, 64), (32, 1)])
def test_sell_warp_slices_all_and_staged(g, C, sigma):
    """C = 32 runs the warp-per-slice kernel; slices wider than 64 columns
    (one_long_row, powerlaw1k) are shared by the whole CTA."""
    S = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], C, sigma)
    tol = tol_for(g["Val"].dtype)
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    y_all = run(S, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y_all, yref) < tol
    y = dev(g["y0"])
    for st in (R.SPARSE_MATRIX_MV_PREPARATION, R.SPARSE_MATRIX_MV_MULT, R.SPARSE_MATRIX_MV_GET_RESULTS):
        assert R.sparse_mv(NT, g["alpha"], S, R.sparse_matrix_descr(), dev(g["x"]), g["beta"], y, st).code == 0
    torch.cuda.synchronize()
    assert O.normwise_relerr(y.cpu().numpy(), yref) < tol
