"""GPU parity: CSR5 builder (bit-exact with the oracle builder, whose layout
is the one the reference RVV kernel decodes) and CSR5 SpMV (fp64 <= 1e-12,
fp32 <= 1e-5 vs the long-double CSR oracle; mixed <= 1e-6 vs fp64)."""
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


def build(m, n, Rst, Col, Val, omega=32, sigma=16, dt=None):
    dt = dt or TDT[np.asarray(Val).dtype]
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=dt)
    C5 = R.spMtxCSR5()
    R.convert(C5, A, R.convertParams(omega=omega, sigma=sigma))
    return C5


def run(mat, alpha, x, beta, y0, mixed=False):
    y = dev(y0)
    fn = R.sparse_mv_mixed if mixed else R.sparse_mv
    st = fn(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def assert_same_layout(gpu: dict, o):
    for k in ("p", "tail_tile_start", "bit_y_offset", "bit_seg_offset", "tile_desc_len", "num_offsets"):
        assert gpu[k] == int(o[k]), k
    assert np.array_equal(gpu["csr_row_pointer"], o["csr_row_pointer"])
    for k in ("csr_column_index", "tile_pointer", "tile_descriptor", "tile_empty_offset_pointer",
              "tile_empty_offset"):
        assert np.array_equal(gpu[k].view(np.uint32), o[k]), k
    assert np.array_equal(gpu["csr_value"], o["csr_value"])


@pytest.mark.parametrize("omega,sigma", [(32, 16), (32, 4), (32, 24), (32, 40), (8, 8), (4, 4)])
def test_csr5_builder_bitexact_golden(g, omega, sigma):
    C5 = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], omega, sigma)
    o = O.build_csr5(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), omega, sigma)
    assert_same_layout(C5.to_host(), o)


def test_csr5_builder_bitexact_powerlaw():
    m, n, Rst, Col, Val = W.powerlaw(200000, seed=8)
    C5 = build(m, n, Rst, Col, Val)
    o = O.build_csr5(O.crs(m, n, Rst, Col, Val), 32, 16)
    assert_same_layout(C5.to_host(), o)


@pytest.mark.parametrize("sigma", [16, 4, 24, 40])
def test_csr5_spmv_golden(g, sigma):
    C5 = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], 32, sigma)
    y = run(C5, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol_for(g["Val"].dtype)
    # the restated reference kernel agrees on the same layout
    o = O.build_csr5(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), 32, sigma)
    yo = O.spmv(o, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yo) < tol_for(g["Val"].dtype)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_csr5_full_size_powerlaw(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    C5 = build(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(C5, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)
    assert np.array_equal(y, run(C5, 1.0, x, 0.5, y0))  # bitwise reproducible
    code = __import__("ctypes").c_int(-1)
    assert R.load().rvvla_device_status(__import__("ctypes").byref(code), None) == 0 and code.value == 0


def test_csr5_rows_crossing_warps_and_short_rows():
    # one row of 200k entries (spans many warps' tile ranges) amid length-1 rows
    rng = np.random.default_rng(3)
    m, n = 5000, 300000
    lens = np.ones(m, np.int64)
    lens[1234] = 200000
    Rst = np.zeros(m + 1, np.int32)
    Rst[1:] = np.cumsum(lens)
    Col = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]).astype(np.int32)
    Val = rng.uniform(-1, 1, len(Col))
    x = rng.uniform(-1, 1, n)
    C5 = build(m, n, Rst, Col, Val, 32, 8)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    assert O.normwise_relerr(run(C5, 1.0, x, 0.0, np.zeros(m)), yref) < 1e-12


@pytest.mark.parametrize("kind", ["powerlaw", "stencil"])
def test_csr5_mixed_within_1e6(kind):
    if kind == "powerlaw":
        m, n, Rst, Col, Val = W.powerlaw(1 << 20, seed=1)
    else:
        m, n, Rst, Col, Val = W.stencil27(64, seed=3)
    x = W.vector(n, 0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    C5 = build(m, n, Rst, Col, Val.astype(np.float32))
    y = run(C5, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(y, yref) <= 1e-6
    yb = run(C5.astype(torch.bfloat16), 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(yb, yref) < 1e-2


def test_csr5_rejects_non_warp_omega_for_spmv():
    m, n, Rst, Col, Val = W.laplace2d(16)
    C5 = build(m, n, Rst, Col, Val, omega=8, sigma=8)
    y = dev(np.zeros(m))
    st = R.sparse_mv(NT, 1.0, C5, R.sparse_matrix_descr(), dev(np.ones(n)), 0.0, y)
    assert st.code == 4  # RVVLA_ERR_UNSUPPORTED
