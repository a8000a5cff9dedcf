"""GPU: HCSR SpMV for every (R, C) the reference accepts, run-to-run
reproducibility, the global-accumulator path for tall block rows, unaligned
arrays, the mixed forms on the full 128^3 stencil, and the GPU builder against
the reference's own convert<double, spMtxHCSR, false> at the 4M-row size.

Bars as elsewhere: fp64 <= 1e-12, fp32 <= 1e-5 normwise against the
long-double CSR oracle; mixed (fp32 values) <= 1e-6 against the fp64 oracle.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import tol_for
from rvvlasparse_b200 import _capi
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
NT = R.SPARSE_OPERATION_NON_TRANSPOSE


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def hcsr(m, n, Rst, Col, Val, dt, **prm):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=dt)
    H = R.spMtxHCSR()
    R.convert(H, A, R.convertParams(prm))
    return H


def run(mat, alpha, x, beta, y0, mixed=False):
    y = dev(y0)
    fn = R.sparse_mv_mixed if mixed else R.sparse_mv
    st = fn(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_hcsr_small_shapes_against_oracle():
    """Block shapes around the kernel's edges on a small matrix: one row per
    block row, block rows of fewer than 16 rows (warps without rows), 3-column
    blocks (tens of thousands of block columns, many windows), p small and
    large (CSR and COO blocks), alpha/beta both non-trivial."""
    m, n, Rst, Col, Val = W.powerlaw(20000, band=256, seed=11)
    x, y0 = W.vector(n, 1), W.vector(m, 2)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.5, x, -0.5, y0)
    for R_, C_, p in ((512, 1024, 2.0), (1, 700, 2.0), (7, 3, 2.0), (100, 5000, 0.01), (3000, 300, 50.0)):
        H = hcsr(m, n, Rst, Col, Val, torch.float64, R=R_, C=C_, p=p)
        assert O.normwise_relerr(run(H, 1.5, x, -0.5, y0), yref) < 1e-12, (R_, C_, p)


@pytest.fixture(scope="module")
def powerlaw4m():
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    x, y0 = W.vector(n, 0), W.vector(m, 1)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, -0.5, y0)
    return m, n, Rst, Col, Val, x, y0, yref


@pytest.mark.parametrize("R_,C_", [(256, 256), (2000, 64), (64, 65536)])
def test_hcsr_any_blocks_full_size_powerlaw(powerlaw4m, R_, C_):
    """Block shapes whose block rows hold tens of thousands of block columns
    (metadata beyond any one staging of a block row) and a block row of 64
    rows spanning all columns; fp64 against the oracle, fp32 too for 256^2."""
    m, n, Rst, Col, Val, x, y0, yref = powerlaw4m
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=R_, C=C_, p=2.0)
    assert O.normwise_relerr(run(H, 1.0, x, -0.5, y0), yref) < 1e-12
    del H
    if R_ == 256:
        H32 = hcsr(m, n, Rst, Col, Val.astype(np.float32), torch.float32, R=R_, C=C_, p=2.0)
        y32 = run(H32, 1.0, x.astype(np.float32), -0.5, y0.astype(np.float32))
        assert O.normwise_relerr(y32, yref) < 1e-5


@pytest.mark.parametrize("R_,C_,p", [(2000, 2000, 2.0), (4000, 4000, 2.0), (300, 70, 0.25), (1, 1 << 16, 2.0),
                                     (5000, 3, 2.0)])
def test_hcsr_run_to_run_bitwise(R_, C_, p):
    """No float atomics: repeated products are bitwise equal (fp64, fp32 and
    the mixed form), here with many COO blocks per block row."""
    m, n, Rst, Col, Val = W.powerlaw(300000, seed=7)
    x, y0 = W.vector(n, 2), W.vector(m, 3)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.5, x, 0.5, y0)
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=R_, C=C_, p=p)
    outs = [run(H, 1.5, x, 0.5, y0) for _ in range(3)]
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    assert O.normwise_relerr(outs[0], yref) < 1e-12
    H32 = hcsr(m, n, Rst, Col, Val.astype(np.float32), torch.float32, R=R_, C=C_, p=p)
    for mixed, tol in ((False, 1e-5), (True, 1e-6)):
        o32 = [run(H32, 1.5, x.astype(np.float32), 0.5, y0.astype(np.float32), mixed) for _ in range(3)]
        assert all(np.array_equal(o32[0], o) for o in o32[1:])
        assert O.normwise_relerr(o32[0], yref) < tol


@pytest.mark.parametrize("R_", [30000, 1 << 20])
def test_hcsr_tall_block_rows(R_):
    """Block rows too tall for a shared-memory accumulator (the accumulator
    moves to a global scratch slice per block row), including one block row
    holding the whole matrix."""
    m, n, Rst, Col, Val = W.powerlaw(200000, seed=8)
    x, y0 = W.vector(n, 4), W.vector(m, 5)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 2.0, y0)
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=R_, C=4096, p=2.0)
    a = run(H, 1.0, x, 2.0, y0)
    assert O.normwise_relerr(a, yref) < 1e-12
    assert np.array_equal(a, run(H, 1.0, x, 2.0, y0))


@pytest.mark.parametrize("how", ["reversed", "ends_swapped"])
def test_hcsr_coo_rows_out_of_order(how):
    """COO blocks whose nonzeros are not in row order (a hand-made HCSR; the
    builder writes them in order): the large ones, which the kernel splits
    among its warps by row, fall back to the COO stream and the product stays
    within the fp64 bar.  Every COO block reversed, or only its first and
    last nonzeros swapped."""
    m, n, Rst, Col, Val = W.powerlaw(300000, seed=12)
    x, y0 = W.vector(n, 1), W.vector(m, 2)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=3000, C=1 << 16, p=50.0)
    ordered = run(H, 1.0, x, 0.5, y0)
    h = H.to_host()
    bp = h["block_ptr"].astype(np.int64)
    ro = h["row_offset"].view(np.uint32)
    rows, cols, vals = h["row_ptr"].copy(), h["col_idx"].copy(), h["values"].copy()
    n_large = 0
    for b in range(len(bp) - 1):
        lo, hi = int(bp[b]), int(bp[b + 1])
        if hi - lo < 2 or (ro[b] >> 30) == 1:
            continue
        off = int(ro[b] & 0x3FFFFFFF)
        if rows[off] == rows[off + hi - lo - 1]:
            continue
        sel = np.arange(hi - lo)[::-1] if how == "reversed" else np.r_[hi - lo - 1, 1:hi - lo - 1, 0]
        rows[off:off + hi - lo] = rows[off:off + hi - lo][sel]
        cols[lo:hi] = cols[lo:hi][sel]
        vals[lo:hi] = vals[lo:hi][sel]
        n_large += hi - lo >= 2048
    assert n_large > 10
    H.row_ptr, H.col_idx, H.values = dev(rows), dev(cols), dev(vals)
    a = run(H, 1.0, x, 0.5, y0)
    assert O.normwise_relerr(a, yref) < 1e-12
    assert O.normwise_relerr(ordered, yref) < 1e-12
    assert np.array_equal(a, run(H, 1.0, x, 0.5, y0))


@pytest.mark.parametrize("p_", [50.0, 2.0])
def test_hcsr_coo_row_beyond_block_row_is_skipped(p_):
    """A hand-made HCSR whose COO nonzero names a row beyond its block row
    (the reference would write out of range): that nonzero is left out and
    every other row is right."""
    m, n, Rst, Col, Val = W.powerlaw(50000, seed=14)
    x, y0 = W.vector(n, 5), W.vector(m, 6)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=512, C=4096, p=p_)
    h = H.to_host()
    bp = h["block_ptr"].astype(np.int64)
    ro = h["row_offset"].view(np.uint32)
    rows = h["row_ptr"].view(np.uint32).copy()
    cnt = np.diff(bp)
    b = int(np.flatnonzero((cnt > 0) & ((ro[:-1] >> 30) != 1))[len(np.flatnonzero((cnt > 0) & ((ro[:-1] >> 30) != 1))) // 2])
    off = int(ro[b] & 0x3FFFFFFF)
    r_loc = int(rows[off])
    rows[off] = 60000  # beyond the 512 rows of the block row
    b_row, b_col = b // H.b_n, b % H.b_n
    k = int(bp[b])
    c_glob = b_col * H.C + int(h["col_idx"].view(np.uint16)[k])
    expect = yref.copy()
    expect[b_row * H.R + r_loc] -= h["values"][k] * x[c_glob]
    H.row_ptr = dev(rows.view(np.int32))
    a = run(H, 1.0, x, 0.5, y0)
    assert O.normwise_relerr(a, expect) < 1e-12


def test_hcsr_large_coo_blocks_all_forms():
    """COO blocks of thousands of nonzeros (p large: every block COO), which
    the kernel streams by row range: fp64, fp32 and the mixed forms against
    the oracle, and bitwise repeatable."""
    m, n, Rst, Col, Val = W.powerlaw(300000, seed=13)
    x, y0 = W.vector(n, 3), W.vector(m, 4)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    H = hcsr(m, n, Rst, Col, Val, torch.float64, R=4000, C=1 << 16, p=50.0)
    cnt = np.diff(H.block_ptr.cpu().numpy())
    assert (cnt >= 1024).sum() > 20  # the row-range path is taken
    a = run(H, 1.0, x, 0.5, y0)
    assert O.normwise_relerr(a, yref) < 1e-12
    assert np.array_equal(a, run(H, 1.0, x, 0.5, y0))
    H32 = hcsr(m, n, Rst, Col, Val.astype(np.float32), torch.float32, R=4000, C=1 << 16, p=50.0)
    x32, y32 = x.astype(np.float32), y0.astype(np.float32)
    assert O.normwise_relerr(run(H32, 1.0, x32, 0.5, y32), yref) < 1e-5
    mixed = run(H32, 1.0, x32, 0.5, y32, mixed=True)
    assert O.normwise_relerr(mixed, yref) < 1e-6
    assert np.array_equal(mixed, run(H32, 1.0, x32, 0.5, y32, mixed=True))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_hcsr_unaligned_arrays(dt):
    """values / col_idx not 16-byte aligned (scalar loads) give the same
    result as the aligned arrays."""
    m, n, Rst, Col, Val = W.powerlaw(100000, seed=9)
    Val = Val.astype(dt)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    H = hcsr(m, n, Rst, Col, Val, tdt, R=1000, C=3000, p=2.0)
    x, y0 = W.vector(n, 1).astype(dt), W.vector(m, 2).astype(dt)
    a = run(H, 1.0, x, 0.5, y0)
    vb = torch.zeros(H.nz + 1, dtype=tdt, device="cuda")
    cb = torch.zeros(H.nz + 1, dtype=torch.int16, device="cuda")
    vb[1:] = H.values
    cb[1:] = H.col_idx
    d = H.desc()
    d.values = vb[1:].data_ptr()
    d.col_idx = cb[1:].data_ptr()
    y = dev(y0)
    lib = R.load()
    fn = lib.rvvla_hcsr_spmv_f64 if dt == np.float64 else lib.rvvla_hcsr_spmv_f32
    rc = fn(C.byref(d), 1.0, dev(x).data_ptr(), 0.5, y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.rvvla_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), a)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(a, yref) < tol_for(dt)


def test_hcsr_degenerate_shapes():
    """A matrix with no nonzeros (y = beta y), a single long row, and
    beta = 0 with NaN in y."""
    Rst = np.zeros(11, np.int32)
    H = hcsr(10, 7, Rst, np.zeros(0, np.int32), np.zeros(0), torch.float64, R=4, C=3, p=2.0)
    y0 = np.arange(10, dtype=np.float64)
    assert np.array_equal(run(H, 1.0, np.ones(7), -2.0, y0), -2.0 * y0)
    rng = np.random.default_rng(3)
    Col = np.sort(rng.choice(50000, 3000, replace=False)).astype(np.int32)
    Val = rng.uniform(-1, 1, 3000)
    H = hcsr(1, 50000, np.array([0, 3000], np.int32), Col, Val, torch.float64, R=1, C=100, p=2.0)
    x = rng.uniform(-1, 1, 50000)
    y = run(H, 1.0, x, 0.0, np.full(1, np.nan))
    assert abs(y[0] - np.dot(Val, x[Col])) < 1e-12 * np.abs(Val * x[Col]).sum()


@pytest.mark.parametrize("fmt", ["hcsr", "csr5"])
def test_mixed_within_1e6_full_stencil128(fmt):
    """The precision form's bar on its own workload: 27-point stencil on the
    128^3 grid (n = 2,097,152, 56.6M nonzeros), fp32 values, fp32 x, error
    against the fp64 oracle <= 1e-6 normwise; bf16 values within their own
    rounding."""
    m, n, Rst, Col, Val = W.stencil27(128, seed=3)
    x = W.vector(n, 0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val.astype(np.float32), dtype=torch.float32)
    M = R.spMtxHCSR() if fmt == "hcsr" else R.spMtxCSR5()
    R.convert(M, A, R.convertParams(dict(R=4000, C=4000, p=2.0) if fmt == "hcsr" else dict(omega=32, sigma=24)))
    y = run(M, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(y, yref) <= 1e-6
    Mb = M.astype(torch.bfloat16)
    yb = run(Mb, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(yb, yref) < 1e-2


@pytest.mark.skipif(not O.ref_available(), reason="reference scalar library not built (oracle/_ref)")
def test_hcsr_builder_bitexact_vs_live_reference_full_size(powerlaw4m):
    """The GPU builder against the reference's convert<double, spMtxHCSR,
    false> run here on the 4M-row power-law matrix with its default R, C, p."""
    m, n, Rst, Col, Val, *_ = powerlaw4m
    ref = O.ref_hcsr_convert(O.crs(m, n, Rst, Col, Val))
    H = hcsr(m, n, Rst, Col, Val, torch.float64)
    h = H.to_host()
    assert (H.R, H.C, H.b_m, H.b_n) == (ref["R"], ref["C"], ref["b_m"], ref["b_n"])
    assert np.array_equal(h["block_ptr"], ref["block_ptr"])
    assert np.array_equal(h["row_offset"].view(np.uint32), ref["row_offset"])
    assert np.array_equal(h["row_ptr"].view(np.uint32), ref["row_ptr"])
    assert np.array_equal(h["col_idx"].view(np.uint16), ref["col_idx"])
    assert np.array_equal(h["values"], ref["values"])


def test_hcsr_c_abi_rejects_bad_descriptors():
    lib = R.load()
    d = _capi.rvvla_hcsr(4, 0, 8, 8, 0, 2, 0, None, None, None, None, None, 0)
    assert lib.rvvla_hcsr_spmv_f64(C.byref(d), 1.0, None, 0.0, None, None) == _capi.RVVLA_ERR_INVALID_ARG
    d = _capi.rvvla_hcsr(4, 70000, 8, 8, 0, 2, 1, None, None, None, None, None, 0)
    assert lib.rvvla_hcsr_spmv_f64(C.byref(d), 1.0, None, 0.0, None, None) != 0
