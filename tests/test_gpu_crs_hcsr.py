"""GPU parity: CRS and HCSR SpMV, the GPU HCSR builder, mixed precision.

Bars: fp64 <= 1e-12 and fp32 <= 1e-5 normwise relative error against the
long-double CSR oracle; mixed (fp32 values and x, compensated fp32 sums)
<= 1e-6 against the fp64 oracle on the fp64 matrix; the HCSR builder equals
the reference's convert<T, spMtxHCSR, false> bit for bit.
"""
import ctypes as C

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


def dev(a, dt=None):
    t = torch.as_tensor(np.ascontiguousarray(a)).cuda()
    return t if dt is None else t.to(dt)


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def gpu_crs(m, n, Rst, Col, Val, dt=None):
    dt = dt or TDT[np.asarray(Val).dtype]
    return R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=dt)


def run(mat, alpha, x, beta, y0, mixed=False):
    y = dev(y0)
    fn = R.sparse_mv_mixed if mixed else R.sparse_mv
    st = fn(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_crs_golden(g):
    A = gpu_crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    y = run(A, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    assert O.normwise_relerr(y, yref) < tol
    assert O.normwise_relerr(y, g["crs_y"]) < tol


def test_crs_run_to_run_bitwise():
    m, n, Rst, Col, Val = W.powerlaw(200000, seed=2)
    A = gpu_crs(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 1), W.vector(m, 2)
    a = run(A, 1.0, x, 0.5, y0)
    b = run(A, 1.0, x, 0.5, y0)
    assert np.array_equal(a, b)


def test_crs_beta_zero_does_not_read_y():
    m, n, Rst, Col, Val = W.laplace2d(64)
    A = gpu_crs(m, n, Rst, Col, Val)
    x = W.vector(n, 3)
    y = run(A, 2.0, x, 0.0, np.full(m, np.nan))
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 2.0, x, 0.0, np.zeros(m))
    assert np.all(np.isfinite(y)) and O.normwise_relerr(y, yref) < 1e-12


def test_crs_empty_and_all_empty_rows():
    A = gpu_crs(0, 5, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    assert run(A, 1.0, np.ones(5), 0.0, np.zeros(0)).size == 0
    A = gpu_crs(7, 5, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0))
    y0 = np.arange(7, dtype=np.float64)
    assert np.array_equal(run(A, 1.0, np.ones(5), 3.0, y0), 3.0 * y0)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_crs_full_size_powerlaw_vs_oracle(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    A = gpu_crs(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(A, 1.0, x, -0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, -0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)


def test_crs_linearity_full_size():
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    A = gpu_crs(m, n, Rst, Col, Val)
    x1, x2 = W.vector(n, 5), W.vector(n, 6)
    z = np.zeros(m)
    y1, y2, y12 = run(A, 1.0, x1, 0.0, z), run(A, 1.0, x2, 0.0, z), run(A, 1.0, x1 + 2 * x2, 0.0, z)
    assert O.normwise_relerr(y12, y1 + 2 * y2) < 1e-13


@pytest.mark.parametrize("kind", ["powerlaw", "stencil"])
def test_crs_mixed_within_1e6(kind):
    if kind == "powerlaw":
        m, n, Rst, Col, Val = W.powerlaw(1 << 20, seed=1)
    else:
        m, n, Rst, Col, Val = W.stencil27(64, seed=3)
    x = W.vector(n, 0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    A = gpu_crs(m, n, Rst, Col, Val.astype(np.float32), torch.float32)
    y = run(A, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(y, yref) <= 1e-6
    Ab = gpu_crs(m, n, Rst, Col, Val.astype(np.float32), torch.bfloat16)
    yb = run(Ab, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(yb, yref) < 1e-2  # bf16 values: ~2^-9 relative rounding


# ---------------------------------------------------------------- HCSR
def gpu_hcsr(g_or_arrays, R_=None, C_=None, p=None, dt=None):
    m, n, Rst, Col, Val = g_or_arrays
    A = gpu_crs(m, n, Rst, Col, Val, dt)
    prm = {}
    if R_ is not None:
        prm["R"] = R_
    if C_ is not None:
        prm["C"] = C_
    if p is not None:
        prm["p"] = p
    H = R.spMtxHCSR()
    R.convert(H, A, R.convertParams(prm))
    return H


def test_hcsr_gpu_builder_bitexact_vs_reference(g):
    H = gpu_hcsr((g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), int(g["hcsr_R"]), int(g["hcsr_C"]),
                 float(g["hcsr_p"]))
    h = H.to_host()
    assert np.array_equal(h["block_ptr"], g["hcsr_block_ptr"])
    assert np.array_equal(h["row_offset"].view(np.uint32), g["hcsr_row_offset"])
    assert np.array_equal(h["row_ptr"].view(np.uint32), g["hcsr_row_ptr"])
    assert np.array_equal(h["col_idx"].view(np.uint16), g["hcsr_col_idx"])
    assert np.array_equal(h["values"], g["hcsr_values"])


def test_hcsr_gpu_builder_defaults_bitexact(g):
    H = gpu_hcsr((g["m"], g["n"], g["Rst"], g["Col"], g["Val"]))
    h = H.to_host()
    assert np.array_equal(h["row_offset"].view(np.uint32), g["hcsrdef_row_offset"])
    assert np.array_equal(h["block_ptr"], g["hcsrdef_block_ptr"])
    assert np.array_equal(h["row_ptr"].view(np.uint32), g["hcsrdef_row_ptr"])


@pytest.mark.parametrize("R_,C_,p", [(2000, 2000, 2.0), (512, 4096, 0.5), (64, 65536, 8.0), (4096, 1000, 2.0)])
def test_hcsr_gpu_builder_bitexact_vs_oracle_powerlaw(R_, C_, p):
    m, n, Rst, Col, Val = W.powerlaw(300000, seed=4)
    H = gpu_hcsr((m, n, Rst, Col, Val), R_, C_, p).to_host()
    o = O.build_hcsr(O.crs(m, n, Rst, Col, Val), R_, C_, p)
    assert np.array_equal(H["block_ptr"], o["block_ptr"])
    assert np.array_equal(H["row_offset"].view(np.uint32), o["row_offset"])
    assert np.array_equal(H["row_ptr"].view(np.uint32), o["row_ptr"])
    assert np.array_equal(H["col_idx"].view(np.uint16), o["col_idx"])
    assert np.array_equal(H["values"], o["values"])


def test_hcsr_builder_errors_mirror_reference():
    m, n, Rst, Col, Val = W.laplace2d(8)
    with pytest.raises(ValueError):
        gpu_hcsr((m, n, Rst, Col, Val), 0, 4, 2.0)
    # p = 0 makes every non-empty block CSR (R+1 row pointers each): 16384
    # blocks x 65537 entries overflow the 30-bit row_offset field.
    mm = 65536
    Rst = np.arange(mm + 1, dtype=np.int32)
    Col = ((np.arange(mm) * 4) % mm).astype(np.int32)
    with pytest.raises(OverflowError, match="30-bit"):
        gpu_hcsr((mm, mm, Rst, Col, np.ones(mm)), 65536, 4, 0.0)


def test_hcsr_spmv_golden(g):
    H = gpu_hcsr((g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), int(g["hcsr_R"]), int(g["hcsr_C"]),
                 float(g["hcsr_p"]))
    y = run(H, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    assert O.normwise_relerr(y, yref) < tol
    assert O.normwise_relerr(y, g["hcsr_y"]) < tol


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_hcsr_full_size_powerlaw_default_blocks(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    H = gpu_hcsr((m, n, Rst, Col, Val))
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(H, 1.0, x, 0.25, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.25, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)


@pytest.mark.parametrize("kind", ["powerlaw", "stencil"])
def test_hcsr_mixed_within_1e6(kind):
    if kind == "powerlaw":
        m, n, Rst, Col, Val = W.powerlaw(1 << 20, seed=1)
    else:
        m, n, Rst, Col, Val = W.stencil27(64, seed=3)
    x = W.vector(n, 0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    H = gpu_hcsr((m, n, Rst, Col, Val.astype(np.float32)), dt=torch.float32)
    y = run(H, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(y, yref) <= 1e-6
    Hb = H.astype(torch.bfloat16)
    yb = run(Hb, 1.0, x.astype(np.float32), 0.0, np.zeros(m, np.float32), mixed=True)
    assert O.normwise_relerr(yb, yref) < 1e-2


def test_host_vectors_end_to_end():
    m, n, Rst, Col, Val = W.laplace2d(32)
    A = gpu_crs(m, n, Rst, Col, Val)
    x = W.vector(n, 1)
    y = np.zeros(m)
    st = R.sparse_mv(NT, 1.0, A, R.sparse_matrix_descr(), x, 0.0, y)
    assert st.code == 0
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    assert O.normwise_relerr(y, yref) < 1e-12


def test_crs_all_rows_plan_and_edge_rows():
    # no empty rows -> lane-run kernel over all rows (plan kind 1); rows of
    # length 1 (8 row starts per lane), exactly 32, and one row far longer
    # than a warp range
    rng = np.random.default_rng(1)
    m, n = 9000, 40000
    lens = np.ones(m, np.int64)
    lens[100:164] = 32
    lens[5000] = 9000
    lens[7000:7010] = 2048
    Rst = np.zeros(m + 1, np.int32)
    Rst[1:] = np.cumsum(lens)
    Col = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]).astype(np.int32)
    Val = rng.uniform(-1, 1, len(Col))
    A = gpu_crs(m, n, Rst, Col, Val)
    assert A.plan(0)[2] == 1  # all rows
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, m)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, 2.0, y0)
    assert O.normwise_relerr(run(A, 0.5, x, 2.0, y0), yref) < 1e-12
    A32 = gpu_crs(m, n, Rst, Col, Val.astype(np.float32))
    y32 = run(A32, 0.5, x.astype(np.float32), 2.0, y0.astype(np.float32))
    assert O.normwise_relerr(y32, yref) < 1e-5


def test_crs_plan_kinds_and_merge_path(g):
    """Matrices with empty rows get the lane-run kernel over the compacted
    non-empty rows (kind 2), others over all rows (kind 1); a descriptor
    without a plan runs the merge-path kernel.  All agree with the oracle."""
    A = gpu_crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    has_empty = np.any(np.diff(g["Rst"]) == 0)
    assert A.plan(0)[2] == (2 if has_empty else 1)
    tol = tol_for(g["Val"].dtype)
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(run(A, g["alpha"], g["x"], g["beta"], g["y0"]), yref) < tol
    lib = R.load()
    d = A.desc()  # no plan: merge path
    y = dev(g["y0"])
    fn = lib.rvvla_crs_spmv_f64 if g["Val"].dtype == np.float64 else lib.rvvla_crs_spmv_f32
    assert fn(C.byref(d), g["alpha"], dev(g["x"]).data_ptr(), g["beta"], y.data_ptr(),
              torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert O.normwise_relerr(y.cpu().numpy(), yref) < tol


@pytest.mark.parametrize("empty_frac", [0.05, 0.6, 0.99])
def test_crs_plan_over_nonempty_rows(empty_frac):
    """Kind 2 with few, many and almost all rows empty, fp64 and fp32, beta
    on the empty rows included; NaN in y must not survive beta = 0."""
    rng = np.random.default_rng(int(empty_frac * 100))
    m, n = 50000, 30000
    lens = rng.poisson(12, m)
    lens[rng.random(m) < empty_frac] = 0
    Rst = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    Col = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    Val = rng.uniform(-1, 1, len(Col))
    A = gpu_crs(m, n, Rst, Col, Val)
    assert A.plan(0)[2] == 2
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, m)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, 2.0, y0)
    assert O.normwise_relerr(run(A, 0.5, x, 2.0, y0), yref) < 1e-12
    A32 = gpu_crs(m, n, Rst, Col, Val.astype(np.float32))
    y32 = run(A32, 0.5, x.astype(np.float32), 2.0, y0.astype(np.float32))
    assert O.normwise_relerr(y32, yref) < 1e-5
    y0n = np.full(m, np.nan)
    yz = run(A, 1.0, x, 0.0, y0n)
    assert np.all(np.isfinite(yz))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_crs_run_kernel_unaligned_and_tails(dt):
    """The lane-run kernel with Col/Val not 16-byte aligned (scalar loads),
    a nonzero count that leaves a partial chunk and a partial lane, rows of
    length 1 (8 row starts in a lane), rows ending exactly at lane, chunk and
    warp boundaries, and a row longer than a warp's span."""
    rng = np.random.default_rng(5)
    m, n = 6001, 9000
    lens = rng.integers(1, 20, m)
    lens[10:300] = 1
    lens[400:410] = 8
    lens[500:508] = 256
    lens[3000] = 7777
    Rst = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    nz = int(Rst[-1])
    assert nz % 8 != 0
    Col = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    Val = rng.uniform(-1, 1, nz).astype(dt)
    x, y0 = rng.uniform(-1, 1, n).astype(dt), rng.uniform(-1, 1, m).astype(dt)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, -1.5, y0)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    cbig = torch.zeros(nz + 1, dtype=torch.int32, device="cuda")
    vbig = torch.zeros(nz + 1, dtype=tdt, device="cuda")
    cbig[1:] = dev(Col)
    vbig[1:] = dev(Val)
    for Cv, Vv in ((cbig[1:], vbig[1:]), (dev(Col), dev(Val))):
        A = R.spMtxCRS(m, n, nz, dev(Rst), Cv, Vv)
        assert A.plan(0 if dt == np.float64 else 1)[2] == 1
        y = run(A, 0.5, x, -1.5, y0)
        assert O.normwise_relerr(y, yref) < tol_for(dt)
