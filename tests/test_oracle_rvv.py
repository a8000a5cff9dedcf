"""Pinning the oracle's CSR5, VHCC and VNEC restatements to the reference's
own RVV-only kernels (src/rvv/spmv_mtx_csr5.cpp, src/rvv/spmv_vhcc.cpp,
src/rvv/spmv_mtx_vnec.cpp), compiled unmodified for x86-64 against the
scalar intrinsic stand-in oracle/rvv_emul/riscv_vector.h (VLEN 256) into
oracle/_ref/libref_rvv.so.

The reference has no builder for CSR5 or VHCC and fills none of VNEC's
kernel structures, so both sides run on the same layout from the oracle's
builders; the reference computes with its own vector code (fused
multiply-adds, its reductions, its thread split), so the check is normwise,
at the restatement tolerances (1e-12 fp64, 1e-5 fp32), against the
restatement and against the long-double CSR oracle.  The reference defects
met on the way are pinned as such (CSR5 sigma > omega, VNEC-D rows spanning
threads).  The reference's RVV versions of the CRS, HCSR, SELL-C-sigma and
LAV products (sparse_mv<T, Fmt, true>, its default) are checked the same
way at the end."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_files, golden_id, load_golden, tol_for
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.skipif(not O.refv_available(), reason="reference RVV library not built")
GOLD = golden_files()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def omegas(dt):
    sew = 64 if np.dtype(dt) == np.float64 else 32
    return [O.refv_lanes(sew, k) for k in (1, 2, 4, 8)]


def test_stand_in_known_answers():
    """oracle/rvv_shim.cpp refv_selftest: mask bit order, viota, vcompress,
    slides, out-of-range gathers, mask-undisturbed adds, the fused vfmacc,
    reductions, byte-offset indexed loads, the vl clamp (0 = all hold)."""
    assert O._refv().refv_selftest() == 0


def test_stand_in_vector_lengths():
    assert O.refv_vlen() == 256
    assert omegas(np.float64) == [4, 8, 16, 32] and omegas(np.float32) == [8, 16, 32, 64]


@pytest.mark.parametrize("omega_sigma", [(32, 8), (32, 16), (32, 24), (32, 32), (16, 16), (8, 4)])
def test_csr5_reference_kernel_golden(g, omega_sigma):
    """The GPU path's tiles (omega 32, sigma 8..32) and smaller ones."""
    omega, sigma = omega_sigma
    dt = g["Val"].dtype
    if omega not in omegas(dt):
        pytest.skip(f"omega {omega} is no VLMAX for {dt}")
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    b = O.build_csr5(src, omega, sigma)
    yr = O.refv_csr5(b).spmv(g["alpha"], g["x"], g["beta"], g["y0"])
    yo = O.spmv(b, g["alpha"], g["x"], g["beta"], g["y0"])
    yld = O.crs_spmv_ld(src, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(yr, yo) < tol_for(dt)
    assert O.normwise_relerr(yr, yld) < tol_for(dt)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_csr5_reference_kernel_powerlaw_all_omegas(dt):
    m, n, R, C, V = W.powerlaw(3000, seed=3)
    V = V.astype(dt)
    src = O.crs(m, n, R, C, V)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    yld = O.crs_spmv_ld(src, 1.25, x, 0.5, y0)
    for omega in omegas(dt):
        for sigma in (4, 8, 16, 32):
            if sigma > omega:
                continue
            b = O.build_csr5(src, omega, sigma)
            yr = O.refv_csr5(b).spmv(1.25, x, 0.5, y0)
            assert O.normwise_relerr(yr, O.spmv(b, 1.25, x, 0.5, y0)) < tol_for(dt), (omega, sigma)
            assert O.normwise_relerr(yr, yld) < tol_for(dt), (omega, sigma)


def test_csr5_reference_sigma_above_omega_skips_part_of_single_row_tiles():
    """The reference passes (sigma, omega) to a simple-tile routine declared
    (omega, sigma) (src/rvv/spmv_mtx_csr5.cpp:161-163 against :44-46): with
    sigma > omega it asks for sigma lanes per step, gets omega (VLMAX), and
    steps sigma elements, so a tile that lies inside one row loses part of its
    sum.  The restatement and the GPU kernels sum the whole tile (the GPU
    tests include sigma 40 > omega 32); only sigma <= omega is pinned."""
    g = load_golden([p for p in GOLD if "one_long_row_f64" in p][0])
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    b = O.build_csr5(src, 4, 16)
    yld = O.crs_spmv_ld(src, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(O.spmv(b, g["alpha"], g["x"], g["beta"], g["y0"]), yld) < 1e-12
    assert O.normwise_relerr(O.refv_csr5(b).spmv(g["alpha"], g["x"], g["beta"], g["y0"]), yld) > 1e-3


def test_csr5_reference_rejects_omega_without_vector_length():
    m, n, R, C, V = W.powerlaw(500, seed=2)
    b = O.build_csr5(O.crs(m, n, R, C, V), 12, 4)
    with pytest.raises(ValueError):
        O.refv_csr5(b)


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_vhcc_reference_kernel_golden(g, threads):
    dt = g["Val"].dtype
    sew = 64 if dt == np.float64 else 32
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    b = O.build_vhcc(src, threads, O.refv_lanes(sew, 2))
    ref = O.refv_vhcc(b)
    for alpha, beta in ((g["alpha"], g["beta"]), (1.0, 0.0)):
        yr = ref.spmv(alpha, g["x"], beta, g["y0"])
        assert O.normwise_relerr(yr, O.spmv(b, alpha, g["x"], beta, g["y0"])) < tol_for(dt)
        assert O.normwise_relerr(yr, O.crs_spmv_ld(src, alpha, g["x"], beta, g["y0"])) < tol_for(dt)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vhcc_reference_kernel_powerlaw(dt):
    m, n, R, C, V = W.powerlaw(3000, seed=3)
    V = V.astype(dt)
    src = O.crs(m, n, R, C, V)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    sew = 64 if dt == np.float64 else 32
    for threads in (1, 3, 8):
        b = O.build_vhcc(src, threads, O.refv_lanes(sew, 2))
        for alpha, beta in ((1.25, 0.5), (1.0, 0.0), (-0.5, 2.0)):
            yr = O.refv_vhcc(b).spmv(alpha, x, beta, y0)
            assert O.normwise_relerr(yr, O.spmv(b, alpha, x, beta, y0)) < tol_for(dt)
            assert O.normwise_relerr(yr, O.crs_spmv_ld(src, alpha, x, beta, y0)) < tol_for(dt)


def test_vhcc_reference_rejects_other_vector_sizes():
    m, n, R, C, V = W.powerlaw(500, seed=2)
    with pytest.raises(ValueError):
        O.refv_vhcc(O.build_vhcc(O.crs(m, n, R, C, V), 2, 32))


# ------------------------------------------------------------------ VNEC
def inside_one_row(b, Rst):
    """Some thread's range starts inside a row and ends in the same row."""
    tcs = np.asarray(b["thread_coord_start"]).reshape(-1, 2)
    tce = np.asarray(b["thread_coord_end"]).reshape(-1, 2)
    return any(s[0] == e[0] and s[1] > Rst[s[0]] for s, e in zip(tcs, tce))


def test_vnec_d_reference_double_counts_rows_spanning_threads():
    """The reference's VNEC-D carry for a thread that starts and ends inside
    one row sums that row from the row's own start (src/rvv/
    spmv_mtx_vnec.cpp:364-446), counting the previous threads' share again;
    the restatement and the GPU kernel start at max(row start, thread
    start).  One 10,000-entry row split over 4 threads shows it."""
    g = load_golden([p for p in GOLD if "one_long_row_f64" in p][0])
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    b = O.build_vnec(src, 4, 0)
    assert inside_one_row(b, g["Rst"])
    yld = O.crs_spmv_ld(src, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(O.spmv(b, g["alpha"], g["x"], g["beta"], g["y0"]), yld) < 1e-12
    assert O.normwise_relerr(O.refv_vnec(src, b).spmv(g["alpha"], g["x"], g["beta"], g["y0"]), yld) > 1e-3


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_vnec_reference_kernels_golden(g, variant):
    """D (0), S (1) and L (2): the reference's kernels (src/rvv/
    spmv_mtx_vnec.cpp:192-586) run on the structures of the oracle's builder,
    which the reference itself never fills."""
    dt = g["Val"].dtype
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    for threads in (1, 4):
        b = O.build_vnec(src, threads, variant)
        ref = O.refv_vnec(src, b)
        assert ref.info()["vnec_t"] == variant and ref.info()["threads"] == threads
        if variant in (0, 2) and inside_one_row(b, g["Rst"]):
            # D: the reference's carry bug, pinned separately below; L: its
            # carry fix-up adds the carries of threads that end in the same
            # row concurrently (src/rvv/spmv_mtx_vnec.cpp:580-585), a race
            continue
        for alpha, beta in ((g["alpha"], g["beta"]), (1.0, 0.0)):
            yr = ref.spmv(alpha, g["x"], beta, g["y0"])
            assert O.normwise_relerr(yr, O.spmv(b, alpha, g["x"], beta, g["y0"])) < tol_for(dt)
            assert O.normwise_relerr(yr, O.crs_spmv_ld(src, alpha, g["x"], beta, g["y0"])) < tol_for(dt)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vnec_reference_kernels_powerlaw(dt):
    m, n, R, C, V = W.powerlaw(3000, seed=3)
    src = O.crs(m, n, R, C, V.astype(dt))
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    for variant in (0, 1, 2):
        for threads in (1, 8):
            b = O.build_vnec(src, threads, variant)
            yr = O.refv_vnec(src, b).spmv(1.25, x, 0.5, y0)
            assert O.normwise_relerr(yr, O.spmv(b, 1.25, x, 0.5, y0)) < tol_for(dt), (variant, threads)
            assert O.normwise_relerr(yr, O.crs_spmv_ld(src, 1.25, x, 0.5, y0)) < tol_for(dt), (variant, threads)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vnec_ird_and_variant_match_reference_single_thread(dt):
    """The reference constructor's IRD and D/S choice (include/VNEC.h:78-227)
    on one OpenMP thread; with more threads its IRD_VNEC races on a shared
    group counter, so only the one-thread value is a fixed point."""
    for m, n, R, C, V in (W.powerlaw(3000, seed=3), W.powerlaw(2500, band=8, seed=9)):
        src = O.crs(m, n, R, C, V.astype(dt))
        info = O.refv_vnec(src, threads=1).info()
        ours = O.build_vnec(src, 1, -1)
        assert info["threads"] == 1
        assert abs(info["IRD_mat"] - float(ours["IRD_mat"])) <= 1e-6 * max(1.0, abs(info["IRD_mat"]))
        assert info["vnec_t"] == int(ours["vnec_t"])


# ------------------------------------------- the reference's simd = true path
def test_rvv_library_has_no_simd_cvr():
    """src/rvv/spmv_mtx_cvr.cpp holds the scalar CVR product again (simd =
    false only), so the RVV build exports no CVR entry points."""
    L = O._ref(simd=True)
    assert not hasattr(L, "refr_cvr_spmv_f64") and hasattr(L, "refr_crs_spmv_f64")


def test_rvv_products_golden(g):
    """sparse_mv<T, Fmt, true> — the reference's default — for CRS, HCSR,
    SELL-C-sigma and LAV (src/rvv/spmv_mtx_{crs,hcsr,sell_c_sigma,lav}.cpp)
    on the oracle's layouts, against the restatement and the long-double
    oracle."""
    dt = g["Val"].dtype
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    a, x, be, y0 = g["alpha"], g["x"], g["beta"], g["y0"]
    yld = O.crs_spmv_ld(src, a, x, be, y0)
    hb, sb, lb = O.build_hcsr(src, 64, 128), O.build_sell(src, 32, 256), O.build_lav(src, 8, 0.2, 40000)
    for name, ref, mine in (("crs", O.ref_crs(src, simd=True), src), ("hcsr", O.ref_hcsr(hb, simd=True), hb),
                            ("sell", O.ref_sell(sb, simd=True), sb), ("lav", O.ref_lav(lb, simd=True), lb)):
        yr = ref.spmv(a, x, be, y0)
        assert O.normwise_relerr(yr, O.spmv(mine, a, x, be, y0)) < tol_for(dt), name
        assert O.normwise_relerr(yr, yld) < tol_for(dt), name


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_rvv_products_powerlaw(dt):
    m, n, R, C, V = W.powerlaw(3000, seed=3)
    src = O.crs(m, n, R, C, V.astype(dt))
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    yld = O.crs_spmv_ld(src, 1.25, x, 0.5, y0)
    for R_, C_ in ((256, 256), (2000, 2000)):
        hb = O.build_hcsr(src, R_, C_)
        assert O.normwise_relerr(O.ref_hcsr(hb, simd=True).spmv(1.25, x, 0.5, y0), yld) < tol_for(dt)
    for C_, sigma in ((8, 1), (32, 256)):
        sb = O.build_sell(src, C_, sigma)
        assert O.normwise_relerr(O.ref_sell(sb, simd=True).spmv(1.25, x, 0.5, y0), yld) < tol_for(dt)
    assert O.normwise_relerr(O.ref_crs(src, simd=True).spmv(1.25, x, 0.5, y0), yld) < tol_for(dt)
    lb = O.build_lav(src, 8, 0.2, 1000)
    assert O.normwise_relerr(O.ref_lav(lb, simd=True).spmv(1.25, x, 0.5, y0), yld) < tol_for(dt)
