"""CPU: the oracle restatement against the reference's own outputs.

Golden fixtures (tests/golden, written by the reference scalar library) pin
the restated CRS / HCSR kernels and the HCSR builder bit for bit, and the
reference SELL / LAV / CVR kernels run on our builders' layouts.  The
RVV-only kernels (CSR5, VNEC, VHCC) are checked against the long-double CSR
product within the plain-precision tolerances (1e-12 fp64, 1e-5 fp32).
"""
import numpy as np
import pytest

import oracle as O
from helpers import golden_files, golden_id, load_golden, tol_for

GOLD = golden_files()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def _crs(g):
    return O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])


def test_golden_fixtures_present():
    assert len(GOLD) >= 8


def test_crs_spmv_bitexact_vs_reference(g):
    y = O.spmv(_crs(g), g["alpha"], g["x"], g["beta"], g["y0"])
    assert np.array_equal(y, g["crs_y"])


def test_hcsr_builder_bitexact_vs_reference(g):
    h = O.build_hcsr(_crs(g), int(g["hcsr_R"]), int(g["hcsr_C"]), float(g["hcsr_p"]))
    for k in ("block_ptr", "row_offset", "row_ptr", "col_idx", "values"):
        assert np.array_equal(h[k], g["hcsr_" + k]), k


def test_hcsr_builder_default_params_bitexact(g):
    A = _crs(g)
    R = 2000 if g["Val"].dtype == np.float64 else 4000
    h = O.build_hcsr(A, R, R, 2.0)
    for k in ("row_offset", "block_ptr", "row_ptr"):
        assert np.array_equal(h[k], g["hcsrdef_" + k]), k


def test_hcsr_spmv_bitexact_vs_reference(g):
    h = O.build_hcsr(_crs(g), int(g["hcsr_R"]), int(g["hcsr_C"]), float(g["hcsr_p"]))
    y = O.spmv(h, g["alpha"], g["x"], g["beta"], g["y0"])
    assert np.array_equal(y, g["hcsr_y"])


@pytest.mark.parametrize("fmt", ["sell", "lav", "cvr"])
def test_builders_reproduce_fixture_layouts_and_outputs(g, fmt):
    A = _crs(g)
    b = {"sell": lambda: O.build_sell(A, 8, 32), "lav": lambda: O.build_lav(A, 8, 0.2, 300),
         "cvr": lambda: O.build_cvr(A, 8, 3)}[fmt]()
    for k, v in b.arrays.items():
        assert np.array_equal(v, g[f"{fmt}_{k}"]), k
    y = O.spmv(b, g["alpha"], g["x"], g["beta"], g["y0"])
    assert np.array_equal(y, g[f"{fmt}_y"])


@pytest.mark.parametrize("fmt,params", [
    ("csr5", (4, 4)), ("csr5", (32, 16)), ("csr5", (8, 40)),
    ("vnec", (8, 0)), ("vnec", (8, 1)), ("vnec", (8, 2)), ("vnec", (37, -1)),
    ("vhcc", (8, 8)), ("vhcc", (5, 16)), ("vhcc", (64, 32)),
])
def test_rvv_only_restatements_vs_fp64_oracle(g, fmt, params):
    A = _crs(g)
    b = {"csr5": O.build_csr5, "vnec": O.build_vnec, "vhcc": O.build_vhcc}[fmt](A, *params)
    y = O.spmv(b, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(A, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol_for(g["Val"].dtype)


@pytest.mark.parametrize("fmt", ["hcsr", "sell", "csr5"])
def test_round_trip_to_crs(g, fmt):
    A = _crs(g)
    b = {"hcsr": lambda: O.build_hcsr(A, 64, 100, 2.0), "sell": lambda: O.build_sell(A, 32, 256),
         "csr5": lambda: O.build_csr5(A, 32, 16)}[fmt]()
    back = O.to_crs(b)
    assert np.array_equal(back["Rst"], A["Rst"])
    assert np.array_equal(back["Col"], A["Col"])
    assert np.array_equal(back["Val"], A["Val"])


def test_hcsr_builder_rejects_zero_block_size():
    g = load_golden(GOLD[0])
    with pytest.raises(RuntimeError, match="must be positive"):
        O.build_hcsr(_crs(g), 0, 10, 2.0)


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_reference_convert_defaults_match_oracle_live():
    from rvvlasparse_b200 import workloads as W
    m, n, R, C, V = W.powerlaw(5000, band=200, seed=3)
    for dt in (np.float64, np.float32):
        A = O.crs(m, n, R, C, V.astype(dt))
        r = O.ref_hcsr_convert(A, 300, 700, 1.5)
        o = O.build_hcsr(A, 300, 700, 1.5)
        for k in r.arrays:
            assert np.array_equal(r[k], o[k])


def test_merge_path_split_matches_definition():
    Rst = np.array([0, 3, 3, 3, 9, 10], np.int32)
    ends = Rst[1:]
    nnz = int(Rst[-1])
    for d in range(len(ends) + nnz + 1):
        x, y = O.merge_path(d, ends, nnz)
        assert x + y == d
        # every row end consumed is <= the nonzeros consumed
        assert all(ends[i] <= y for i in range(x))
        if x < len(ends) and y > 0:
            assert not (ends[x] <= y - 1)


def test_transpose_and_sddmm_definitions(g):
    """The oracle's transpose (with permutation) and SDDMM against scipy and
    the definitions (they anchor the GPU adjoint tests)."""
    import scipy.sparse as sp

    m, n = g["m"], g["n"]
    A = O.crs(m, n, g["Rst"], g["Col"], g["Val"])
    t = O.transpose(A)
    S = sp.csr_matrix((g["Val"], g["Col"], g["Rst"]), shape=(m, n)).T.tocsr()
    S.sort_indices()
    assert np.array_equal(t["Rst"], S.indptr) and np.array_equal(t["Col"], S.indices)
    assert np.array_equal(t["Val"], S.data)
    assert np.array_equal(t["Val"], g["Val"][t["perm"]])
    rows = np.repeat(np.arange(m), np.diff(g["Rst"]))
    gv = np.linspace(-1, 1, m)
    dv = O.sddmm(A, gv, g["x"])
    assert np.array_equal(dv, gv[rows] * g["x"].astype(np.float64)[g["Col"]])


def test_rvv_kernel_fixtures(g):
    """The reference's RVV-only kernels' outputs stored in the fixtures
    (tests/golden/make_golden.py, rvv_outputs: CSR5 omega 32 / sigma 16, VHCC,
    VNEC D/S/L on one thread, all on the oracle builders' layouts) against the
    restatements — the pin that holds where the reference sources are absent."""
    dt = g["Val"].dtype
    src = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    a, x, be, y0 = g["alpha"], g["x"], g["beta"], g["y0"]
    tol = tol_for(dt)
    c5 = O.build_csr5(src, int(g["csr5_omega"]), int(g["csr5_sigma"]))
    assert O.normwise_relerr(O.spmv(c5, a, x, be, y0), g["csr5_y"]) < tol
    vh = O.build_vhcc(src, int(g["vhcc_threads"]), int(g["vhcc_lanes"]))
    assert O.normwise_relerr(O.spmv(vh, a, x, be, y0), g["vhcc_y"]) < tol
    for variant in (0, 1, 2):
        vn = O.build_vnec(src, 1, variant)
        assert O.normwise_relerr(O.spmv(vn, a, x, be, y0), g[f"vnec{variant}_y"]) < tol, variant
