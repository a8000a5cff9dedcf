"""Writes tests/golden/*.npz from the REFERENCE scalar library.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture holds its inputs (CSR arrays, x, y0, alpha, beta) and the
reference's outputs: sparse_mv<T, spMtxCRS, false>, convert<T, spMtxHCSR,
false> (all five arrays) and sparse_mv<T, spMtxHCSR, false>, plus the
reference SELL-C-sigma / LAV / CVR kernels run on the layouts our builders
produce (layout arrays stored too).  Inputs come from the library's seeded
generators; the fixtures are what tests compare against, so they are never
regenerated at test time.

Also stored (``add_rvv_outputs``; ``--rvv-only`` adds them to existing
fixtures without touching their other keys): the reference's RVV-only
kernels, built from its src/rvv/ sources on the oracle's intrinsic stand-in
(VLEN 256), run on the oracle builders' layouts — CSR5 (omega 32, sigma 16),
VHCC (3 threads, 8 fp64 / 16 fp32 lanes) and VNEC D, S and L (one thread,
so none of the reference's multi-thread defects applies).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from rvvlasparse_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def cases():
    yield "laplace16", W.laplace2d(16)
    yield "powerlaw1k", W.powerlaw(1000, band=64, seed=7)
    yield "poisson_empty_rows", W.random_rows(700, 900, "poisson", 2.0, "uniform", seed=9)
    yield "one_long_row", _one_long_row()


def _one_long_row():
    # 40 rows; row 17 holds 5000 entries (longer than any tile), others 0..3
    rng = np.random.default_rng(5)
    n = 6000
    rows = []
    for i in range(40):
        k = 5000 if i == 17 else int(rng.integers(0, 4))
        rows.append(np.sort(rng.choice(n, size=k, replace=False)))
    Rst = np.zeros(41, np.int32)
    Rst[1:] = np.cumsum([len(r) for r in rows])
    Col = np.concatenate(rows).astype(np.int32)
    Val = rng.uniform(-1, 1, len(Col))
    return 40, n, Rst, Col, Val


def main():
    O.build(ref=True)
    for name, (m, n, Rst, Col, Val) in cases():
        for dt in (np.float64, np.float32):
            A = O.crs(m, n, Rst, Col, Val.astype(dt))
            x = W.vector(n, 21).astype(dt)
            y0 = W.vector(m, 22).astype(dt)
            alpha, beta = 0.75, -0.5
            d = {"m": m, "n": n, "Rst": Rst, "Col": Col, "Val": Val.astype(dt), "x": x, "y0": y0,
                 "alpha": alpha, "beta": beta}
            d["crs_y"] = O.ref_crs(A).spmv(alpha, x, beta, y0)
            R_, C_ = (64, 128) if m > 64 else (8, 1000)
            h = O.ref_hcsr_convert(A, R_, C_, 2.0)
            d["hcsr_R"], d["hcsr_C"], d["hcsr_p"] = R_, C_, 2.0
            for k in ("block_ptr", "row_offset", "row_ptr", "col_idx", "values"):
                d["hcsr_" + k] = h[k]
            d["hcsr_y"] = O.ref_hcsr(h).spmv(alpha, x, beta, y0)
            hd = O.ref_hcsr_convert(A)  # reference default R, C, p
            d["hcsrdef_row_offset"] = hd["row_offset"]
            d["hcsrdef_block_ptr"] = hd["block_ptr"]
            d["hcsrdef_row_ptr"] = hd["row_ptr"]
            s = O.build_sell(A, 8, 32)
            for k in ("vCl", "vCs", "vBs", "vSBs", "vCol", "vPerm", "vVal"):
                d["sell_" + k] = s[k]
            d["sell_y"] = O.ref_sell(s).spmv(alpha, x, beta, y0)
            lv = O.build_lav(A, 8, 0.2, 300)
            for k, v in lv.arrays.items():
                d["lav_" + k] = v
            d["lav_y"] = O.ref_lav(lv).spmv(alpha, x, beta, y0)
            cv = O.build_cvr(A, 8, 3)
            for k, v in cv.arrays.items():
                d["cvr_" + k] = v
            d["cvr_y"] = O.ref_cvr(cv).spmv(alpha, x, beta, y0)
            rvv_outputs(A, d)
            fn = os.path.join(OUT, f"{name}_{'f64' if dt == np.float64 else 'f32'}.npz")
            np.savez_compressed(fn, **d)
            print("wrote", os.path.relpath(fn, ROOT), os.path.getsize(fn))


def rvv_outputs(A, d):
    """Adds the reference RVV kernels' outputs for the fixture's inputs to d."""
    alpha, beta, x, y0 = float(d["alpha"]), float(d["beta"]), d["x"], d["y0"]
    lanes = 8 if A.dtype == np.float64 else 16
    d["csr5_omega"], d["csr5_sigma"] = 32, 16
    d["csr5_y"] = O.refv_csr5(O.build_csr5(A, 32, 16)).spmv(alpha, x, beta, y0)
    d["vhcc_threads"], d["vhcc_lanes"] = 3, lanes
    d["vhcc_y"] = O.refv_vhcc(O.build_vhcc(A, 3, lanes)).spmv(alpha, x, beta, y0)
    for variant in (0, 1, 2):
        d[f"vnec{variant}_y"] = O.refv_vnec(A, O.build_vnec(A, 1, variant)).spmv(alpha, x, beta, y0)


def add_rvv_outputs():
    O.build(ref=True)
    for fn in sorted(f for f in os.listdir(OUT) if f.endswith(".npz")):
        path = os.path.join(OUT, fn)
        with np.load(path) as z:
            d = {k: z[k] for k in z.files}
        A = O.crs(int(d["m"]), int(d["n"]), d["Rst"], d["Col"], d["Val"])
        rvv_outputs(A, d)
        np.savez_compressed(path, **d)
        print("updated", os.path.relpath(path, ROOT), os.path.getsize(path))


if __name__ == "__main__":
    add_rvv_outputs() if "--rvv-only" in sys.argv[1:] else main()
