"""On-disk formats: the native Matrix Market reader/writer and the binary
CRS container (CPU only)."""
import numpy as np
import pytest

import oracle as O
from rvvlasparse_b200 import io as RIO
from rvvlasparse_b200 import workloads as W


def _rand_crs(m, n, seed, density=0.05):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(m):
        k = rng.binomial(n, density)
        rows.append(np.sort(rng.choice(n, k, replace=False)))
    Rst = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    Col = (np.concatenate(rows) if rows else np.zeros(0)).astype(np.int32)
    Val = rng.standard_normal(len(Col))
    return m, n, Rst, Col, Val


def test_matrix_market_round_trip_bit_exact(tmp_path):
    m, n, Rst, Col, Val = _rand_crs(300, 250, 1)
    p = tmp_path / "a.mtx"
    RIO.write_matrix_market(p, m, n, Rst, Col, Val)
    m2, n2, R2, C2, V2 = RIO.read_matrix_market(p)
    assert (m2, n2) == (m, n)
    assert np.array_equal(R2, Rst) and np.array_equal(C2, Col) and np.array_equal(V2, Val)  # %.17g round-trips


def test_matrix_market_symmetric_pattern_duplicates_and_comments(tmp_path):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n"
                 "% a comment\n"
                 "\n"
                 "4 4 5\n"
                 "1 1 2.0\n"
                 "3 1 -1.5\n"
                 "4 2 0.25\n"
                 "3 1 0.5\n"      # duplicate of (3,1): summed, and mirrored
                 "4 4 7\n")
    m, n, R, Cc, V = RIO.read_matrix_market(p)
    dense = np.zeros((4, 4))
    for i in range(m):
        for k in range(R[i], R[i + 1]):
            dense[i, Cc[k]] += V[k]
        assert np.all(np.diff(Cc[R[i]:R[i + 1]]) > 0)  # ascending, merged
    want = np.array([[2.0, 0, -1.0, 0], [0, 0, 0, 0.25], [-1.0, 0, 0, 0], [0, 0.25, 0, 7.0]])
    assert np.array_equal(dense, want)
    q = tmp_path / "p.mtx"
    q.write_text("%%MatrixMarket matrix coordinate pattern general\n2 3 2\n1 3\n2 1\n")
    m, n, R, Cc, V = RIO.read_matrix_market(q)
    assert (m, n) == (2, 3) and list(R) == [0, 1, 2] and list(Cc) == [2, 0] and list(V) == [1.0, 1.0]
    k = tmp_path / "k.mtx"
    k.write_text("%%MatrixMarket matrix coordinate integer skew-symmetric\n3 3 1\n3 2 4\n")
    m, n, R, Cc, V = RIO.read_matrix_market(k)
    assert list(R) == [0, 0, 1, 2] and list(Cc) == [2, 1] and list(V) == [-4.0, 4.0]


@pytest.mark.parametrize("text,exc", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", ValueError),        # dense array
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", ValueError),  # complex
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n", ValueError),     # truncated
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", ValueError),     # row outside
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1\n", ValueError),         # missing value
    ("hello\n", ValueError),                                                              # no banner
])
def test_matrix_market_rejects_malformed(tmp_path, text, exc):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(exc):
        RIO.read_matrix_market(p)


def test_matrix_market_missing_file(tmp_path):
    with pytest.raises(OSError):
        RIO.read_matrix_market(tmp_path / "none.mtx")


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_binary_crs_round_trip_and_mtx2bin(tmp_path, dt):
    m, n, Rst, Col, Val = W.laplace2d(64)
    p = tmp_path / "a.crs"
    RIO.save_crs(p, m, n, Rst, Col, Val.astype(dt))
    m2, n2, R2, C2, V2 = RIO.load_crs(p)
    assert (m2, n2) == (m, n) and V2.dtype == dt
    assert np.array_equal(R2, Rst) and np.array_equal(C2, Col) and np.array_equal(V2, Val.astype(dt))
    mtx = tmp_path / "a.mtx"
    RIO.write_matrix_market(mtx, m, n, Rst, Col, Val)
    out = tmp_path / "b.crs"
    assert RIO.main(["mtx2bin", str(mtx), str(out)] + (["--fp32"] if dt == np.float32 else [])) == 0
    m3, n3, R3, C3, V3 = RIO.load_crs(out)
    assert np.array_equal(R3, Rst) and np.array_equal(C3, Col) and np.array_equal(V3, Val.astype(dt))
    # the loaded matrix multiplies like the original (oracle CRS SpMV)
    x = W.vector(n, 2)
    y = O.crs_spmv_ld(O.crs(m3, n3, R3, C3, V3.astype(np.float64)), 1.0, x, 0.0, np.zeros(m))
    assert O.normwise_relerr(y, O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))) < 1e-6


def test_binary_crs_rejects_corruption(tmp_path):
    m, n, Rst, Col, Val = _rand_crs(50, 40, 3)
    p = tmp_path / "a.crs"
    RIO.save_crs(p, m, n, Rst, Col, Val)
    raw = bytearray(p.read_bytes())
    bad_magic = tmp_path / "m.crs"
    bad_magic.write_bytes(b"X" + bytes(raw[1:]))
    with pytest.raises(ValueError):
        RIO.load_crs(bad_magic)
    short = tmp_path / "s.crs"
    short.write_bytes(bytes(raw[:-8]))
    with pytest.raises(ValueError):
        RIO.load_crs(short)
    badcol = bytearray(raw)
    off = 48 + 4 * (m + 1)
    badcol[off:off + 4] = np.int32(n + 5).tobytes()
    bc = tmp_path / "c.crs"
    bc.write_bytes(bytes(badcol))
    with pytest.raises(ValueError):
        RIO.load_crs(bc)
    with pytest.raises(ValueError):
        RIO.save_crs(tmp_path / "x.crs", m, n, Rst, Col, Val.astype(np.int64))
