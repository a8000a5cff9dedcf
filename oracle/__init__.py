"""CPU checkers for the SpMV path — TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``_build/liboracle.so`` — our C++ restatement of the reference algorithms
  (oracle.cpp; each function cites the reference file:line it follows);
* ``_ref/libref_scalar.so`` — the reference's own scalar sources
  (RVVLASparse src/scalar/*.cpp) compiled where they lie, behind the
  ``extern "C"`` shim ref_shim.cpp.  Built only where the reference sources
  are present; the built file travels with the repository snapshot.
* ``_ref/libref_rvv.so`` — the reference's RVV sources (src/rvv/*.cpp: the
  CSR5, VNEC and VHCC kernels, which exist only there, and the RVV CRS, HCSR,
  SELL and LAV products) compiled where they lie against the scalar intrinsic
  stand-in ``rvv_emul/riscv_vector.h`` (VLEN 256), behind the shims
  rvv_shim.cpp (names refv_*) and ref_shim.cpp built for simd = true (refr_*).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker / the timed CPU
baseline.  The product (``rvvlasparse_b200``) never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_scalar.so")
REFV_LIB = os.path.join(HERE, "_ref", "libref_rvv.so")
# The reference checkout: RVVLA_REFERENCE_SRC, else a "reference" directory
# beside the repository.  Only building oracle/_ref reads it.
REF_SRC = os.environ.get("RVVLA_REFERENCE_SRC",
                         os.path.normpath(os.path.join(HERE, "..", "..", "reference")))

I32, U32, U16, U8, F32, F64, I64, U64 = range(8)
_NP = {I32: np.int32, U32: np.uint32, U16: np.uint16, U8: np.uint8, F32: np.float32, F64: np.float64,
       I64: np.int64, U64: np.uint64}
_CODE = {np.dtype(v): k for k, v in _NP.items()}

_olib = None
_rlib = None
_vlib = None


def build(ref: bool = True) -> None:
    """make -C oracle (and the reference libraries, scalar and RVV, when its
    sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True, capture_output=True)
    if ref and os.path.isdir(os.path.join(REF_SRC, "src", "scalar")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True, capture_output=True)


def _lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            build(ref=False)
        L = C.CDLL(ORACLE_LIB)
        vp, i64, dbl, cint = C.c_void_p, C.c_int64, C.c_double, C.c_int
        sig = {
            "orc_bundle_new": (vp, [C.c_char_p]), "orc_bundle_free": (None, [vp]),
            "orc_bundle_fmt": (C.c_char_p, [vp]),
            "orc_bundle_put": (None, [vp, C.c_char_p, cint, vp, i64]),
            "orc_bundle_count": (cint, [vp]), "orc_bundle_name": (C.c_char_p, [vp, cint]),
            "orc_bundle_dtype": (cint, [vp, cint]), "orc_bundle_len": (i64, [vp, cint]),
            "orc_bundle_data": (vp, [vp, cint]), "orc_bundle_set": (None, [vp, C.c_char_p, dbl]),
            "orc_bundle_nscalars": (cint, [vp]), "orc_bundle_scalar_name": (C.c_char_p, [vp, cint]),
            "orc_bundle_scalar": (dbl, [vp, cint]), "orc_last_error": (C.c_char_p, []),
            "orc_build_hcsr": (vp, [vp, i64, i64, dbl]), "orc_build_sell": (vp, [vp, i64, i64]),
            "orc_build_csr5": (vp, [vp, i64, i64]), "orc_build_lav": (vp, [vp, i64, dbl, i64]),
            "orc_build_vnec": (vp, [vp, i64, i64]), "orc_build_vhcc": (vp, [vp, i64, i64]),
            "orc_build_cvr": (vp, [vp, i64, i64]), "orc_to_crs": (vp, [vp]), "orc_transpose": (vp, [vp]),
            "orc_spmv": (cint, [vp, dbl, vp, dbl, vp, cint]),
            "orc_crs_spmv_ld": (None, [vp, dbl, vp, dbl, vp]),
            "orc_sddmm": (None, [vp, vp, vp, vp]),
            "orc_merge_path": (None, [i64, vp, i64, i64, vp]),
            # the seeded workload generators (the library's gen.cpp)
            "rvvla_gen_laplace2d": (i64, [i64, vp, vp, vp]),
            "rvvla_gen_stencil27": (i64, [i64, C.c_uint64, vp, vp, vp]),
            "rvvla_gen_powerlaw": (i64, [i64, dbl, dbl, i64, i64, dbl, C.c_uint64, vp, vp, vp]),
            "rvvla_gen_random_rows": (i64, [i64, i64, cint, dbl, cint, C.c_uint64, vp, vp, vp]),
            "rvvla_gen_vector": (None, [i64, C.c_uint64, cint, dbl, dbl, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _olib = L
    return _olib


# ------------------------------------------------------------ workloads
# The same seeded generators the CUDA library exports (gen.cpp is compiled
# into both), for callers that must not load the CUDA library: the bench's
# CPU-only reference arm.  tests/test_bench_reference_arm.py checks that both
# give equal bits.
def _gen_two_pass(name, m, *args):
    fn = getattr(_lib(), "rvvla_gen_" + name)
    nz = int(fn(*args, None, None, None))
    if nz < 0:
        raise ValueError("generator rejected its arguments")
    Rst = np.empty(m + 1, dtype=np.int32)
    Col = np.empty(nz, dtype=np.int32)
    Val = np.empty(nz, dtype=np.float64)
    fn(*args, Rst.ctypes.data, Col.ctypes.data, Val.ctypes.data)
    return Rst, Col, Val


def gen_laplace2d(g: int):
    Rst, Col, Val = _gen_two_pass("laplace2d", g * g, g)
    return g * g, g * g, Rst, Col, Val


def gen_stencil27(g: int, seed: int = 3):
    Rst, Col, Val = _gen_two_pass("stencil27", g ** 3, g, seed)
    return g ** 3, g ** 3, Rst, Col, Val


def gen_powerlaw(n: int, mean: float = 16.0, sigma: float = 1.2, cap: int = 4096, band: int = 1024,
                 band_frac: float = 0.7, seed: int = 1):
    Rst, Col, Val = _gen_two_pass("powerlaw", n, n, mean, sigma, cap, band, band_frac, seed)
    return n, n, Rst, Col, Val


def gen_vector(n: int, seed: int = 0, normal: bool = False, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    _lib().rvvla_gen_vector(n, seed, 1 if normal else 0, lo, hi, out.ctypes.data)
    return out


class Bundle:
    """A format as named numpy arrays + named scalars (``fmt`` tag)."""

    def __init__(self, fmt: str, arrays: dict | None = None, scalars: dict | None = None):
        self.fmt = fmt
        self.arrays = dict(arrays or {})
        self.scalars = dict(scalars or {})

    def __getitem__(self, k):
        return self.arrays[k] if k in self.arrays else self.scalars[k]

    @property
    def dtype(self):
        return np.float32 if int(self.scalars.get("dtype", F64)) == F32 else np.float64

    def astype(self, dt) -> "Bundle":
        """The same layout with its value arrays cast to ``dt`` (layouts
        depend on the sparsity structure only)."""
        src = np.dtype(self.dtype)
        arrays = {k: (a.astype(dt) if a.dtype == src else a) for k, a in self.arrays.items()}
        b = Bundle(self.fmt, arrays, dict(self.scalars))
        b.scalars["dtype"] = F32 if np.dtype(dt) == np.float32 else F64
        return b

    def _handle(self):
        L = _lib()
        h = L.orc_bundle_new(self.fmt.encode())
        for k, a in self.arrays.items():
            a = np.ascontiguousarray(a)
            L.orc_bundle_put(h, k.encode(), _CODE[a.dtype], a.ctypes.data, a.size)
        for k, v in self.scalars.items():
            L.orc_bundle_set(h, k.encode(), float(v))
        return h

    @staticmethod
    def _from_handle(h) -> "Bundle":
        L = _lib()
        b = Bundle(L.orc_bundle_fmt(h).decode())
        for i in range(L.orc_bundle_count(h)):
            n, dt, ln = L.orc_bundle_name(h, i).decode(), L.orc_bundle_dtype(h, i), L.orc_bundle_len(h, i)
            arr = np.empty(ln, dtype=_NP[dt])
            if ln:
                C.memmove(arr.ctypes.data, L.orc_bundle_data(h, i), arr.nbytes)
            b.arrays[n] = arr
        for i in range(L.orc_bundle_nscalars(h)):
            b.scalars[L.orc_bundle_scalar_name(h, i).decode()] = L.orc_bundle_scalar(h, i)
        L.orc_bundle_free(h)
        return b


def crs(m, n, Rst, Col, Val) -> Bundle:
    Val = np.ascontiguousarray(Val)
    code = F32 if Val.dtype == np.float32 else F64
    return Bundle("crs", {"Rst": np.asarray(Rst, np.int32), "Col": np.asarray(Col, np.int32), "Val": Val},
                  {"m": m, "n": n, "nz": len(Col), "dtype": code})


def _run_builder(fn, src: Bundle, *args) -> Bundle:
    L = _lib()
    h = src._handle()
    out = fn(h, *args)
    L.orc_bundle_free(h)
    if not out:
        raise RuntimeError(L.orc_last_error().decode())
    return Bundle._from_handle(out)


def build_hcsr(src, R, C_, p=2.0):
    return _run_builder(_lib().orc_build_hcsr, src, R, C_, p)


def build_sell(src, C_=32, sigma=256):
    return _run_builder(_lib().orc_build_sell, src, C_, sigma)


def build_csr5(src, omega=32, sigma=16):
    return _run_builder(_lib().orc_build_csr5, src, omega, sigma)


def build_lav(src, lanes=8, T=0.2, segment_len=40000):
    return _run_builder(_lib().orc_build_lav, src, lanes, T, segment_len)


def build_vnec(src, nthreads=8, variant=-1):
    return _run_builder(_lib().orc_build_vnec, src, nthreads, variant)


def build_vhcc(src, nthreads=8, vec_size=8):
    return _run_builder(_lib().orc_build_vhcc, src, nthreads, vec_size)


def build_cvr(src, simd_len=8, nthreads=1):
    return _run_builder(_lib().orc_build_cvr, src, simd_len, nthreads)


def to_crs(fmt: Bundle) -> Bundle:
    return _run_builder(_lib().orc_to_crs, fmt)


def transpose(src: Bundle) -> Bundle:
    return _run_builder(_lib().orc_transpose, src)


def spmv(fmt: Bundle, alpha, b, beta, y, stage: int = 3) -> np.ndarray:
    """Restated reference SpMV; returns the new y (input y is not modified)."""
    L = _lib()
    dt = fmt.dtype
    b = np.ascontiguousarray(b, dtype=dt)
    out = np.array(y, dtype=dt, copy=True)
    h = fmt._handle()
    rc = L.orc_spmv(h, float(alpha), b.ctypes.data, float(beta), out.ctypes.data, stage)
    L.orc_bundle_free(h)
    if rc != 0:
        raise RuntimeError(L.orc_last_error().decode())
    return out


class OracleMatrix:
    """A format held by the oracle library (marshalled once) for timing the
    CPU port of kernels the reference only has as RVV intrinsics."""

    def __init__(self, fmt: Bundle):
        self.fmt = fmt
        self.dt = np.dtype(fmt.dtype)
        self.h = fmt._handle()

    def __del__(self):
        try:
            _lib().orc_bundle_free(self.h)
        except Exception:
            pass

    def time(self, alpha, b, beta, iters: int) -> float:
        import time as _t

        L = _lib()
        b = np.ascontiguousarray(b, dtype=self.dt)
        y = np.zeros(int(self.fmt.scalars.get("m", self.fmt.scalars.get("num_rows", 0))), dtype=self.dt)
        L.orc_spmv(self.h, float(alpha), b.ctypes.data, float(beta), y.ctypes.data, 3)
        ts = []
        for _ in range(iters):
            t0 = _t.perf_counter()
            L.orc_spmv(self.h, float(alpha), b.ctypes.data, float(beta), y.ctypes.data, 3)
            ts.append(_t.perf_counter() - t0)
        return float(np.median(ts))


def crs_spmv_ld(src: Bundle, alpha, b, beta, y) -> np.ndarray:
    """fp64 result of a long-double accumulated CSR SpMV (the FP64 oracle)."""
    L = _lib()
    s64 = Bundle("crs", {k: (v.astype(np.float64) if k == "Val" else v) for k, v in src.arrays.items()},
                 dict(src.scalars, dtype=F64))
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.array(y, dtype=np.float64, copy=True)
    h = s64._handle()
    L.orc_crs_spmv_ld(h, float(alpha), b.ctypes.data, float(beta), out.ctypes.data)
    L.orc_bundle_free(h)
    return out


def sddmm(src: Bundle, g, x) -> np.ndarray:
    L = _lib()
    s64 = Bundle("crs", {k: (v.astype(np.float64) if k == "Val" else v) for k, v in src.arrays.items()},
                 dict(src.scalars, dtype=F64))
    g = np.ascontiguousarray(g, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(len(src.arrays["Col"]), np.float64)
    h = s64._handle()
    L.orc_sddmm(h, g.ctypes.data, x.ctypes.data, out.ctypes.data)
    L.orc_bundle_free(h)
    return out


def merge_path(diagonal: int, a: np.ndarray, b_len: int):
    L = _lib()
    a = np.ascontiguousarray(a, np.int32)
    out = np.zeros(2, np.int64)
    L.orc_merge_path(diagonal, a.ctypes.data, len(a), b_len, out.ctypes.data)
    return int(out[0]), int(out[1])


def normwise_relerr(y, yref) -> float:
    y = np.asarray(y, np.float64)
    yref = np.asarray(yref, np.float64)
    den = np.linalg.norm(yref)
    return float(np.linalg.norm(y - yref) / (den if den > 0 else 1.0))


# ------------------------------------------------------------------ reference
def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref(simd: bool = False):
    """The reference library: its scalar specialisations sparse_mv<T, Fmt,
    false> (libref_scalar.so, names refx_*) or, with ``simd``, its RVV ones
    sparse_mv<T, Fmt, true> on the intrinsic stand-in (libref_rvv.so, names
    refr_*; CRS, HCSR, SELL, LAV — the reference has no RVV CVR)."""
    global _rlib
    if _rlib is None:
        _rlib = {}
    if simd not in _rlib:
        path, pre = (REFV_LIB, "refr_") if simd else (REF_LIB, "refx_")
        if not os.path.exists(path):
            raise RuntimeError(f"reference library {os.path.basename(path)} not built (make -C oracle ref)")
        L = C.CDLL(path)
        vp, i64, dbl, flt, cint = C.c_void_p, C.c_int64, C.c_double, C.c_float, C.c_int
        getattr(L, pre + "last_error").restype = C.c_char_p
        getattr(L, pre + "num_threads").restype = cint
        for S, T in (("f64", dbl), ("f32", flt)):
            def p(name, res, args):
                name = name.replace("refx_", pre).replace("@", S)
                if not hasattr(L, name):  # CVR in the RVV library
                    return
                f = getattr(L, name)
                f.restype, f.argtypes = res, args
            p("refx_crs_new_@", vp, [i64, i64, i64, vp, vp, vp])
            p("refx_crs_free_@", None, [vp])
            p("refx_crs_spmv_@", cint, [vp, T, vp, T, vp])
            p("refx_crs_time_@", dbl, [vp, T, vp, T, cint])
            p("refx_hcsr_convert_@", vp, [vp, cint, cint, dbl, cint, cint, cint])
            p("refx_hcsr_new_@", vp, [vp, vp, vp, vp, vp, vp, vp])
            p("refx_hcsr_free_@", None, [vp])
            p("refx_hcsr_info_@", None, [vp, vp, vp])
            p("refx_hcsr_export_@", None, [vp, vp, vp, vp, vp, vp])
            p("refx_hcsr_spmv_@", cint, [vp, T, vp, T, vp])
            p("refx_hcsr_time_@", dbl, [vp, T, vp, T, cint])
            p("refx_sell_new_@", vp, [vp, vp, vp, vp, vp, vp, vp, vp, i64])
            p("refx_sell_free_@", None, [vp])
            p("refx_sell_spmv_@", cint, [vp, cint, T, vp, T, vp])
            p("refx_sell_time_@", dbl, [vp, T, vp, T, cint])
            p("refx_lav_new_@", vp, [vp, dbl, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp])
            p("refx_lav_free_@", None, [vp])
            p("refx_lav_spmv_@", cint, [vp, T, vp, T, vp])
            p("refx_lav_time_@", dbl, [vp, T, vp, T, cint])
            p("refx_cvr_new_@", vp, [vp, vp, vp, vp, vp, vp])
            p("refx_cvr_free_@", None, [vp])
            p("refx_cvr_spmv_@", cint, [vp, T, vp, T, vp])
            p("refx_cvr_time_@", dbl, [vp, T, vp, T, cint])
        L.prefix = pre
        _rlib[simd] = L
    return _rlib[simd]


def _sfx(dt) -> str:
    return "f32" if np.dtype(dt) == np.float32 else "f64"


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


class RefMatrix:
    """A matrix held by the reference library (owning handle); ``simd``
    selects its RVV specialisations."""

    def __init__(self, kind: str, handle, dt, keep=(), simd: bool = False):
        self.kind, self.h, self.dt, self._keep, self.simd = kind, handle, np.dtype(dt), keep, simd

    def _fn(self, what: str):
        L = _ref(self.simd)
        return getattr(L, f"{L.prefix}{self.kind}_{what}_{_sfx(self.dt)}")

    def __del__(self):
        try:
            self._fn("free")(self.h)
        except Exception:
            pass

    def spmv(self, alpha, b, beta, y, stage: int | None = None) -> np.ndarray:
        b = _a(b, self.dt)
        out = np.array(y, dtype=self.dt, copy=True)
        if self.kind == "sell":
            rc = self._fn("spmv")(self.h, 3 if stage is None else stage, alpha, b.ctypes.data, beta, out.ctypes.data)
        else:
            rc = self._fn("spmv")(self.h, alpha, b.ctypes.data, beta, out.ctypes.data)
        assert rc == 0
        return out

    def time(self, alpha, b, beta, iters: int) -> float:
        b = _a(b, self.dt)
        return self._fn("time")(self.h, alpha, b.ctypes.data, beta, iters)


def ref_crs(src: Bundle, simd: bool = False) -> RefMatrix:
    dt = src.dtype
    L = _ref(simd)
    Rst, Col, Val = _a(src["Rst"], np.int32), _a(src["Col"], np.int32), _a(src["Val"], dt)
    h = getattr(L, f"{L.prefix}crs_new_{_sfx(dt)}")(int(src["m"]), int(src["n"]), int(src["nz"]), Rst.ctypes.data,
                                                Col.ctypes.data, Val.ctypes.data)
    return RefMatrix("crs", h, dt, simd=simd)


def ref_hcsr_convert(src: Bundle, R=None, C_=None, p=None) -> Bundle:
    """Runs the reference convert<T, spMtxHCSR, false>; returns the HCSR arrays."""
    L = _ref()
    dt = src.dtype
    s = _sfx(dt)
    crs_m = ref_crs(src)
    h = getattr(L, f"refx_hcsr_convert_{s}")(crs_m.h, int(R or 0), int(C_ or 0), float(p or 0.0), R is not None,
                                            C_ is not None, p is not None)
    if not h:
        raise RuntimeError(L.refx_last_error().decode())
    info = np.zeros(7, np.int64)
    sizes = np.zeros(5, np.int64)
    getattr(L, f"refx_hcsr_info_{s}")(h, info.ctypes.data, sizes.ctypes.data)
    arrs = {"block_ptr": np.empty(sizes[0], np.int32), "row_offset": np.empty(sizes[1], np.uint32),
            "row_ptr": np.empty(sizes[2], np.uint32), "col_idx": np.empty(sizes[3], np.uint16),
            "values": np.empty(sizes[4], dt)}
    getattr(L, f"refx_hcsr_export_{s}")(h, *(arrs[k].ctypes.data for k in
                                            ("block_ptr", "row_offset", "row_ptr", "col_idx", "values")))
    getattr(L, f"refx_hcsr_free_{s}")(h)
    sc = dict(zip(("R", "C", "m", "n", "nz", "b_m", "b_n"), (int(v) for v in info)))
    sc["dtype"] = F32 if dt == np.float32 else F64
    return Bundle("hcsr", arrs, sc)


def ref_hcsr(b: Bundle, simd: bool = False) -> RefMatrix:
    L = _ref(simd)
    dt = b.dtype
    info = np.array([b[k] for k in ("R", "C", "m", "n", "nz", "b_m", "b_n")], np.int64)
    arrs = [_a(b["block_ptr"], np.int32), _a(b["row_offset"], np.uint32), _a(b["row_ptr"], np.uint32),
            _a(b["col_idx"], np.uint16), _a(b["values"], dt)]
    sizes = np.array([len(a) for a in arrs], np.int64)
    h = getattr(L, f"{L.prefix}hcsr_new_{_sfx(dt)}")(info.ctypes.data, *(a.ctypes.data for a in arrs), sizes.ctypes.data)
    return RefMatrix("hcsr", h, dt, simd=simd)


def ref_sell(b: Bundle, simd: bool = False) -> RefMatrix:
    L = _ref(simd)
    dt = b.dtype
    ints = np.array([b[k] for k in ("m", "n", "cnt_b", "nz", "C", "Sigma")], np.int64)
    arrs = [_a(b[k], np.int32) for k in ("vCl", "vCs", "vBs", "vSBs")]
    col, perm, val = _a(b["vCol"], np.uint32), _a(b["vPerm"], np.uint32), _a(b["vVal"], dt)
    h = getattr(L, f"{L.prefix}sell_new_{_sfx(dt)}")(ints.ctypes.data, *(a.ctypes.data for a in arrs), col.ctypes.data,
                                                perm.ctypes.data, val.ctypes.data, len(col))
    return RefMatrix("sell", h, dt, keep=(arrs, col, perm, val), simd=simd)


def ref_lav(b: Bundle, simd: bool = False) -> RefMatrix:
    L = _ref(simd)
    dt = b.dtype
    ints = np.array([b[k] for k in ("SIMD_Lanes", "m", "n", "nz", "segment_count", "chunk_count", "segment_len")]
                    + [0], np.int64)
    co, cf = _a(b["chunk_offsets"], np.int32), _a(b["chunk_offsets_full_mask"], np.int32)
    sp, oo, mk = _a(b["segment_ptr"], np.uint64), _a(b["out_order"], np.uint32), _a(b["mask"], np.uint16)
    val, ci = _a(b["val"], dt), _a(b["col_id"], np.uint32)
    sR, sC, sV = _a(b["sp_Rst"], np.int32), _a(b["sp_Col"], np.int32), _a(b["sp_Val"], dt)
    lens = np.array([len(co), len(cf), len(sp), len(oo), len(mk), len(val), len(sC)], np.int64)
    h = getattr(L, f"{L.prefix}lav_new_{_sfx(dt)}")(ints.ctypes.data, float(b["T"]), lens.ctypes.data, co.ctypes.data,
                                               cf.ctypes.data, sp.ctypes.data, oo.ctypes.data, mk.ctypes.data,
                                               val.ctypes.data, ci.ctypes.data, sR.ctypes.data, sC.ctypes.data,
                                               sV.ctypes.data)
    return RefMatrix("lav", h, dt, simd=simd)


def ref_cvr(b: Bundle) -> RefMatrix:
    L = _ref()
    dt = b.dtype
    ints = np.array([b[k] for k in ("nItems", "numRows", "numCols", "SIMD_LEN", "Nthreads", "Nthreads_avail")],
                    np.int64)
    vals, cols = _a(b["vPack_vec_vals"], dt), _a(b["vPack_vec_cols"], np.uint32)
    rec, wb = _a(b["vPack_vec_record"], np.int32), _a(b["writeback_pos_record"], np.int32)
    lens = np.array([len(vals), len(rec), len(wb)], np.int64)
    h = getattr(L, f"refx_cvr_new_{_sfx(dt)}")(ints.ctypes.data, lens.ctypes.data, vals.ctypes.data,
                                               cols.ctypes.data, rec.ctypes.data, wb.ctypes.data)
    return RefMatrix("cvr", h, dt)


# ------------------------------------------------ reference RVV kernels
def refv_available() -> bool:
    return os.path.exists(REFV_LIB)


def _refv():
    global _vlib
    if _vlib is None:
        if not os.path.exists(REFV_LIB):
            raise RuntimeError("reference RVV library not built (make -C oracle ref-rvv)")
        L = C.CDLL(REFV_LIB)
        vp, i64, dbl, flt, cint = C.c_void_p, C.c_int64, C.c_double, C.c_float, C.c_int
        L.refv_last_error.restype = C.c_char_p
        L.refv_num_threads.restype = cint
        L.refv_vlen.restype = cint
        L.refv_selftest.restype = cint
        for S, T in (("f64", dbl), ("f32", flt)):
            def p(name, res, args):
                f = getattr(L, name.replace("@", S))
                f.restype, f.argtypes = res, args
            p("refv_csr5_new_@", vp, [vp, vp, vp, vp, vp, vp, vp, vp, vp])
            p("refv_csr5_free_@", None, [vp])
            p("refv_csr5_spmv_@", cint, [vp, cint, T, vp, T, vp])
            p("refv_vhcc_new_@", vp, [vp, vp, vp, vp, vp, vp, vp, vp])
            p("refv_vhcc_free_@", None, [vp])
            p("refv_vhcc_spmv_@", cint, [vp, T, vp, T, vp])
            p("refv_vnec_new_@", vp, [i64, i64, i64, vp, vp, vp, cint])
            p("refv_vnec_free_@", None, [vp])
            p("refv_vnec_info_@", None, [vp, vp, vp])
            p("refv_vnec_spmv_@", cint, [vp, T, vp, T, vp])
            p("refv_vnec_fill_@", cint, [vp] * 20)
        _vlib = L
    return _vlib


def refv_vlen() -> int:
    """VLEN (bits) of the intrinsic stand-in the RVV library was built with."""
    return int(_refv().refv_vlen())


def refv_lanes(sew: int, lmul: int) -> int:
    """VLMAX for SEW-bit elements at LMUL on that VLEN."""
    return refv_vlen() * lmul // sew


class RefRvvMatrix:
    """A matrix held by the reference RVV library (owning handle); spmv runs
    the reference's sparse_mv<T, Fmt, true>."""

    def __init__(self, kind: str, handle, dt, keep=()):
        if not handle:
            raise RuntimeError(_refv().refv_last_error().decode())
        self.kind, self.h, self.dt, self._keep = kind, handle, np.dtype(dt), keep

    def __del__(self):
        try:
            getattr(_refv(), f"refv_{self.kind}_free_{_sfx(self.dt)}")(self.h)
        except Exception:
            pass

    def spmv(self, alpha, b, beta, y) -> np.ndarray:
        b = _a(b, self.dt)
        out = np.array(y, dtype=self.dt, copy=True)
        fn = getattr(_refv(), f"refv_{self.kind}_spmv_{_sfx(self.dt)}")
        if self.kind == "csr5":
            rc = fn(self.h, self.threads, alpha, b.ctypes.data, beta, out.ctypes.data)
        else:
            rc = fn(self.h, alpha, b.ctypes.data, beta, out.ctypes.data)
        assert rc == 0, rc
        return out


def refv_max_threads() -> int:
    return int(_refv().refv_num_threads())


def refv_csr5(b: Bundle, threads: int = 0) -> RefRvvMatrix:
    """The reference's RVV CSR5 kernel (src/rvv/spmv_mtx_csr5.cpp:33-586) on
    a layout from build_csr5; omega must equal a VLMAX of the stand-in
    (e64 m1..m8 / e32 m1..m8), or the reference's entry asserts."""
    dt = b.dtype
    ints = np.array([b[k] for k in ("m", "n", "nnz", "bit_y_offset", "bit_seg_offset", "tile_desc_len",
                                    "tail_tile_start", "p", "omega", "sigma", "num_offsets")], np.int64)
    sew = 64 if dt == np.float64 else 32
    if int(b["omega"]) not in [refv_lanes(sew, k) for k in (1, 2, 4, 8)]:
        raise ValueError(f"refv_csr5: omega {int(b['omega'])} is no VLMAX of e{sew} at VLEN {refv_vlen()}")
    rp, col, val = _a(b["csr_row_pointer"], np.int32), _a(b["csr_column_index"], np.uint32), _a(b["csr_value"], dt)
    tp, td = _a(b["tile_pointer"], np.uint32), _a(b["tile_descriptor"], np.uint32)
    tep, te = _a(b["tile_empty_offset_pointer"], np.uint32), _a(b["tile_empty_offset"], np.uint32)
    lens = np.array([len(rp), len(col), len(tp), len(td), len(tep), len(te)], np.int64)
    h = getattr(_refv(), f"refv_csr5_new_{_sfx(dt)}")(ints.ctypes.data, lens.ctypes.data, rp.ctypes.data,
                                                      col.ctypes.data, val.ctypes.data, tp.ctypes.data,
                                                      td.ctypes.data, tep.ctypes.data, te.ctypes.data)
    mat = RefRvvMatrix("csr5", h, dt)
    # With fewer full tiles than OpenMP threads the reference's CSR5 gives wrong
    # sums in a few per cent of calls (a race in its tile split, observed on
    # 4-tile matrices with 8 threads and never at 1-2 threads or at >= 6 tiles a
    # thread); it runs here with at least 8 full tiles a thread unless told.
    mat.threads = int(threads) if threads else max(1, min(refv_max_threads(), (int(b["p"]) - 1) // 8))
    return mat


def refv_vhcc(b: Bundle) -> RefRvvMatrix:
    """The reference's RVV VHCC kernel (src/rvv/spmv_vhcc.cpp:27-434) on a
    layout from build_vhcc; vec_size must be the kernel's vector length
    (e64m2 / e32m2 VLMAX: 8 fp64 / 16 fp32 at VLEN 256)."""
    dt = b.dtype
    sew = 64 if dt == np.float64 else 32
    if int(b["vec_size"]) != refv_lanes(sew, 2):
        raise ValueError(f"refv_vhcc: vec_size must be {refv_lanes(sew, 2)} for e{sew}m2")
    ints = np.array([b[k] for k in ("num_rows", "num_cols", "num_entries", "num_vectors", "pad_entries",
                                    "pad_rows", "num_threads", "vec_size")], np.int64)
    thr, veo = _a(b["thr_info"], np.int32), _a(b["veceor_ptr"], np.uint32)
    sm = np.ascontiguousarray(b["scan_mask"]).view(np.uint8)
    ra, ca, va = _a(b["row_arr"], np.uint32), _a(b["col_arr"], np.uint32), _a(b["vals_arr"], dt)
    lens = np.array([len(thr), len(veo), len(sm), len(ra), len(ca)], np.int64)
    h = getattr(_refv(), f"refv_vhcc_new_{_sfx(dt)}")(ints.ctypes.data, lens.ctypes.data, thr.ctypes.data,
                                                      veo.ctypes.data, sm.ctypes.data, ra.ctypes.data,
                                                      ca.ctypes.data, va.ctypes.data)
    return RefRvvMatrix("vhcc", h, dt, keep=(thr, veo, sm, ra, ca, va))


def refv_vnec(src: Bundle, layout: Bundle | None = None, threads: int = 0) -> RefRvvMatrix:
    """The reference's own VNEC (constructor include/VNEC.h:200-227, kernels
    src/rvv/spmv_mtx_vnec.cpp:18-738) on a CRS; ``.info()`` gives the variant,
    thread count and IRD (``threads``: the OpenMP team size the constructor
    runs with; 0 = the default).  The reference fills none of the structures its
    kernels read, so ``layout`` (a build_vnec bundle of the same matrix) is
    needed before ``spmv``: its arrays, variant and thread count are set on
    the reference object (rvv_shim.cpp, refv_vnec_fill)."""
    dt = src.dtype
    R, Cc, V = _a(src["Rst"], np.int32), _a(src["Col"], np.int32), _a(src["Val"], dt)
    h = getattr(_refv(), f"refv_vnec_new_{_sfx(dt)}")(int(src["m"]), int(src["n"]), int(src["nz"]), R.ctypes.data,
                                                      Cc.ctypes.data, V.ctypes.data, int(threads))
    keep = [R, Cc, V]
    mat = RefRvvMatrix("vnec", h, dt, keep=keep)
    if layout is not None:
        def arr(k, t):
            if k not in layout.arrays:
                return None
            a = _a(layout[k], t)
            keep.append(a)
            return a

        names = [("thread_coord_start", np.int32), ("thread_coord_end", np.int32), ("NEC_NUM", np.int32),
                 ("use_x_ptr", np.int32), ("use_x_indices", np.int32), ("ecr_indices", np.int32),
                 ("v_row_ptr", np.int32), ("col_start", np.int32), ("val_align", dt), ("tasks", np.int32),
                 ("task_start", np.int32), ("task_end", np.int32), ("spvv_len", np.int32), ("row_begin", np.int32),
                 ("row_end", np.int32), ("reorder_col", np.int32), ("reorder_nnz", dt)]
        got = {k: arr(k, t) for k, t in names}
        ln = lambda k: 0 if got[k] is None else len(got[k])  # noqa: E731
        ints = np.array([int(layout["vnec_t"]), int(layout["NUM_THREADS_VNEC"])], np.int64)
        lens = np.array([ln("ecr_indices"), ln("use_x_indices"), ln("v_row_ptr"), ln("col_start"), ln("val_align"),
                         ln("tasks"), ln("row_begin"), ln("reorder_col")], np.int64)
        keep += [ints, lens]
        ptrs = [None if got[k] is None else got[k].ctypes.data for k, _ in names]
        rc = getattr(_refv(), f"refv_vnec_fill_{_sfx(dt)}")(h, ints.ctypes.data, lens.ctypes.data, *ptrs)
        if rc != 0:
            raise RuntimeError(_refv().refv_last_error().decode())

    def info():
        out = np.zeros(2, np.int64)
        ird = C.c_double()
        getattr(_refv(), f"refv_vnec_info_{_sfx(dt)}")(mat.h, out.ctypes.data, C.byref(ird))
        return {"vnec_t": int(out[0]), "threads": int(out[1]), "IRD_mat": float(ird.value)}

    mat.info = info
    return mat


def ref_num_threads() -> int:
    return int(_ref().refx_num_threads())
