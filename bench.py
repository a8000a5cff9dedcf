#!/usr/bin/env python
"""SpMV throughput benchmark (GB/s and % of HBM peak per format).

Workload (default): the power-law matrix n = 4,194,304 (lognormal rows, mean
16, sigma 1.2, cap 4096; 70 % of entries within +-1024 of the diagonal, 30 %
uniform; values U[-1,1]; seed 1), nnz ~ 67.1 M, synthetic.

One step = one y = A x pass (alpha 1, beta 0) for every (format, precision)
case below, one after another on one stream.  ``value`` = algorithmic bytes of
all cases / device time of the step (GB/s, whole job over all ranks).  The
algorithmic bytes of a case are the format's own arrays read once, x read
once and y written once (no re-reads counted).  The matrix (>= 0.5 GB per
case) is larger than the 126 MB L2, so every step streams it from HBM; x
(16-32 MB) is meant to stay L2-resident.

``--impl reference`` times the reference's own scalar/OpenMP code on the host
(RVVLASparse src/scalar compiled by oracle/Makefile) on the same workload and
prints the same JSON line.  Under torchrun each rank runs a replica of the
whole workload (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV GB/s & % of HBM peak per format; mixed vs FP64 GPU at <=1e-6 rel err"
N_DEFAULT = 1 << 22


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_table() -> dict:
    p = os.path.join(ROOT, "profiles", "traffic.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def workload(name: str, n: int, cpu_only: bool = False):
    """The synthetic matrix.  cpu_only: generated by the oracle's copy of the
    generators (the same bits), so the reference arm never loads the CUDA
    library."""
    if cpu_only:
        import oracle as W

        gens = {"powerlaw": lambda: W.gen_powerlaw(n, seed=1), "stencil": lambda: W.gen_stencil27(128, seed=3),
                "laplace": lambda: W.gen_laplace2d(256)}
    else:
        from rvvlasparse_b200 import workloads as W

        gens = {"powerlaw": lambda: W.powerlaw(n, seed=1), "stencil": lambda: W.stencil27(128, seed=3),
                "laplace": lambda: W.laplace2d(256)}
    if name not in gens:
        raise SystemExit(f"unknown workload {name}")
    return gens[name]()


def config_for(args, m: int, nnz: int, case_names: list, world: int) -> dict:
    """The workload description, identical in both arms."""
    cfg = {"workload": f"{args.workload} n={m} nnz={nnz}", "cases": case_names, "alpha": 1.0, "beta": 0.0,
           "parallelism": f"replicas{world}",
           "l2": "matrix arrays larger than the 126 MB L2 (streamed from HBM every step); x L2-resident"}
    if getattr(args, "params", ""):
        cfg["params"] = parse_params(args.params)
    return cfg


# formats the reference implements in C++ (src/scalar, built unmodified into
# oracle/_ref); CSR5, VNEC and VHCC exist there only as RVV intrinsics, so
# their CPU timings are the oracle's single-threaded restatements
REF_LIBRARY_FORMATS = ("crs", "hcsr", "sell", "lav", "cvr")


# ----------------------------------------------------------------- GPU cases
class Case:
    """One (format, precision) SpMV on the device."""

    def __init__(self, name, mat, prec, nbytes, nnz, m, n, csr_bytes_=None):
        import torch

        self.name, self.mat, self.prec, self.bytes, self.nnz = name, mat, prec, nbytes, nnz
        # the same product's bytes in plain CSR (values of this precision,
        # int32 columns and row pointers, x, y): padding and format metadata
        # do not count as useful work there
        self.csr_bytes = csr_bytes_ if csr_bytes_ is not None else nbytes
        vt = torch.float64 if prec == "f64" else torch.float32  # mixed forms: fp32 x and y
        self.vt = vt
        self.x = torch.empty(n, dtype=vt, device="cuda")
        self.y = torch.zeros(m, dtype=vt, device="cuda")
        self.kernel_ms = []

    def launch(self):
        import rvvlasparse_b200 as R

        fn = R.sparse_mv_mixed if self.prec.startswith("mixed") else R.sparse_mv
        st = fn(R.SPARSE_OPERATION_NON_TRANSPOSE, 1.0, self.mat, R.sparse_matrix_descr(), self.x, 0.0, self.y)
        if st.code != 0:
            raise RuntimeError(f"{self.name}: status {st.code}: {R.load().rvvla_last_error().decode()}")


def crs_bytes(m, n, nnz, vb, xb):
    return nnz * (vb + 4) + (m + 1) * 4 + n * xb + m * xb


def hcsr_bytes(H, vb, xb):
    nb1 = H.b_m * H.b_n + 1
    return H.nz * (vb + 2) + H.row_ptr.numel() * 4 + nb1 * 8 + H.n * xb + H.m * xb


def csr5_bytes(m, n, nnz, p, omega, tdl, nofs, vb, xb):
    # values + columns, row pointer (tail rows), tile pointers, descriptors,
    # empty-offset pointers/map, x and y
    return (nnz * (vb + 4) + (m + 1) * 4 + (p + 1) * 4 + max(p - 1, 0) * omega * tdl * 4 + p * 4 + nofs * 4
            + n * xb + m * xb)


def sell_bytes(S, vb, xb):
    # values + columns (padded slices), four slice arrays, permutation, x, y
    return S.len * (vb + 4) + S.cnt_b * 16 + S.m * 4 + S.n * xb + S.m * xb


def lav_bytes(Lv, vb, xb):
    # dense steps (values, columns, masks), chunk offsets (both), segment
    # pointers, the row placement the kernel reads (one-pass kernel: the
    # 1-byte slot->lane map and the row order; otherwise out_order), then the
    # sparse part as CRS (with x and y)
    L, cc, ns = Lv.SIMD_Lanes, Lv.chunk_count, Lv.segment_count
    fused = getattr(Lv, "lane_of_slot", None) is not None and L <= 32 and 32 % L == 0
    place = ns * cc * L + Lv.m * 4 if fused else ns * cc * L * 4
    dense = Lv.n_steps * L * (vb + 4) + Lv.n_steps * 2 + place + (2 * cc + 1) * ns * 4 + (ns + 1) * 8
    return dense + crs_bytes(Lv.m, Lv.n, Lv.sparse_part.nz, vb, xb)


def vnec_bytes(Vn, vb, xb):
    # the source CRS arrays plus the per-thread merge coordinates
    return crs_bytes(Vn.m, Vn.n, Vn.nz, vb, xb) + Vn.NUM_THREADS_VNEC * 16


def vhcc_bytes(Vh, vb, xb):
    # vectors (values, columns), end-of-row vector list, scan/write masks,
    # row list, per-thread info, x, y
    return (Vh.num_vectors * Vh.vec_size * (vb + 4) + Vh.n_eor * 4 + Vh.scan_mask_bytes + Vh.n_rowarr * 4
            + Vh.num_threads * 40 + Vh.num_cols * xb + Vh.num_rows * xb)


def cvr_bytes(Cv, vb, xb):
    return Cv.nItems * (vb + 4) + Cv.n_record * 4 + Cv.n_writeback * 4 + Cv.numCols * xb + Cv.numRows * xb


# formats whose SpMV has a mixed-precision form
MIXED = ("crs", "hcsr", "csr5", "sell")


def parse_params(text: str) -> dict:
    """--params "hcsr:R=2000,C=65536;csr5:sigma=24" -> {fmt: {key: number}}."""
    out = {}
    for part in filter(None, (t.strip() for t in text.split(";"))):
        fmt, _, kv = part.partition(":")
        d = out.setdefault(fmt.strip(), {})
        for item in filter(None, kv.split(",")):
            k, _, v = item.partition("=")
            d[k.strip()] = float(v) if "." in v else int(v)
    return out


def build_cases(m, n, Rst, Col, Val, formats, precs, overrides=None):
    """One Case per (format, precision).  Precisions: f64, f32, mixed (fp32
    values, compensated fp32 sums, fp64 carry merges) and mixed_bf16 (the
    same with bf16 values); the mixed forms exist for CRS, HCSR, CSR5, SELL.
    overrides: {fmt: convertParams entries} over the defaults below."""
    import torch

    import rvvlasparse_b200 as R

    cases = []
    A64 = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    A32 = A64.astype(torch.float32)
    nnz = A64.nz
    x64 = torch.as_tensor(np.random.default_rng(0).uniform(-1, 1, n)).cuda()
    vbytes = {"f64": 8, "f32": 4, "mixed": 4, "mixed_bf16": 2}
    spec = {
        "crs": (None, {}, lambda M, vb, xb: crs_bytes(m, n, nnz, vb, xb)),
        "hcsr": (R.spMtxHCSR, {}, lambda M, vb, xb: hcsr_bytes(M, vb, xb)),
        "csr5": (R.spMtxCSR5, dict(omega=32, sigma=16),
                 lambda M, vb, xb: csr5_bytes(m, n, nnz, M.p, M.omega, M.tile_desc_len, M.num_offsets, vb, xb)),
        "sell": (R.spMtxSELL_C_Sigma, dict(C=32, sigma=256), sell_bytes),
        # x stays in L2, so the GPU needs no column segments for cache
        # blocking: one segment (segment_len = n) also avoids the padding that
        # many short segments add (2.6x the dense part at the CPU default
        # segment_len = 40000 on this matrix)
        "lav": (R.spMtxLAV, dict(SIMD_Lanes=8, T=0.2, segment_len=max(n, 1)), lav_bytes),
        "vnec": (R.spMtxVNEC, {}, vnec_bytes),
        "vhcc": (R.spMtxVHCC, {}, vhcc_bytes),
        "cvr": (R.spMtxCVR, {}, cvr_bytes)}
    for fmt in formats:
        cls, params, nbytes = spec[fmt]
        params = {**params, **(overrides or {}).get(fmt, {})}
        built = {}
        for p in precs:
            if p.startswith("mixed") and fmt not in MIXED:
                continue
            key = "f64" if p == "f64" else "f32"
            if key not in built:
                src = A64 if key == "f64" else A32
                if cls is None:
                    built[key] = src
                else:
                    M = cls()
                    R.convert(M, src, R.convertParams(**params))
                    built[key] = M
            mat = built[key].astype(torch.bfloat16) if p == "mixed_bf16" else built[key]
            vb, xb = vbytes[p], (8 if p == "f64" else 4)
            cases.append(Case(f"{fmt}_{p}", mat, p, nbytes(mat, vb, xb), nnz, m, n, crs_bytes(m, n, nnz, vb, xb)))
    for c in cases:
        c.x.copy_(x64.to(c.vt))
    return cases


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during timing."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(v: float, world: int, device: str) -> float:
    """The slowest rank's value (every rank must call it, in the same order);
    world 1 returns v unchanged."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gbs(bytes_per_rank: int, world: int, step_ms: float) -> float:
    """Whole-job throughput of `world` replicas that each move bytes_per_rank
    in a step whose slowest rank took step_ms."""
    return bytes_per_rank * world / (step_ms * 1e-3) / 1e9


def run_gpu(args):
    import torch
    import torch.distributed as dist

    import rvvlasparse_b200 as R

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib = R.load()
    m, n, Rst, Col, Val = workload(args.workload, args.n)
    cases = build_cases(m, n, Rst, Col, Val, args.formats.split(","), args.precisions.split(","),
                        parse_params(args.params))
    stream = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 3)):
        for c in cases:
            c.launch()
    torch.cuda.synchronize()

    # ---- device-timed step (inputs resident in HBM)
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in cases]
          for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    for c in cases:  # one untimed pass: the clocks come back up after the pause
        c.launch()
    torch.cuda.synchronize()
    l0 = lib.rvvla_kernel_launch_count()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()  # no collector pause of the launching thread inside the timed region
    t_start.record(stream)
    for s in range(args.steps):
        for c, (e0, e1) in zip(cases, ev[s]):
            e0.record(stream)
            c.launch()
            e1.record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    launches = lib.rvvla_kernel_launch_count() - l0
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    step_ms = t_start.elapsed_time(t_end) / args.steps
    for s in range(args.steps):
        for c, (e0, e1) in zip(cases, ev[s]):
            c.kernel_ms.append(e0.elapsed_time(e1))
    step_ms = max_over_ranks(step_ms, world, "cuda")
    total_bytes = sum(c.bytes for c in cases)
    value = job_gbs(total_bytes, world, step_ms)
    value_csr_equiv = job_gbs(sum(c.csr_bytes for c in cases), world, step_ms)

    # ---- end to end through the reference-facing API: the C++ drop-in's
    # sparse_mv with host std::vector b and y (a harness process on this
    # rank's GPU); the Python API with pinned buffers and copies overlapped
    # across cases is reported beside it
    e2e_ms_py, h2d_py, d2h_py = e2e_time(cases, args, torch)
    e2e_ms_py = max_over_ranks(e2e_ms_py, world, "cuda")
    drop = None if args.no_e2e else e2e_dropin(args, [c.name for c in cases], local)
    e2e_ms = max_over_ranks(drop["ms_per_step"] if drop else float("inf"), world, "cuda")

    pk = peaks()
    per = {}
    for c in cases:
        ms = statistics.median(c.kernel_ms)
        gbs = c.bytes / (ms * 1e-3) / 1e9
        ceq = c.csr_bytes / (ms * 1e-3) / 1e9
        per[c.name] = {"ms": round(ms, 4), "gbs": round(gbs, 1), "frac_of_hbm": round(gbs / pk["hbm_gbs"], 4),
                       "gflops": round(2 * c.nnz / (ms * 1e-3) / 1e9, 1), "bytes": int(c.bytes),
                       "csr_equiv_bytes": int(c.csr_bytes), "csr_equiv_gbs": round(ceq, 1),
                       "csr_equiv_frac": round(ceq / pk["hbm_gbs"], 4)}
    dom = max(cases, key=lambda c: statistics.mean(c.kernel_ms))
    dom_ms = statistics.mean(dom.kernel_ms)
    achieved = dom.bytes / (dom_ms * 1e-3) / 1e9
    tr = traffic_table().get(f"{args.workload}:{dom.name}")
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, m, n, Rst, Col, Val)
    case_names = [c.name for c in cases]
    case_precs = sorted({c.prec for c in cases})
    forms = None
    if world == 1 and not args.no_forms:
        del cases
        torch.cuda.empty_cache()
        forms = run_forms(torch, pk)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": ",".join(case_precs), "data": "synthetic",
        "config": config_for(args, m, len(Col), case_names, world),
        "value_csr_equiv": round(value_csr_equiv, 1),
        "per_format": per,
        "roofline": {"bound": "hbm", "kernel": dom.name, "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
                     "peak_source": pk["source"], "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                     "traffic": tr, "algorithmic_bytes": int(dom.bytes)},
        "e2e": ({"value": round(job_gbs(total_bytes, world, e2e_ms), 1), "unit": "GB/s",
                 "h2d_bytes_per_step": drop["h2d_bytes_per_step"], "d2h_bytes_per_step": drop["d2h_bytes_per_step"],
                 "ms_per_step": round(e2e_ms, 4), "path": "C++ drop-in sparse_mv / sparse_mv_mixed, host "
                 "std::vector b and y (pageable), one synchronous call per case", "per_case_ms": drop["per_case_ms"]}
                if drop else {"value": None, "unit": "GB/s",
                              "error": "skipped (--no-e2e)" if args.no_e2e else "drop-in harness unavailable"}),
        "e2e_python_pinned_overlapped": {"value": round(job_gbs(total_bytes, world, e2e_ms_py), 1), "unit": "GB/s",
                                         "h2d_bytes_per_step": h2d_py, "d2h_bytes_per_step": d2h_py,
                                         "ms_per_step": round(e2e_ms_py, 4)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if forms is not None:
        line["forms"] = forms
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- added forms
def _time_ms(torch, fn, warmup=3, iters=20):
    """Median CUDA-event time of fn() on the current stream.  The calls are
    queued back to back (one synchronisation at the end), so each event pair
    brackets the device work of one call, not the host time between calls."""
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(iters)]
    torch.cuda.synchronize()
    for e0, e1 in ev:
        e0.record(st)
        fn()
        e1.record(st)
    torch.cuda.synchronize()
    return statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)


def form_precision(torch, pk):
    """The 27-point stencil on a 128^3 grid (periodic, 56,623,104 nonzeros,
    values 1 + 0.1 N(0,1)) and the 4,194,304-row power-law matrix, x U[-1,1]:
    plain fp64 against the mixed forms (fp32 or bf16 values, fp32 x/y,
    compensated fp32 row sums, fp64 carry merges) for CSR5 and HCSR, each
    precision with the parameters the autotuner picks (CSR5 sigma, HCSR block
    size).  Errors are normwise and per-row against the long-double oracle on
    the fp64 values ("vs_fp64") and on the stored (rounded) values and x
    ("vs_stored": the accumulation error alone)."""
    import oracle as O
    import rvvlasparse_b200 as R
    from rvvlasparse_b200 import autotune as AT
    from rvvlasparse_b200 import workloads as W

    def errs(y, r):
        nz = np.abs(r) > 0
        rel = np.abs(y[nz] - r[nz]) / np.abs(r[nz])
        return {"normwise": float(O.normwise_relerr(y, r)), "row_max": float(rel.max()),
                "row_median": float(np.median(rel))}

    out = {}
    for wname, gen in (("stencil27 128^3", lambda: W.stencil27(128, seed=3)),
                       ("powerlaw", lambda: W.powerlaw(N_DEFAULT, seed=1))):
        m, n, Rst, Col, Val = gen()
        nnz = len(Col)
        x = W.vector(n, 0)
        z = np.zeros(m)
        ref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, z)
        x32 = x.astype(np.float32)
        ref32 = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val.astype(np.float32)), 1.0, x32.astype(np.float64), 0.0, z)
        vbf = torch.as_tensor(Val).to(torch.bfloat16).to(torch.float64).numpy()
        refbf = O.crs_spmv_ld(O.crs(m, n, Rst, Col, vbf), 1.0, x32.astype(np.float64), 0.0, z)
        A64 = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
        A32 = A64.astype(torch.float32)
        xd64 = torch.as_tensor(x).cuda()
        xd32 = xd64.float()
        wout = {"workload": f"{wname} n={m} nnz={nnz}", "formats": {}}
        for fmt in ("csr5", "hcsr"):
            cls = R.spMtxCSR5 if fmt == "csr5" else R.spMtxHCSR
            res = {}
            for name, mdt, mixed, xd, vb, xb, rr in (("f64", None, False, xd64, 8, 8, None),
                                                     ("mixed_f32", torch.float32, True, xd32, 4, 4, ref32),
                                                     ("mixed_bf16", torch.bfloat16, True, xd32, 2, 4, refbf)):
                params = AT.tune(fmt, A64, mdt, iters=3)[0]
                M = cls()
                R.convert(M, A32 if mixed else A64, R.convertParams(**params))
                if mdt == torch.bfloat16:
                    M = M.astype(torch.bfloat16)
                y = torch.zeros(m, dtype=xd.dtype, device="cuda")
                fn = R.sparse_mv_mixed if mixed else R.sparse_mv

                def go():
                    st = fn(R.SPARSE_OPERATION_NON_TRANSPOSE, 1.0, M, R.sparse_matrix_descr(), xd, 0.0, y)
                    if st.code:
                        raise RuntimeError(f"{fmt} {name}: {st.code}")

                ms = _time_ms(torch, go)
                yh = y.double().cpu().numpy()
                b = (csr5_bytes(m, n, nnz, M.p, M.omega, M.tile_desc_len, M.num_offsets, vb, xb) if fmt == "csr5"
                     else hcsr_bytes(M, vb, xb))
                e = {"params": params, "ms": round(ms, 4), "gbs": round(b / (ms * 1e-3) / 1e9, 1),
                     "frac_of_hbm": round(b / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4),
                     "gnnz_per_s": round(nnz / (ms * 1e-3) / 1e9, 2), "vs_fp64": errs(yh, ref)}
                if rr is not None:
                    e["vs_stored"] = errs(yh, rr)
                res[name] = e
                del M
            for name in ("mixed_f32", "mixed_bf16"):
                res[name]["speedup_vs_f64"] = round(res["f64"]["ms"] / res[name]["ms"], 3)
            wout["formats"][fmt] = res
        out[wname] = wout
        del A64, A32
    return out


def form_batched(torch, pk):
    """1,024 independent matrices (n log-uniform in [1024, 65536], average
    nonzeros per row U[4, 64], Poisson rows, uniform columns, fp32 U[-1,1]),
    k in {1, 4, 8, 32} right-hand sides; autotuned; one persistent launch per
    product, replayed from a CUDA graph.  Bytes = 8*nnz + 4*(m+1) + 4*k*(n+m)
    summed over the matrices."""
    import oracle as O
    import rvvlasparse_b200 as R
    from rvvlasparse_b200 import batched as BT
    from rvvlasparse_b200 import workloads as W

    host = W.batch(1024, seed=7)
    mats = [R.spMtxCRS.from_host(m, n, Rst, Col, Val.astype(np.float32), dtype=torch.float32)
            for m, n, Rst, Col, Val in host]
    snz = sum(len(h[3]) for h in host)
    sm = sum(h[0] for h in host)
    sn = sum(h[1] for h in host)
    out = {"workload": f"1024 matrices, sum n = {sn}, sum nnz = {snz}, fp32", "k": {}}
    s = torch.cuda.Stream()
    for k in (1, 4, 8, 32):
        with torch.cuda.stream(s):
            B = BT.SpMVBatch(mats, k=k, tune=True)
            X = torch.empty(B.x_len, dtype=torch.float32, device="cuda").uniform_(-1, 1)
            Y = torch.zeros(B.y_len, dtype=torch.float32, device="cuda")
            g = B.graph(1.0, X, 0.0, Y)
            ms = _time_ms(torch, g.launch)
            byts = 8 * snz + 4 * (sm + len(mats)) + 4 * k * (sn + sm)
            # spot check: first matrix, first right-hand side
            m0, n0, R0, C0, V0 = host[0]
            xs = X[B.x_off[0]:B.x_off[1]].view(n0, k)[:, 0].double().cpu().numpy()
            ys = Y[B.y_off[0]:B.y_off[1]].view(m0, k)[:, 0].double().cpu().numpy()
            err = O.normwise_relerr(ys, O.crs_spmv_ld(O.crs(m0, n0, R0, C0, V0.astype(np.float32)), 1.0, xs, 0.0,
                                                       np.zeros(m0)))
            out["k"][str(k)] = {"ms": round(ms, 4), "gbs": round(byts / (ms * 1e-3) / 1e9, 1),
                                "frac_of_hbm": round(byts / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4),
                                "gflops": round(2 * snz * k / (ms * 1e-3) / 1e9, 1), "bytes": int(byts),
                                "tuned_ms": round(B.tuned_ms, 4), "sell_matrices": int((B.mode == 1).sum()),
                                "grid": B.grid, "tiles": B.ntiles, "spot_relerr": float(err)}
            del g
    torch.cuda.synchronize()
    return out


def form_adjoint(torch, pk):
    """y = A(v) x on a random matrix (n = 1,048,576, geometric rows of mean
    19, uniform columns, fp32 N(0,1) values): forward, dx = A^T g (the CRS
    lane-run kernel on the GPU-built transpose, A's values read through the
    permutation) and dvalues = g_i x_j (SDDMM); the transpose build is timed
    once."""
    import time as _t

    from rvvlasparse_b200 import autograd as AG
    from rvvlasparse_b200 import workloads as W

    m, n, Rst, Col, Val = W.random_rows(1 << 20, 1 << 20, "geometric", 1.0 / 19.0, "normal", seed=31)
    nnz = len(Col)
    Rd = torch.as_tensor(Rst).cuda()
    Cd = torch.as_tensor(Col).cuda()
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    P = AG.CrsPattern(m, n, Rd, Cd, torch.float32)
    torch.cuda.synchronize()
    build_ms = (_t.perf_counter() - t0) * 1e3
    v = torch.as_tensor(Val.astype(np.float32)).cuda()
    x = torch.randn(n, device="cuda")
    g = torch.randn(m, device="cuda")
    fwd = 8 * nnz + 4 * (m + 1) + 4 * n + 4 * m
    adj = 12 * nnz + 4 * (n + 1) + 4 * m + 4 * n  # A^T columns, permutation, values through it
    sdd = 8 * nnz + 4 * (m + 1) + 4 * m + 4 * n
    out = {"workload": f"random rows n={m} nnz={nnz} fp32", "transpose_build_ms": round(build_ms, 2)}
    for name, fn, b in (("forward", lambda: P.forward(v, x, 1.0), fwd), ("dx", lambda: P.adjoint_x(v, g, 1.0), adj),
                        ("dvalues", lambda: P.sddmm(g, x), sdd)):
        ms = _time_ms(torch, fn)
        out[name] = {"ms": round(ms, 4), "gbs": round(b / (ms * 1e-3) / 1e9, 1),
                     "frac_of_hbm": round(b / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4)}
    return out


def form_solver(torch, pk):
    """Conjugate gradients, then BiCGStab, on the 5-point Laplacian of a
    2048 x 2048 grid (n = 4,194,304, 20.97M nonzeros, fp64, diagonal shifted
    by 0.01): 100 iterations each (one read of r.r at the end).  Bytes per iteration = the CRS
    SpMV's (p gathered once) + the fused x/r update (reads x, r, p, q, writes
    x, r) + the p update (reads r, p, writes p)."""
    import rvvlasparse_b200 as R
    from rvvlasparse_b200 import solvers as S
    from rvvlasparse_b200 import workloads as W

    g = 2048
    m, n, Rst, Col, Val = W.laplace2d(g)
    Val = Val.copy()
    Val[Val == 4.0] += 0.01
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    b = torch.as_tensor(W.vector(n, 5)).cuda()
    iters = 100
    S.cg(A, b, rtol=0.0, max_iter=5, check_every=5)  # warm-up: analysis, scratch pool
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    _, it, rel = S.cg(A, b, rtol=0.0, max_iter=iters, check_every=iters)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / it
    byts = crs_bytes(m, n, len(Col), 8, 8) + 6 * 8 * n + 3 * 8 * n
    out = {"workload": f"laplace2d {g}^2 n={m} nnz={len(Col)} fp64", "iterations": it,
           "ms_per_iteration": round(ms, 4), "gbs": round(byts / (ms * 1e-3) / 1e9, 1),
           "frac_of_hbm": round(byts / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4), "rel_res": rel}
    # BiCGStab on the same matrix (a general solver; the matrix being SPD does
    # not change its work): 2 SpMVs, the p / s / x-r passes and three dot
    # passes per iteration = 2 SpMV + 18 n values
    S.bicgstab(A, b, rtol=0.0, max_iter=3, check_every=3)
    torch.cuda.synchronize()
    e0.record()
    _, itb, relb, bd = S.bicgstab(A, b, rtol=0.0, max_iter=iters, check_every=iters)
    e1.record()
    torch.cuda.synchronize()
    msb = e0.elapsed_time(e1) / max(itb, 1)
    bb = 2 * crs_bytes(m, n, len(Col), 8, 8) + 18 * 8 * n
    out["bicgstab"] = {"iterations": itb, "ms_per_iteration": round(msb, 4), "gbs": round(bb / (msb * 1e-3) / 1e9, 1),
                       "frac_of_hbm": round(bb / (msb * 1e-3) / 1e9 / pk["hbm_gbs"], 4), "rel_res": relb,
                       "breakdown": bd}
    return out


def run_forms(torch, pk):
    out = {}
    for name, fn in (("precision", form_precision), ("batched", form_batched), ("adjoint", form_adjoint),
                     ("solver", form_solver)):
        try:
            out[name] = fn(torch, pk)
        except Exception as e:  # reported, never hidden
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    return out


def e2e_time(cases, args, torch):
    """Per step and case: pinned host x -> device, SpMV, device y -> pinned
    host.  Copies in, products and copies out run on three streams, so case
    i+1's x crosses while case i computes and case i-1's y comes back (a
    case's device x is refilled only after its product read it, its device y
    overwritten only after the copy out read it)."""
    stream = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    hx = [torch.empty(c.x.numel(), dtype=c.vt, pin_memory=True).copy_(c.x.cpu()) for c in cases]
    hy = [torch.empty(c.y.numel(), dtype=c.vt, pin_memory=True) for c in cases]
    h2d = sum(h.numel() * h.element_size() for h in hx)
    d2h = sum(h.numel() * h.element_size() for h in hy)
    nc = len(cases)
    x_free = [None] * nc   # the product of the case's previous step has read x
    y_free = [None] * nc   # the copy out of the case's previous step has read y

    def one():
        for i, (c, x, y) in enumerate(zip(cases, hx, hy)):
            ev_in = torch.cuda.Event()
            with torch.cuda.stream(s_in):
                if x_free[i] is not None:
                    s_in.wait_event(x_free[i])
                c.x.copy_(x, non_blocking=True)
                ev_in.record(s_in)
            stream.wait_event(ev_in)
            if y_free[i] is not None:
                stream.wait_event(y_free[i])
            c.launch()
            ev_prod = torch.cuda.Event()
            ev_prod.record(stream)
            x_free[i] = ev_prod
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_prod)
                y.copy_(c.y, non_blocking=True)
                ev_out = torch.cuda.Event()
                ev_out.record(s_out)
            y_free[i] = ev_out

    for _ in range(2):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    for _ in range(args.steps):
        one()
    for sx in (s_in, s_out):
        ev = torch.cuda.Event()
        ev.record(sx)
        stream.wait_event(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / args.steps, h2d, d2h


def e2e_dropin(args, case_names, local: int):
    """Runs the drop-in harness (rvvlasparse_b200/_build/bench_dropin) on
    this rank's GPU; returns per-step ms (the sum of the per-case medians of
    one synchronous sparse_mv each), bytes copied per step and per-case ms,
    or None when the harness is missing or fails (the error is printed)."""
    exe = os.path.join(ROOT, "rvvlasparse_b200", "_build", "bench_dropin")
    if not os.path.exists(exe):
        print("e2e: drop-in harness not built", file=sys.stderr)
        return None
    env = dict(os.environ)
    vis = env.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = vis.split(",")[local] if vis else str(local)
    cmd = [exe, args.workload, str(args.n), args.formats, args.precisions, str(args.steps), str(max(args.warmup, 3))]
    res = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if res.returncode != 0:
        print(f"e2e: drop-in harness failed: {res.stderr[-2000:]}", file=sys.stderr)
        return None
    d = json.loads(res.stdout.strip().splitlines()[-1])
    per = {k: v["ms"] for k, v in d["cases"].items()}
    if sorted(per) != sorted(case_names):
        print(f"e2e: harness cases {sorted(per)} differ from {sorted(case_names)}", file=sys.stderr)
        return None
    return {"ms_per_step": sum(per.values()), "h2d_bytes_per_step": d["h2d_bytes_per_step"],
            "d2h_bytes_per_step": d["d2h_bytes_per_step"], "per_case_ms": {k: round(v, 4) for k, v in per.items()}}


# ----------------------------------------------------------------- CPU side
def cpu_cases(m, n, Rst, Col, Val, formats, precs):
    import oracle as O

    out = []
    crs = {}
    lay = {}

    def layout(fmt, dt, make):
        # one oracle build per format (f64); the f32 layout casts its values
        if fmt not in lay:
            lay[fmt] = make(crs[np.float64] if np.float64 in crs else O.crs(m, n, Rst, Col, Val.astype(np.float64)))
        return lay[fmt] if dt == np.float64 else lay[fmt].astype(dt)

    for fmt in formats:
        for p in precs:
            if p.startswith("mixed") and fmt not in MIXED:
                continue
            # the reference has no mixed-precision kernels: its fp32 kernel
            # stands in for the mixed forms
            dt = np.float64 if p == "f64" else np.float32
            vb, xb = (8, 8) if p == "f64" else (4, 4)
            if dt not in crs:
                crs[dt] = O.crs(m, n, Rst, Col, Val.astype(dt))
            A = crs[dt]
            if fmt == "crs":
                out.append((f"crs_{p}", O.ref_crs(A), crs_bytes(m, n, len(Col), vb, xb), dt))
            elif fmt == "hcsr":
                h = O.ref_hcsr_convert(A)
                nb1 = int(h["b_m"]) * int(h["b_n"]) + 1
                b = len(Col) * (vb + 2) + len(h["row_ptr"]) * 4 + nb1 * 8 + n * xb + m * xb
                out.append((f"hcsr_{p}", O.ref_hcsr(h), b, dt))
            elif fmt == "csr5":
                # the reference has CSR5 only as RVV intrinsics: time the
                # oracle's single-threaded restatement of that kernel
                c5 = layout("csr5", dt, lambda a: O.build_csr5(a, 32, 16))
                b = csr5_bytes(m, n, len(Col), int(c5["p"]), 32, int(c5["tile_desc_len"]), int(c5["num_offsets"]),
                               vb, xb)
                out.append((f"csr5_{p}", O.OracleMatrix(c5), b, dt))
            elif fmt == "sell":
                sb = layout("sell", dt, lambda a: O.build_sell(a, 32, 256))
                b = len(sb["vVal"]) * (vb + 4) + int(sb["cnt_b"]) * 16 + m * 4 + n * xb + m * xb
                out.append((f"sell_{p}", O.ref_sell(sb), b, dt))
            elif fmt == "lav":
                lb = layout("lav", dt, lambda a: O.build_lav(a, 8, 0.2, max(n, 1)))
                L, cc, ns, st = 8, int(lb["chunk_count"]), int(lb["segment_count"]), len(lb["mask"])
                b = (st * L * (vb + 4) + st * 2 + ns * cc * L * 4 + (2 * cc + 1) * ns * 4 + (ns + 1) * 8
                     + crs_bytes(m, n, int(lb["sparse_nz"]), vb, xb))
                out.append((f"lav_{p}", O.ref_lav(lb), b, dt))
            elif fmt == "cvr":
                # the reference kernel runs one OpenMP thread per CVR thread block
                cb = layout("cvr", dt, lambda a: O.build_cvr(a, 8, O.ref_num_threads()))
                b = len(cb["vPack_vec_vals"]) * (vb + 4) + len(cb["vPack_vec_record"]) * 4 \
                    + len(cb["writeback_pos_record"]) * 4 + n * xb + m * xb
                out.append((f"cvr_{p}", O.ref_cvr(cb), b, dt))
            elif fmt in ("vnec", "vhcc"):
                # RVV-only in the reference: the oracle's single-threaded port
                if fmt == "vnec":
                    ob = layout("vnec", dt, lambda a: O.build_vnec(a, 16, -1))
                    b = crs_bytes(m, n, len(Col), vb, xb) + 16 * 16
                else:
                    ob = layout("vhcc", dt, lambda a: O.build_vhcc(a, 16, 8))
                    b = (len(ob["vals_arr"]) * (vb + 4) + len(ob["veceor_ptr"]) * 4 + len(ob["scan_mask"])
                         + len(ob["row_arr"]) * 4 + 16 * 40 + n * xb + m * xb)
                out.append((f"{fmt}_{p}", O.OracleMatrix(ob), b, dt))
    return out


def cpu_baseline(args, m, n, Rst, Col, Val):
    """Reference scalar/OpenMP SpMV timed on this host (bounded sample)."""
    import oracle as O

    if not O.ref_available():
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference library not built"}
    cases = cpu_cases(m, n, Rst, Col, Val, args.formats.split(","), args.precisions.split(","))
    x = np.random.default_rng(0).uniform(-1, 1, n)
    times = {}
    per = {}
    for name, mat, b, dt in cases:
        t = mat.time(1.0, x.astype(dt), 0.0, args.cpu_iters)
        times[name] = (b, t)
        per[name] = round(b / t / 1e9, 2)
    parts = cpu_parts(times, O.ref_num_threads())
    head = parts.get("reference_library") or parts.get("oracle_port")
    return {"value": head["value"], "unit": "GB/s", "cores": head["cores"], "kind": head["kind"],
            "per_format": per, "parts": parts,
            "sample": f"median of {args.cpu_iters} sparse_mv calls per case on the full matrix; value = the "
                      f"reference library's own formats ({', '.join(head['cases'])}) on all host threads; "
                      f"mixed forms timed as the reference fp32 kernels"}


def cpu_parts(times: dict, ref_threads: int) -> dict:
    """Aggregate CPU GB/s in two parts: the reference library's own C++
    formats (OpenMP, all host threads) and the RVV-only formats, timed as the
    oracle's single-threaded restatements.  times: case -> (bytes, seconds)."""
    out = {}
    for part, sel, cores, kind in (("reference_library", True, ref_threads, "reference"),
                                   ("oracle_port", False, 1, "port")):
        names = [k for k in times if (k.split("_")[0] in REF_LIBRARY_FORMATS) == sel]
        if not names:
            continue
        b = sum(times[k][0] for k in names)
        t = sum(times[k][1] for k in names)
        out[part] = {"value": round(b / t / 1e9, 2), "unit": "GB/s", "cores": cores, "kind": kind, "cases": names}
    return out


def run_sharded(args):
    """--sharded: one product of the whole matrix split across the ranks
    (rvvlasparse_b200.distributed.RowShardedCRS: nonzero-balanced row ranges,
    the x halo exchanged over NCCL while the diagonal block multiplies) per
    step, CRS fp64.  Strong scaling: the matrix is the same at every N;
    value = the whole product's CRS bytes / the slowest rank's step time."""
    import datetime

    import torch
    import torch.distributed as dist

    import rvvlasparse_b200 as R
    from rvvlasparse_b200.distributed import RowShardedCRS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl" if world > 1 else "gloo", timeout=datetime.timedelta(seconds=120),
                            **({} if world > 1 else {"init_method": "tcp://127.0.0.1:0", "rank": 0,
                                                     "world_size": 1}))
    try:
        lib = R.load()
        m, n, Rst, Col, Val = workload(args.workload, args.n)
        S = RowShardedCRS(m, n, Rst, Col, Val, device="cuda", exchange=args.exchange)
        x = torch.as_tensor(np.random.default_rng(0).uniform(-1, 1, n)[S.r0:S.r1].copy()).cuda()
        y = torch.zeros(S.local_rows, dtype=torch.float64, device="cuda")
        for _ in range(max(args.warmup, 3)):
            S.spmv(x, 1.0, 0.0, y)
        torch.cuda.synchronize()
        dist.barrier()
        l0 = lib.rvvla_kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            S.spmv(x, 1.0, 0.0, y)
        e1.record()
        torch.cuda.synchronize()
        launches = lib.rvvla_kernel_launch_count() - l0
        dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda") if world > 1 else \
            e0.elapsed_time(e1) / args.steps
        byts = crs_bytes(m, n, len(Col), 8, 8)
        exchanged = S.exchanged_per_spmv
    finally:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": round(byts / (ms * 1e-3) / 1e9, 1), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload} n={m} nnz={len(Col)}", "cases": ["crs_f64_row_sharded"],
                       "parallelism": f"rows{world}", "exchange": args.exchange,
                       "x_entries_sent_by_rank0_per_step": exchanged},
            "gpu_launches": int(launches)}), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference scalar library not built (make -C oracle ref)"}))
        return
    # the matrix comes from the oracle's copy of the generators: this arm
    # loads no part of the CUDA library
    m, n, Rst, Col, Val = workload(args.workload, args.n, cpu_only=True)
    precs = args.precisions.split(",")
    cases = cpu_cases(m, n, Rst, Col, Val, args.formats.split(","), precs)
    x = np.random.default_rng(0).uniform(-1, 1, n)
    for _ in range(max(args.warmup, 1)):
        for name, mat, b, dt in cases:
            mat.time(1.0, x.astype(dt), 0.0, 1)
    step_s = {name: [] for name, *_ in cases}
    for _ in range(args.steps):
        for name, mat, b, dt in cases:
            step_s[name].append(mat.time(1.0, x.astype(dt), 0.0, 1))
    times = {name: (b, statistics.median(step_s[name])) for name, mat, b, dt in cases}
    parts = cpu_parts(times, O.ref_num_threads())
    head = parts.get("reference_library") or parts.get("oracle_port")
    # value: the reference library's own formats only; the single-threaded
    # restatements of its RVV-only formats are reported beside it
    ms = sum(times[k][1] for k in head["cases"]) * 1e3
    value = head["value"]
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    line = {
        # n_gpus: the N this arm was launched with (its work runs on the host cores)
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": ",".join(sorted(set(precs))), "data": "synthetic",
        "config": config_for(args, m, len(Col), [c[0] for c in cases], world),
        "value_basis": "reference library formats only (" + ", ".join(head["cases"]) + "); per-case median of "
                       "the timed steps",
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": head["cores"], "kind": head["kind"],
                         "parts": parts,
                         "sample": "full matrix, one sparse_mv per case per step; reference library on all host "
                                   "threads (OpenMP); mixed forms timed as the reference fp32 kernels"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 50 on the GPU arm, so each case's median is over 50 launches; "
                         "20 on the reference arm, whose steps take seconds)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="powerlaw", choices=["powerlaw", "stencil", "laplace"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--formats", default="crs,hcsr,csr5,sell,lav,vnec,vhcc,cvr")
    ap.add_argument("--precisions", default="f64,f32,mixed")
    ap.add_argument("--cpu-iters", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sharded", action="store_true",
                    help="time one row-sharded CRS fp64 product across the ranks per step (strong scaling) "
                         "instead of a replica of every case per rank")
    ap.add_argument("--exchange", default="halo", choices=["halo", "allgather"],
                    help="x exchange of --sharded")
    ap.add_argument("--params", default="",
                    help='convertParams per format over the defaults, e.g. "hcsr:R=2000,C=65536;csr5:sigma=24"')
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the drop-in end-to-end leg (a child process; for profiling runs)")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the precision (stencil), batched and adjoint forms reported under 'forms'")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.impl == "reference" else 50
    if args.steps < 1:
        ap.error("--steps must be >= 1")
    if args.impl == "reference":
        run_reference(args)
    elif args.sharded:
        run_sharded(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
