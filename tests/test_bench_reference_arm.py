"""CPU: the bench's reference arm.  It times the reference's own CPU code
and must not load the CUDA library; its configuration must equal the GPU
arm's; its headline value covers the reference library's own formats, with
the oracle's single-threaded restatements of the RVV-only formats reported
beside it.  The oracle's copy of the workload generators gives the same bits
as the library's."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_generators_equal_library_generators():
    from rvvlasparse_b200 import workloads as W

    for a, b in ((O.gen_powerlaw(50000, seed=1), W.powerlaw(50000, seed=1)),
                 (O.gen_stencil27(12, seed=3), W.stencil27(12, seed=3)), (O.gen_laplace2d(40), W.laplace2d(40))):
        assert a[:2] == b[:2]
        for x, y in zip(a[2:], b[2:]):
            assert np.array_equal(x, y)
    assert np.array_equal(O.gen_vector(5000, 7), W.vector(5000, 7))


def test_config_is_shared_by_both_arms():
    sys.path.insert(0, ROOT)
    import bench

    class A:
        workload = "laplace"

    a = bench.config_for(A, 10, 20, ["crs_f64"], 1)
    assert a == bench.config_for(A, 10, 20, ["crs_f64"], 1)
    assert set(a) == {"workload", "cases", "alpha", "beta", "parallelism", "l2"}


def test_cpu_parts_split_reference_library_and_ports():
    sys.path.insert(0, ROOT)
    import bench

    times = {"crs_f64": (10e9, 1.0), "hcsr_f64": (10e9, 1.0), "csr5_f64": (10e9, 5.0), "vhcc_f32": (1e9, 1.0)}
    p = bench.cpu_parts(times, 16)
    assert p["reference_library"]["value"] == 10.0 and p["reference_library"]["cores"] == 16
    assert p["reference_library"]["cases"] == ["crs_f64", "hcsr_f64"]
    assert p["oracle_port"]["value"] == round(11e9 / 6.0 / 1e9, 2) and p["oracle_port"]["cores"] == 1


@pytest.mark.skipif(not O.ref_available(), reason="reference scalar library not built (oracle/_ref)")
def test_reference_arm_loads_no_cuda_library():
    code = (
        "import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'laplace', "
        "'--steps', '1', '--warmup', '1']; "
        "runpy.run_path('bench.py', run_name='__main__'); "
        "maps = open('/proc/self/maps').read(); "
        "print('LOADED', 'librvvla_b200' in maps, 'libcuda' in maps)")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(ln for ln in lines if ln.startswith("{")))
    assert line["impl"] == "reference" and line["value"] > 0
    assert "reference_library" in line["cpu_baseline"]["parts"]
    assert all(c.split("_")[0] in ("crs", "hcsr", "sell", "lav", "cvr")
               for c in line["cpu_baseline"]["parts"]["reference_library"]["cases"])
    assert lines[-1] == "LOADED False False"


def test_params_override_parses_and_is_recorded():
    """--params "fmt:key=value,...;fmt2:..." becomes per-format convertParams
    (ints stay ints, decimals become floats) and is recorded in the config."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    p = bench.parse_params("hcsr:R=2000,C=65536;lav:T=0.2,segment_len=40000; ;csr5:sigma=24")
    assert p == {"hcsr": {"R": 2000, "C": 65536}, "lav": {"T": 0.2, "segment_len": 40000}, "csr5": {"sigma": 24}}
    assert isinstance(p["hcsr"]["R"], int) and isinstance(p["lav"]["T"], float)
    assert bench.parse_params("") == {}
    args = argparse.Namespace(workload="powerlaw", params="hcsr:R=100")
    cfg = bench.config_for(args, 10, 20, ["hcsr_f64"], 1)
    assert cfg["params"] == {"hcsr": {"R": 100}}
    assert "params" not in bench.config_for(argparse.Namespace(workload="powerlaw", params=""), 10, 20, [], 1)
