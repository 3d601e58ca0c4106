"""Host-side pieces of bench.py (no GPU): the roofline byte model, the
traffic figures read from the committed ncu summaries, the clock-sample
summary, and the command line."""
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_algorithmic_bytes_model():
    npore, nvox = 943_600, 128 ** 3
    assert bench.alg_bytes_per_dir_step("fp32", npore, nvox) == npore * 2 * 19 * 4 + nvox / 8
    assert bench.alg_bytes_per_dir_step("fp16", npore, nvox) == npore * 2 * 19 * 2 + nvox / 8
    assert bench.alg_bytes_per_dir_step("fp64", npore, nvox) == npore * 2 * 19 * 8 + nvox / 8
    assert bench.alg_bytes_per_dir_step("md32", npore, nvox) == 21.0 * nvox + 20.0 * npore


def test_profiled_traffic_read_from_profiles():
    for prec in ("fp32", "fp16", "md32"):
        v = bench.profiled_traffic(prec)
        assert v is not None and 1e8 < v < 1e9, (prec, v)
        alg = 3 * bench.alg_bytes_per_dir_step(prec, 943_600, 128 ** 3)
        if prec != "md32":
            # the population kernels move no more DRAM bytes per launch than
            # the algorithmic bytes of three directions: no wasted re-reads
            assert v <= alg, (prec, v, alg)
        else:
            # the dense moment form re-reads the halo rows L2 does not keep
            # (its summary says so): within 2x of its algorithmic bytes
            assert v <= 2 * alg, (prec, v, alg)
    assert bench.profiled_traffic("no-such-path") is None


def test_clock_summary(tmp_path):
    c = bench.Clocks(0)
    f = open(tmp_path / "clk.csv", "w+")
    f.write("0, 1965, 1965, 900.5, 0x0, Not Active, Not Active, Not Active, Not Active, 3996\n")
    f.write("0, 1845, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active, 3996\n")
    f.write("0, 1905, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active, 3996\n")
    f.write("garbage line\n")
    c.p, c.f = object(), f
    s = c.summary()
    assert s["sm_mhz"] == 1905 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["mem_mhz"] == 3996 and s["power_w"] == 990.0
    assert s["reasons"] == ["sw_power_cap"]


def test_k_errors_relative_to_fp64():
    K64 = np.diag([2.0, 3.0, 4.0])
    K = K64.copy()
    K[0, 0] *= 1 + 1e-6
    K[0, 1] = K[1, 0] = 4e-8
    e = bench.k_errors(K, K64)
    assert abs(e["max_rel_diag"] - 1e-6) < 1e-12
    assert abs(e["max_offdiag_over_kmax"] - 1e-8) < 1e-14


def test_command_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload", "--serve-precision", "--serve-variant",
                 "--group2d"):
        assert flag in out.stdout, flag
