"""Host-side pieces of bench.py (no GPU): the roofline byte model, the
traffic figure scaled from the recorded ncu capture, the reference row, the
per-k_ij error matrix, the clock-sample summary, and the command line."""
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


def test_profiled_traffic_scaled_from_the_recorded_capture(tmp_path, monkeypatch):
    rec = {"fp16": {"variant": 7, "dram_bytes_per_update": 70.0, "command": "ncu ..."}}
    f = tmp_path / "traffic.json"
    f.write_text(__import__("json").dumps(rec))
    monkeypatch.setattr(bench, "TRAFFIC", f)
    assert bench.profiled_traffic("fp16", 7, 1000.0) == 70_000.0
    assert bench.profiled_traffic("fp16", 8, 1000.0) is None        # another kernel variant: not this capture
    assert bench.profiled_traffic("fp32", 7, 1000.0) is None
    # several captured variants of one precision
    f.write_text(__import__("json").dumps({"bf16": [{"variant": 150, "dram_bytes_per_update": 61.0},
                                                    {"variant": 71, "dram_bytes_per_update": 60.0}]}))
    assert bench.profiled_traffic("bf16", 71, 10.0) == 600.0
    assert bench.profiled_traffic("bf16", 150, 10.0) == 610.0
    assert bench.profiled_traffic("bf16", 69, 10.0) is None
    monkeypatch.setattr(bench, "TRAFFIC", tmp_path / "absent.json")
    assert bench.profiled_traffic("fp16", 7, 1000.0) is None


def test_recorded_traffic_within_the_algorithmic_bytes():
    """The recorded captures move no more DRAM bytes per update than the
    algorithmic ones (populations read and written once): no wasted re-reads."""
    import json
    if not bench.TRAFFIC.exists():
        return
    for prec, recs in json.loads(bench.TRAFFIC.read_text()).items():
        if prec.startswith("_"):
            continue
        alg = bench.BYTES_PER_UPDATE[prec] + 1.0 / 8 / 0.45
        for rec in (recs if isinstance(recs, list) else [recs]):
            assert 0 < rec["dram_bytes_per_update"] <= 1.05 * alg, (prec, rec)
            assert "ncu" in rec["command"]


def test_reference_row_of_the_workload():
    ref = bench.reference_row()
    if ref is None:
        return
    assert len(ref["steps"]) == 3 and all(s > 0 for s in ref["steps"])
    assert ref["K"].shape == (3, 3) and (np.diag(ref["K"]) > 0).all()


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
    m = np.array(e["matrix"])
    assert m.shape == (3, 3) and abs(m[0, 0] - 1e-6) < 1e-12 and abs(m[0, 1] - 1e-8) < 1e-14
    assert m[1, 1] == 0 and m[2, 0] == 0


def test_command_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload", "--serve-precision", "--serve-variant",
                 "--group2d", "--serve-seconds", "--large-steps", "--count", "--variant", "--structure"):
        assert flag in out.stdout, flag
