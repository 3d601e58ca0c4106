"""The drop-in CLIs on the GPU against rows the REFERENCE binaries wrote.

* Every golden case (tests/golden/case*.raw|.dat with the argv in
  golden.json, rows written by the reference's own builds of
  LMB3d/lbm3d-perm.cpp and LMB2d/main.cpp + lbm.cpp) goes through
  cli3d.main / cli2d.main, the code behind bin/lbm3d-perm and bin/lbm2d-perm,
  and the appended CSV row is compared with the reference's row
  (writers: LMB3d/lbm3d-perm.cpp:574-615, LMB2d/main.cpp:383-411).
* Every call the reference's check scripts made (scripts/validate_solver3d.py
  and scripts/rotation_covariance3d.py, run unchanged; recorded by
  tests/golden/scripts_chain.py) is replayed through cli3d.main the same way.

The drop-in's default path is FP64.  The reference is built with -ffast-math,
so rows agree to roundoff, not bit for bit: fluxes and tensor entries within
5e-9 relative (the FP64 bar is 1e-8), step counts, convergence flags, header
and exit codes exactly.  A blocked direction (no flow possible, the flux is
roundoff ~1e-17) stops at a step decided by roundoff, so for it the test
checks that the drop-in's flux is zero instead of comparing steps.
"""
import contextlib
import io
import json
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

from flow_anizotropy_b200 import cli2d, cli3d
from flow_anizotropy_b200 import tensor as T
from rowcheck import close_row

G = Path(__file__).resolve().parent / "golden"
META = json.loads((G / "golden.json").read_text())
sys.path.insert(0, str(G))
import scripts_chain as SC  # noqa: E402

RTOL64 = 5e-9
TAGS = ("fx", "fy", "fz")


def _blocked(ref_row):
    """Forcing directions whose reference flux is roundoff (no pore path)."""
    cols = T.header3().split(",")
    val = dict(zip(cols, ref_row.split(",")))
    q = {t: np.array([float(val[f"q{c}_{t}"]) for c in "xyz"]) for t in TAGS}
    qmax = max(np.abs(v).max() for v in q.values())
    return [t for t in TAGS if np.abs(q[t]).max() < 1e-10 * qmax], qmax


def _compare3(mine, ref):
    blocked, qmax = _blocked(ref)
    skip = set()
    for t in blocked:
        skip |= {f"steps_{t}", f"conv_{t}"} | {f"q{c}_{t}" for c in "xyz"} | {f"se_q{c}_{t}" for c in "xyz"}
    close_row(mine, ref, T.header3(), rtol=RTOL64, skip=skip)
    cols = T.header3().split(",")
    got = dict(zip(cols, mine.split(",")))
    for t in blocked:
        assert max(abs(float(got[f"q{c}_{t}"])) for c in "xyz") < 1e-10 * qmax, t
    return blocked


def _run_cli(mod, argv, cwd):
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        with _chdir(cwd):
            rc = mod.main(argv)
    return rc, out.getvalue()


@contextlib.contextmanager
def _chdir(d):
    import os
    old = os.getcwd()
    os.chdir(d)
    try:
        yield
    finally:
        os.chdir(old)


@pytest.mark.gpu
@pytest.mark.parametrize("name", [n for n in META if n.startswith("case3d")])
def test_cli3d_row_equals_reference_row(gpu, name, tmp_path):
    m = META[name]
    shutil.copy(G / f"{name}.raw", tmp_path / f"{name}.raw")
    argv = [f"{name}.raw", "out.csv", "--quiet"] + m["argv"]
    if m["binary"].endswith("tau0.8"):
        argv += ["--tau", "0.8"]          # the reference's tau = 0.8 build
    rc, stdout = _run_cli(cli3d, argv, tmp_path)
    mine = (tmp_path / "out.csv").read_text().splitlines()
    ref = (G / f"{name}.csv").read_text().splitlines()
    assert mine[0] == ref[0] == T.header3()
    blocked = _compare3(mine[1], ref[1])
    if not blocked:
        assert rc == m["rc"]
    if "--validate" in m["argv"]:
        meas = [ln for ln in m["stdout"] if "measured" in ln][0]
        got = [ln for ln in stdout.splitlines() if "measured" in ln][0]
        want = [float(v) for v in meas.split("(")[1].rstrip(")").split(",")]
        have = [float(v) for v in got.split("(")[1].rstrip(")").split(",")]
        np.testing.assert_allclose(have, want, rtol=1e-5)     # printed to 6 digits


@pytest.mark.gpu
def test_cli2d_row_equals_reference_row(gpu, tmp_path):
    name = "case2d_a"
    m = META[name]
    shutil.copy(G / f"{name}.dat", tmp_path / f"{name}.dat")
    rc, stdout = _run_cli(cli2d, [f"{name}.dat", "out.csv", "--quiet"] + m["argv"], tmp_path)
    assert rc == m["rc"]
    mine = (tmp_path / "out.csv").read_text().splitlines()
    ref = (G / f"{name}.csv").read_text().splitlines()
    assert mine[0] == ref[0] == T.header2()
    # the 2D path computes in the reference's FP32 arithmetic; only the FP64
    # flux sums can differ in the last digits
    close_row(mine[1], ref[1], T.header2(), rtol=1e-9)
    meas = [ln for ln in m["stdout"] if "measured" in ln][0]
    got = [ln for ln in stdout.splitlines() if "measured" in ln][0]
    assert got == meas


CALLS = json.loads((SC.FIX / "invocations.json").read_text()) if (SC.FIX / "invocations.json").exists() else []


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(CALLS)))
def test_reference_script_calls_through_dropin(gpu, i, tmp_path):
    """One call that validate_solver3d.py / rotation_covariance3d.py made to
    the reference binary, made again to the drop-in: same row, same exit code."""
    c = CALLS[i]
    (tmp_path / c["filename"]).write_bytes(SC.load_raw_bytes(c["sha"]))
    rc, _ = _run_cli(cli3d, [c["filename"], "out.csv"] + c["opts"], tmp_path)
    mine = (tmp_path / "out.csv").read_text().splitlines()
    assert mine[0] == T.header3()
    ref = c["row"].split(",", 1)
    blocked = _compare3(mine[1], c["filename"] + "," + ref[1])
    if not blocked:
        assert rc == c["rc"]
