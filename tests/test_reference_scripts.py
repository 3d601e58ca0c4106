"""The reference's own solver checks, run unchanged, on the drop-in's output.

scripts/validate_solver3d.py and scripts/rotation_covariance3d.py take the
solver executable as --solver and judge it by the CSV rows it appends.  Here
they run unchanged against a --solver stub that answers each call with the
row, exit code and stdout the drop-in (bin/lbm3d-perm, i.e. cli3d on liblbm)
produced on a B200 for that exact structure and argv
(tests/golden/scripts/shim_rows.json, written by
`tests/golden/scripts_chain.py shim-rows` from the calls the same scripts made
to the reference binary).  The scripts' verdict must be PASSED with exit 0,
as it was for the reference binary (tests/golden/scripts/scripts.json).

Needs the reference's scripts (REF, default /root/reference); skipped where
they are absent.  tests/test_gpu_dropin.py checks on the GPU that the drop-in
still writes those rows.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

G = Path(__file__).resolve().parent / "golden"
FIX = G / "scripts"
REF = Path(os.environ.get("REF", "/root/reference"))
ROWS = FIX / "shim_rows.json"
ROOT = G.parent.parent

pytestmark = [
    pytest.mark.skipif(not (REF / "scripts" / "validate_solver3d.py").exists(),
                       reason="reference scripts not present"),
    pytest.mark.skipif(not ROWS.exists(), reason="no recorded drop-in rows"),
]

SCRIPTS = json.loads((FIX / "scripts.json").read_text()) if (FIX / "scripts.json").exists() else {}


def _stub(tmp_path):
    stub = tmp_path / "lbm3d-perm"
    stub.write_text(f"#!/bin/sh\nexec {sys.executable} {G / 'scripts_chain.py'} replay \"$@\"\n")
    stub.chmod(0o755)
    return stub


def test_every_recorded_call_has_a_dropin_row():
    calls = json.loads((FIX / "invocations.json").read_text())
    rows = json.loads(ROWS.read_text())
    assert [(c["sha"], c["opts"]) for c in calls] == [(r["sha"], r["opts"]) for r in rows]
    assert all(r["row"] is not None for r in rows)


@pytest.mark.parametrize("name", sorted(SCRIPTS))
def test_reference_script_passes_on_dropin(name, tmp_path):
    argv = SCRIPTS[name]["argv"]
    env = dict(os.environ, SCRIPTS_CHAIN_ROWS=str(ROWS), PYTHONPATH=str(ROOT), PYTHONDONTWRITEBYTECODE="1")
    p = subprocess.run([sys.executable, str(REF / argv[0]), "--solver", str(_stub(tmp_path))] + argv[1:],
                       cwd=str(REF), env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    verdict = [ln for ln in p.stdout.splitlines() if "PASSED" in ln or "FAILED" in ln]
    assert verdict and verdict[-1].endswith("PASSED"), p.stdout[-3000:]
