"""The reference's own solver checks, run UNCHANGED against the drop-in.

The reference validates a solver build with two scripts that take the solver
executable as ``--solver``: ``scripts/validate_solver3d.py`` (analytic slit,
h^-2 error scaling, k_zz = 0, off-diagonals) and
``scripts/rotation_covariance3d.py`` (K' = P K P^T under the five axis
permutations).  Those scripts live with the reference, which the GPU machine
does not have, and the drop-in needs a GPU, which the reference's machine
does not have.  So the chain runs in three legs, each a subcommand here:

  record      (needs the reference sources and oracle/_ref/lbm3d-perm)
              runs both scripts unchanged with --solver pointing at a proxy
              that forwards every call to the reference binary and records
              the structure it was given (bit-packed, by SHA-256), its options,
              exit code, stdout and the CSV row it appended.  Writes
              tests/golden/scripts/ (invocations.json, structures .npz,
              scripts.json with the scripts' own output).
  shim-rows   (on a GPU) replays every recorded invocation through the
              drop-in (flow_anizotropy_b200.cli3d, the code behind
              bin/lbm3d-perm) and writes its rows, exit codes and stdout to a
              JSON file (committed as tests/golden/scripts/shim_rows.json).
  replay      the --solver stub for the unchanged scripts: it answers each
              call with the drop-in's recorded output for that structure and
              those options (appending the header on an empty file, as the
              solver does), so the scripts' own checks run on the drop-in's
              rows.  tests/test_reference_scripts.py drives it.

    python tests/golden/scripts_chain.py record
    python tests/golden/scripts_chain.py shim-rows OUT.json      (GPU)
"""
from __future__ import annotations

import contextlib
import hashlib
import io
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
FIX = HERE / "scripts"
REF = Path(os.environ.get("REF", "/root/reference"))

# script, argv after --solver, timeout (s)
SCRIPTS = {
    "validate_solver3d": (["scripts/validate_solver3d.py"], 3600),
    "rotation_covariance3d": (["scripts/rotation_covariance3d.py", "--workers", "6"], 7200),
}


def _sha(buf: bytes) -> str:
    return hashlib.sha256(buf).hexdigest()


def _key(sha: str, opts) -> str:
    return sha + " " + " ".join(opts)


def _store_structure(buf: bytes, sha: str) -> None:
    """Bit-packed copy of a .raw (header + packbits payload) under FIX."""
    path = FIX / f"{sha[:16]}.npz"
    if path.exists():
        return
    hdr = np.frombuffer(buf[:12], dtype="<i4")
    vox = np.frombuffer(buf, dtype=np.uint8, offset=12)
    np.savez_compressed(path, dims=hdr, bits=np.packbits(vox))


def load_raw_bytes(sha: str) -> bytes:
    """The exact .raw bytes of a recorded structure."""
    z = np.load(FIX / f"{sha[:16]}.npz")
    dims = z["dims"].astype("<i4")
    n = int(np.prod(dims.astype(np.int64)))
    vox = np.unpackbits(z["bits"])[:n].astype(np.uint8)
    buf = dims.tobytes() + vox.tobytes()
    assert _sha(buf) == sha, "recorded structure does not reproduce its hash"
    return buf


def _appended_row(csv: Path, before: int):
    """(header written?, the row the solver appended) of a CSV that had `before` bytes."""
    if not csv.exists():
        return False, None
    text = csv.read_bytes()[before:].decode()
    lines = [ln for ln in text.splitlines() if ln]
    if not lines:
        return False, None
    return before == 0 and len(lines) > 1, lines[-1]


# ------------------------------------------------------------------- proxy --
def proxy(argv) -> int:
    """--solver for `record`: run the reference binary, log the call."""
    from oracle import oracle as O
    exe = O.ref_binary("lbm3d-perm")
    structure, csv, opts = argv[0], Path(argv[1]), argv[2:]
    buf = Path(structure).read_bytes()
    sha = _sha(buf)
    _store_structure(buf, sha)
    before = csv.stat().st_size if csv.exists() else 0
    p = subprocess.run([str(exe), structure, str(csv)] + opts, capture_output=True, text=True)
    hdr, row = _appended_row(csv, before)
    rec = dict(sha=sha, opts=opts, rc=p.returncode, stdout=p.stdout, stderr=p.stderr[-400:],
               row=row, filename=structure)
    line = json.dumps(rec) + "\n"
    with open(os.environ["SCRIPTS_CHAIN_LOG"], "a") as fh:
        fh.write(line)
    sys.stdout.write(p.stdout)
    sys.stderr.write(p.stderr)
    return p.returncode


def _stub(tmp: Path, mode: str) -> Path:
    """An executable that re-enters this file in `mode` with the solver's argv."""
    stub = tmp / "lbm3d-perm"
    stub.write_text(f"#!/bin/sh\nexec {sys.executable} {Path(__file__).resolve()} {mode} \"$@\"\n")
    stub.chmod(0o755)
    return stub


def record() -> None:
    if not (REF / "scripts" / "validate_solver3d.py").exists():
        sys.exit(f"reference scripts not found under {REF}")
    FIX.mkdir(exist_ok=True)
    tmp = Path(tempfile.mkdtemp(prefix="scripts_chain_"))
    log = tmp / "calls.jsonl"
    env = dict(os.environ, SCRIPTS_CHAIN_LOG=str(log), PYTHONPATH=str(ROOT), PYTHONDONTWRITEBYTECODE="1")
    stub = _stub(tmp, "proxy")
    out = {}
    for name, (args, timeout) in SCRIPTS.items():
        p = subprocess.run([sys.executable, str(REF / args[0]), "--solver", str(stub)] + args[1:],
                           cwd=str(REF), env=env, capture_output=True, text=True, timeout=timeout)
        out[name] = dict(argv=args, rc=p.returncode, stdout=p.stdout.splitlines())
        print(name, "rc", p.returncode, flush=True)
    calls = [json.loads(ln) for ln in log.read_text().splitlines()]
    for c in calls:
        c["filename"] = Path(c["filename"]).name
    (FIX / "invocations.json").write_text(json.dumps(calls, indent=1) + "\n")
    (FIX / "scripts.json").write_text(json.dumps(out, indent=1) + "\n")
    shutil.rmtree(tmp, ignore_errors=True)


# --------------------------------------------------------------- shim rows --
def shim_rows(out_path: str) -> None:
    """Every recorded invocation through the drop-in (needs a GPU)."""
    sys.path.insert(0, str(ROOT))
    from flow_anizotropy_b200 import cli3d
    calls = json.loads((FIX / "invocations.json").read_text())
    res = []
    with tempfile.TemporaryDirectory(prefix="shim_rows_") as tmp:
        for i, c in enumerate(calls):
            raw = Path(tmp) / c["filename"]
            raw.write_bytes(load_raw_bytes(c["sha"]))
            csv = Path(tmp) / f"out{i}.csv"
            so = io.StringIO()
            cwd = os.getcwd()
            os.chdir(tmp)
            try:
                with contextlib.redirect_stdout(so):
                    rc = cli3d.main([raw.name, csv.name] + c["opts"])
            finally:
                os.chdir(cwd)
            _, row = _appended_row(csv, 0)
            res.append(dict(sha=c["sha"], opts=c["opts"], rc=rc, stdout=so.getvalue(), row=row))
            print(i, c["filename"], "rc", rc, flush=True)
    Path(out_path).write_text(json.dumps(res, indent=1) + "\n")


# ------------------------------------------------------------------ replay --
def replay(argv) -> int:
    """--solver stub: the drop-in's recorded answer to this call."""
    sys.path.insert(0, str(ROOT))
    from flow_anizotropy_b200 import tensor as T
    structure, csv, opts = argv[0], Path(argv[1]), argv[2:]
    sha = _sha(Path(structure).read_bytes())
    rows = json.loads(Path(os.environ["SCRIPTS_CHAIN_ROWS"]).read_text())
    hit = {_key(r["sha"], r["opts"]): r for r in rows}.get(_key(sha, opts))
    if hit is None:
        sys.stderr.write(f"lbm3d-perm (replay): no recorded drop-in run for {structure} {' '.join(opts)}\n")
        return 2
    if hit["row"] is not None:
        # the drop-in writes the path it was given in the filename column
        row = hit["row"].split(",", 1)
        line = structure + "," + row[1]
        need_header = not csv.exists() or csv.stat().st_size == 0
        with open(csv, "a") as fh:
            if need_header:
                fh.write(T.header3() + "\n")
            fh.write(line + "\n")
    sys.stdout.write(hit["stdout"])
    return int(hit["rc"])


def main() -> None:
    mode = sys.argv[1] if len(sys.argv) > 1 else ""
    if mode == "record":
        record()
    elif mode == "shim-rows":
        shim_rows(sys.argv[2])
    elif mode == "proxy":
        sys.path.insert(0, str(ROOT))
        sys.exit(proxy(sys.argv[2:]))
    elif mode == "replay":
        sys.exit(replay(sys.argv[2:]))
    else:
        sys.exit(__doc__)


if __name__ == "__main__":
    main()
