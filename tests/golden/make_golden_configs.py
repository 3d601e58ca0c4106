"""Reference rows at the benchmark configurations, written by the REFERENCE solver.

    python tests/golden/make_golden_configs.py [plain64] [precision128]
        (needs oracle/_ref/lbm3d-perm, built by oracle/build_ref.sh)

The structures are too large to commit (the 128^3 packing is 2.1 MB), and they
are deterministic functions of their seeds, so this script commits, per
configuration, the generator call, the SHA-256 of the structure bytes it
produced, the argv, and the CSV row the reference binary appended
(tests/golden/configs/<name>.csv).  The tests rebuild the structure from the
seed, check the hash, solve it on the GPU and compare with the row.

  plain64       64^3 spheres r = 6, phi 0.60, percolating in x (seed 0);
                --ff 4 --lag 1000 --eps 1e-6 --max-steps 50000 (the single-solve
                configuration; hold, min-steps and avg-steps at their defaults)
  precision128  128^3 prolate ellipsoids (4, 4, 12) along z, phi 0.45,
                percolating in x, y, z (seed 0); the same knobs (the
                precision-study tensor the bench times)

The reference solves the three directions one after another in one process
(LMB3d/lbm3d-perm.cpp:518-520); the 128^3 row takes about an hour of one core.
"""
import hashlib
import json
import subprocess
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "configs"
sys.path.insert(0, str(ROOT))

from flow_anizotropy_b200 import structures as st                 # noqa: E402
from flow_anizotropy_b200.structure_io3d import save_structure    # noqa: E402
from oracle import oracle as O                                    # noqa: E402

KNOBS = ["--ff", "4", "--lag", "1000", "--eps", "1e-6", "--max-steps", "50000"]

CONFIGS = {
    "plain64": dict(generator="plain_64", seed=0, argv=KNOBS),
    "precision128": dict(generator="precision_128", seed=0, argv=KNOBS),
}


def structure(name):
    c = CONFIGS[name]
    return getattr(st, c["generator"])(c["seed"])


def sha256(solid):
    return hashlib.sha256(solid.tobytes()).hexdigest()


def run(name):
    exe = O.ref_binary("lbm3d-perm")
    if exe is None:
        sys.exit("lbm3d-perm not built: run oracle/build_ref.sh first")
    c = CONFIGS[name]
    s = structure(name)
    OUT.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="golden_cfg_") as tmp:
        raw = Path(tmp) / f"{name}.raw"
        save_structure(raw, s)
        csv = OUT / f"{name}.csv"
        csv.unlink(missing_ok=True)
        t0 = time.time()
        # the row's filename column is the argv path: run from the temp dir with
        # the bare name so the row does not carry a machine path
        p = subprocess.run([str(exe), raw.name, str(csv), "--quiet"] + c["argv"], cwd=tmp,
                           capture_output=True, text=True)
        dt = time.time() - t0
    meta = dict(generator=c["generator"], seed=c["seed"], shape=list(s.shape), sha256=sha256(s),
                porosity=float((s == 0).mean()), argv=c["argv"], rc=p.returncode,
                stderr=p.stderr.strip().splitlines(), seconds=round(dt, 1))
    (OUT / f"{name}.json").write_text(json.dumps(meta, indent=1) + "\n")
    print(name, "rc", p.returncode, f"{dt:.0f} s", flush=True)


def main():
    names = sys.argv[1:] or list(CONFIGS)
    for n in names:
        run(n)


if __name__ == "__main__":
    main()
