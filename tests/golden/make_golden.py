"""Generate the golden fixtures of tests/golden/ from the REFERENCE solvers.

    python tests/golden/make_golden.py        (needs oracle/_ref/, built by oracle/build_ref.sh)

Each case writes the input structure and the CSV row the reference binary
appended for it.  The structures are tiny and seeded, so the fixtures stay a
few kB; the tests recompute the same solves with the CPU oracle (and, on a
GPU, with liblbm) and compare against these rows.

  case3d_*.raw / .csv   LMB3d/lbm3d-perm.cpp  (tau = 1 binary, and the tau = 0.8 build)
  case2d_*.dat / .csv   LMB2d/main.cpp + lbm.cpp (256 x 256 fixed cell, .dat input)
"""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from flow_anizotropy_b200.structure_io import save_dat          # noqa: E402
from flow_anizotropy_b200.structure_io3d import save_structure  # noqa: E402
from oracle import oracle as O                                  # noqa: E402

CASES3D = [
    # name, shape (nz, ny, nx), seed, solid fraction, binary, extra argv
    ("case3d_a", (12, 14, 16), 1, 0.30, "lbm3d-perm",
     ["--ff", "4", "--lag", "200", "--eps", "1e-8", "--min-steps", "400", "--max-steps", "3000", "--avg-steps", "50"]),
    ("case3d_b", (9, 11, 13), 2, 0.25, "lbm3d-perm",
     ["--ff", "1", "--lag", "100", "--eps", "1e-6", "--hold", "3", "--min-steps", "300", "--max-steps", "1500",
      "--avg-steps", "0", "--validate"]),
    ("case3d_tau08", (10, 12, 14), 3, 0.30, "lbm3d-perm-tau0.8",
     ["--ff", "4", "--lag", "200", "--eps", "1e-8", "--min-steps", "400", "--max-steps", "2500", "--avg-steps", "20"]),
    ("case3d_slit", (16, 8, 8), 0, None, "lbm3d-perm",
     ["--lag", "500", "--eps", "1e-7", "--min-steps", "1000", "--max-steps", "4000", "--avg-steps", "10"]),
]

CASES2D = [
    ("case2d_a", 7, 0.22, ["--lag", "500", "--min-steps", "1000", "--max-steps", "2000", "--avg-steps", "200",
                          "--avg-sample", "50", "--validate", "30"]),
]


def structure3d(shape, seed, frac):
    if frac is None:                      # slit: solid slab normal to z, 10 fluid layers
        s = np.zeros(shape, np.uint8)
        s[: shape[0] - 10] = 1
        return s
    s = (np.random.default_rng(seed).random(shape) < frac).astype(np.uint8)
    s.flat[0] = 0
    return s


def structure2d(seed, frac):
    rng = np.random.default_rng(seed)
    s = np.zeros((256, 256), np.uint8)
    # disc packing, periodic
    yy, xx = np.mgrid[0:256, 0:256]
    while s.mean() < frac:
        cx, cy, r = rng.integers(0, 256), rng.integers(0, 256), rng.integers(4, 12)
        dx = np.minimum(np.abs(xx - cx), 256 - np.abs(xx - cx))
        dy = np.minimum(np.abs(yy - cy), 256 - np.abs(yy - cy))
        s[dx * dx + dy * dy <= r * r] = 1
    return s


def main():
    meta = {}
    for name, shape, seed, frac, binary, argv in CASES3D:
        exe = O.ref_binary(binary)
        if exe is None:
            sys.exit(f"{binary} not built: run oracle/build_ref.sh first")
        s = structure3d(shape, seed, frac)
        raw = HERE / f"{name}.raw"
        save_structure(raw, s)
        csv = HERE / f"{name}.csv"
        csv.unlink(missing_ok=True)
        p = subprocess.run([str(exe), raw.name, csv.name, "--quiet"] + argv, cwd=HERE,
                           capture_output=True, text=True)
        meta[name] = dict(binary=binary, argv=argv, rc=p.returncode, stdout=p.stdout.strip().splitlines())
        print(name, "rc", p.returncode)
    for name, seed, frac, argv in CASES2D:
        exe = O.ref_binary("lbm2d-perm")
        s = structure2d(seed, frac)
        dat = HERE / f"{name}.dat"
        save_dat(dat, s)
        csv = HERE / f"{name}.csv"
        csv.unlink(missing_ok=True)
        p = subprocess.run([str(exe), dat.name, csv.name, "--quiet"] + argv, cwd=HERE,
                           capture_output=True, text=True)
        meta[name] = dict(binary="lbm2d-perm", argv=argv, rc=p.returncode, stdout=p.stdout.strip().splitlines())
        print(name, "rc", p.returncode)
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
