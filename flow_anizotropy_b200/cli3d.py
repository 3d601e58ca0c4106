"""``lbm3d-perm`` drop-in: the argv, CSV row and exit codes of LMB3d/lbm3d-perm.cpp:445-631.

    python -m flow_anizotropy_b200.cli3d <structure.raw> <results.csv> [options]
    flow_anizotropy_b200/bin/lbm3d-perm  <structure.raw> <results.csv> [options]

Solves the cell along +x, +y, +z (plus (1,1,1)/sqrt 3 with --validate) on the
GPU, all directions concurrently, and appends one row with the full tensor.
Exit 0 = all three converged, 3 = a direction did not (row still written),
2 = error (message ``lbm3d-perm: ...`` on stderr, no row).

Options beyond the reference's (all default to the reference's behaviour):
  --tau T            relaxation time (reference: compile-time 1.0)
  --precision P      fp64 (default, the reference's arithmetic) | fp32 | fp16 | bf16
  --criterion C      drift (reference) | block (block means + k-sigma) | batch (block, batch-means SE) | auto
  --device N         CUDA device
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from . import solver as S
from . import tensor as T
from .structure_io3d import StructureError, read_raw_checked

PROG = "lbm3d-perm"

USAGE = """Usage: lbm3d-perm <structure.raw> <results.csv> [options]

Solves a triply periodic cell three times (force along +x, +y, +z) and
appends one row with the full 3x3 permeability tensor to <results.csv>.

  --ff F            force factor; body force = 2.5e-07 * F   (default 1)
  --eps E           drift tolerance, relative to |q|         (default 1e-5)
  --lag N           steps between convergence checks         (default 2000)
  --hold K          consecutive passing checks required      (default 2)
  --min-steps N     no convergence before this step          (default 4000)
  --max-steps N     give up after this many steps            (default 200000)
  --avg-steps N     averaging phase after convergence        (default 2000)
  --velocity PREFIX write PREFIX.fx.vel, PREFIX.fy.vel, PREFIX.fz.vel
  --validate        extra solve along (1,1,1)/sqrt(3); reports the flux
                    predicted by K against the measured one (Koza09 test)
  --quiet           suppress per-check progress
  --tau T           relaxation time                          (default 1)
  --precision P     fp64 | fp32 | fp16 | bf16                (default fp64)
  --criterion C     drift | block | batch | auto             (default auto:
                    drift for fp64/fp32, batch for fp16/bf16)
  --device N        CUDA device                              (default 0)
"""


class Die(Exception):
    pass


def strtol(s: str) -> int:
    """C strtol(s, NULL, 10): leading integer, 0 if none (LMB3d/lbm3d-perm.cpp:467-471)."""
    s = s.lstrip()
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    return int(s[:j]) if j > i else 0


def strtod(s: str) -> float:
    """C strtod: the longest leading float, 0.0 if none."""
    s = s.lstrip()
    for n in range(len(s), 0, -1):
        try:
            return float(s[:n])
        except ValueError:
            continue
    return 0.0


def parse(argv):
    if len(argv) < 2:
        raise SystemExit(_usage_exit(2))
    cfg = dict(ff=1.0, eps=1e-5, lag=2000, hold=2, min_steps=4000, max_steps=200000,
               avg_steps=2000, velocity="", quiet=False, validate=False, tau=1.0,
               precision="fp64", criterion="auto", device=0)
    structure, resultfile = argv[0], argv[1]
    i = 2

    def need(kind):
        nonlocal i
        if i + 1 >= len(argv):
            sys.stderr.write(USAGE)
            raise Die("missing value for " + argv[i])
        i += 1
        return kind(argv[i])

    while i < len(argv):
        a = argv[i]
        if a == "--ff": cfg["ff"] = need(strtod)
        elif a == "--eps": cfg["eps"] = need(strtod)
        elif a == "--lag": cfg["lag"] = need(strtol)
        elif a == "--hold": cfg["hold"] = need(strtol)
        elif a == "--min-steps": cfg["min_steps"] = need(strtol)
        elif a == "--max-steps": cfg["max_steps"] = need(strtol)
        elif a == "--avg-steps": cfg["avg_steps"] = need(strtol)
        elif a == "--velocity": cfg["velocity"] = need(str)
        elif a == "--validate": cfg["validate"] = True
        elif a == "--quiet": cfg["quiet"] = True
        elif a == "--tau": cfg["tau"] = need(strtod)
        elif a == "--precision": cfg["precision"] = need(str)
        elif a == "--criterion": cfg["criterion"] = need(str)
        elif a == "--device": cfg["device"] = need(strtol)
        else:
            sys.stderr.write(USAGE)
            raise Die("unknown option " + a)
        i += 1
    if cfg["precision"] not in ("fp64", "fp32", "fp16", "bf16", "m32", "m64", "md32"):
        raise Die("unknown precision " + cfg["precision"])
    if cfg["criterion"] not in ("drift", "block", "batch", "auto"):
        raise Die("unknown criterion " + cfg["criterion"])
    return structure, resultfile, cfg


def _usage_exit(code):
    sys.stderr.write(USAGE)
    return code


def write_vel(path, u, shape_xyz):
    """``.vel``: int32 {nx, ny, nz, 3} then N x 3 float32, x fastest (LMB3d/lbm3d-perm.cpp:305-317)."""
    nx, ny, nz = shape_xyz
    try:
        with open(path, "wb") as fh:
            fh.write(np.array([nx, ny, nz, 3], dtype="<i4").tobytes())
            fh.write(np.ascontiguousarray(u, dtype="<f4").tobytes())
    except OSError:
        raise Die("cannot write " + path) from None


def run(argv) -> int:
    structure, resultfile, cfg = parse(argv)
    solid = read_raw_checked(structure)
    nz, ny, nx = solid.shape
    n_pore = int((solid == 0).sum())
    porosity = n_pore / float(solid.size)
    F = S.FX_BASE * cfg["ff"]
    tau = cfg["tau"]
    mu = (1.0 / 3.0) * (tau - 0.5)
    if not cfg["quiet"]:
        print(f"# structure {structure}  {nx}x{ny}x{nz}  porosity {porosity:g}  force {F:g}  mu {mu:g}",
              flush=True)

    forces = [[F, 0, 0], [0, F, 0], [0, 0, F]]
    c = 1.0 / math.sqrt(3.0)
    if cfg["validate"]:
        forces.append([F * c, F * c, F * c])
    params = S.Params3D(tau=tau, eps=cfg["eps"], lag=cfg["lag"], hold=cfg["hold"],
                        min_steps=cfg["min_steps"], max_steps=cfg["max_steps"],
                        avg_steps=cfg["avg_steps"], precision=cfg["precision"],
                        criterion=cfg["criterion"])
    if params.lag <= 0:
        raise Die("--lag must be positive")
    want_vel = bool(cfg["velocity"])
    try:
        runs, rc, vel = S.solve3d(solid, forces, params, velocity=want_vel, device=cfg["device"])
    except S.LBMError as e:
        raise Die(str(e)) from None
    tags = ("fx", "fy", "fz", "val")
    for j, r in enumerate(runs):
        if r.status:
            raise Die(f"non-finite flux in run {tags[j]} at step {r.steps}")
        if not r.converged and not cfg["quiet"]:
            sys.stderr.write(f"# {tags[j]}: max-steps reached without convergence\n")
        if not cfg["quiet"]:
            print(f"# {tags[j]} {r.steps}  q=({r.q[0]:g}, {r.q[1]:g}, {r.q[2]:g})  "
                  f"converged {r.converged}", flush=True)
    if want_vel:
        for j in range(3):
            write_vel(cfg["velocity"] + "." + tags[j] + ".vel", vel[j], (nx, ny, nz))
        if cfg["validate"]:
            write_vel(cfg["velocity"] + ".val.vel", vel[3], (nx, ny, nz))

    rx, ry, rz = runs[:3]
    Tn = T.assemble3([rx.q, ry.q, rz.q], mu, F)
    if cfg["validate"]:
        rv = runs[3]
        Ks = Tn.Ks
        pred = [(Ks[r][0] * F * c + Ks[r][1] * F * c + Ks[r][2] * F * c) / mu for r in range(3)]
        err = sum((rv.q[r] - pred[r]) ** 2 for r in range(3))
        qn = sum(rv.q[r] ** 2 for r in range(3))
        print(f"# tensor test along (1,1,1)  (converged {rv.converged}, {rv.steps} steps)")
        print(f"#   predicted q = ({pred[0]:g}, {pred[1]:g}, {pred[2]:g})")
        print(f"#   measured  q = ({rv.q[0]:g}, {rv.q[1]:g}, {rv.q[2]:g})")
        print(f"#   relative error {math.sqrt(err) / (math.sqrt(qn) if qn > 0 else 1):g}", flush=True)

    row = T.row3(structure, cfg["ff"], F, mu, (nx, ny, nz), porosity, [rx, ry, rz], Tn)
    try:
        T.append_csv(resultfile, T.header3(), row)
    except OSError:
        raise Die("cannot open " + resultfile + " for writing") from None

    if not cfg["quiet"]:
        K = Tn.K
        print("# K =")
        for r in range(3):
            print(f"#   [ {K[r][0]:12g} {K[r][1]:12g} {K[r][2]:12g} ]")
        print(f"# reciprocity residuals  xy {Tn.rec_xy:g}  xz {Tn.rec_xz:g}  yz {Tn.rec_yz:g}")
        print(f"# k1 {Tn.val[0]:g}  k2 {Tn.val[1]:g}  k3 {Tn.val[2]:g}  k_mean {Tn.kmean:g}  FA {Tn.fa:g}",
              flush=True)
    return 0 if (rx.converged and ry.converged and rz.converged) else 3


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        return run(argv)
    except (Die, StructureError) as e:
        sys.stderr.write(f"{PROG}: {e}\n")
        return 2
    except SystemExit as e:
        return int(e.code) if isinstance(e.code, int) else 2


if __name__ == "__main__":
    sys.exit(main())
