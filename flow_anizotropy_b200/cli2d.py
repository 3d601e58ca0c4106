"""``lbm2d-perm`` drop-in: argv, CSV row and exit codes of LMB2d/main.cpp:237-427.

    python -m flow_anizotropy_b200.cli2d <structure.gif|ppm|dat> <results.csv> [options]

Solves the doubly periodic cell along +x and +y (plus --validate DEG) with
the reference's D2Q9 operator (raw FP32 populations, velocity-shift forcing,
raw-moment velocity, k = mu q / F with mu = 0.33 (tau - 1/2)) and appends one
row.  Exit 0 = both converged, 3 = one did not, 2 = error, 1 = too few
arguments (as the reference).  Extra options: --tau, --device, and
--size NXxNY for .dat/.ppm input (the reference's fixed cell is 256x256).
"""
from __future__ import annotations

import math
import sys

import numpy as np

from . import solver as S
from . import tensor as T
from .cli3d import Die, strtod, strtol
from .structure_io import load_structure2d

PROG = "lbm2d-perm"

USAGE = """Usage: lbm2d-perm <structure.gif|ppm|dat> <results.csv> [options]

Solves the 256x256 doubly periodic cell twice (force along +x, then +y)
and appends one row with the full permeability tensor to <results.csv>.

  --ff F            force factor; body force = 2.5e-07 * F   (default 1)
  --eps E           per-component relative tolerance         (default 1e-3)
  --lag N           steps between convergence checks         (default 5000)
  --hold K          consecutive passing checks required      (default 3)
  --min-steps N     no convergence before this step          (default 10000)
  --max-steps N     give up after this many steps            (default 500000)
  --avg-steps N     length of the averaging phase            (default 20000)
  --avg-sample N    flux sampling interval                   (default 50)
  --qfloor R        floor for the relative test, as a fraction of |q|
                                                             (default 1e-2)
  --ksigma K        also accept a change within K sigma of the block
                    mean's own standard error               (default 3)
  --velocity PREFIX write PREFIX.fx.dat and PREFIX.fy.dat
  --validate DEG    extra solve with the force at DEG degrees; reports the
                    flux predicted by K against the measured one (Koza09
                    tensor test).  Diagnostic — not written to the CSV.
  --quiet           suppress per-check progress on stdout
  --tau T           relaxation time                          (default 1)
  --size NXxNY      cell size of .dat/.ppm input             (default 256x256)
  --device N        CUDA device                              (default 0)
"""


def mu_2d(tau: float) -> float:
    """``float mu = 0.33*(tau-0.5)`` with float tau (LMB2d/lbm.cpp:86-87)."""
    return float(np.float32(0.33 * (float(np.float32(tau)) - 0.5)))


def parse(argv):
    """(structure, resultfile, cfg) from the lbm2d-perm argv; None after --help."""
    if len(argv) < 2:
        sys.stderr.write(USAGE)
        raise Die("missing arguments")
    structure, resultfile = argv[0], argv[1]
    cfg = dict(ff=1.0, eps=1e-3, lag=5000, hold=3, min_steps=10000, max_steps=500000,
               avg_steps=20000, avg_sample=50, qfloor=1e-2, ksigma=3.0, velocity="",
               quiet=False, validate=-1.0, tau=1.0, size=(256, 256), device=0)
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
        elif a == "--avg-sample": cfg["avg_sample"] = need(strtol)
        elif a == "--qfloor": cfg["qfloor"] = need(strtod)
        elif a == "--ksigma": cfg["ksigma"] = need(strtod)
        elif a == "--velocity": cfg["velocity"] = need(str)
        elif a == "--validate": cfg["validate"] = need(strtod)
        elif a == "--quiet": cfg["quiet"] = True
        elif a == "--tau": cfg["tau"] = need(strtod)
        elif a == "--device": cfg["device"] = need(strtol)
        elif a == "--size":
            v = need(str).lower().split("x")
            if len(v) != 2:
                raise Die("--size wants NXxNY")
            cfg["size"] = (strtol(v[0]), strtol(v[1]))
        elif a in ("-h", "--help"):
            sys.stderr.write(USAGE)
            return None
        else:
            sys.stderr.write(USAGE)
            raise Die("unknown option " + a)
        i += 1
    if cfg["lag"] <= 0 or cfg["avg_sample"] <= 0:
        raise Die("--lag and --avg-sample must be positive")

    return structure, resultfile, cfg


def run(argv) -> int:
    if len(argv) < 2:
        sys.stderr.write(USAGE)
        return 1
    parsed = parse(argv)
    if parsed is None:
        return 0
    structure, resultfile, cfg = parsed
    F = S.FX_BASE * cfg["ff"]
    nx, ny = cfg["size"]
    try:
        solid = load_structure2d(structure, nx, ny)
    except OSError:
        raise Die("cannot open " + structure) from None
    except Exception as e:              # an undecodable image
        raise Die(f"cannot read {structure}: {e}") from None
    ny, nx = solid.shape
    mu = mu_2d(cfg["tau"])
    nfluid = int((solid == 0).sum())
    porosity = float(np.float32(nfluid) / np.float32(nx * ny))    # getporosity_full, float
    if not cfg["quiet"]:
        print(f"# structure {structure}  porosity {porosity:g}  force {F:g} (ff={cfg['ff']:g})  mu {mu:g}",
              flush=True)

    forces = [[F, 0.0], [0.0, F]]
    if cfg["validate"] >= 0.0:
        th = cfg["validate"] * math.pi / 180.0
        forces.append([F * math.cos(th), F * math.sin(th)])
    params = S.Params2D(tau=cfg["tau"], eps=cfg["eps"], lag=cfg["lag"], hold=cfg["hold"],
                        min_steps=cfg["min_steps"], max_steps=cfg["max_steps"],
                        avg_steps=cfg["avg_steps"], avg_sample=cfg["avg_sample"],
                        qfloor=cfg["qfloor"], ksigma=cfg["ksigma"])
    want_vel = bool(cfg["velocity"])
    try:
        runs, rc, vel = S.solve2d(solid, forces, params, velocity=want_vel, device=cfg["device"])
    except S.LBMError as e:
        raise Die(str(e)) from None
    tags = ("fx", "fy", "val")
    for j, r in enumerate(runs):
        if r.status:
            raise Die(f"non-finite flux in run {tags[j]} at step {r.steps}")
        if not r.converged and not cfg["quiet"]:
            sys.stderr.write(f"# {tags[j]}: max-steps reached without convergence\n")
    if want_vel:
        for j in range(2):
            write_vel2d(cfg["velocity"] + "." + tags[j] + ".dat", vel[j])
        if cfg["validate"] >= 0.0:
            write_vel2d(cfg["velocity"] + ".val.dat", vel[2])

    rx, ry = runs[0], runs[1]
    Tn = T.assemble2(rx, ry, mu, F)
    if cfg["validate"] >= 0.0:
        rv = runs[2]
        Fx, Fy = forces[2]
        pred_qx = (Tn.k_xx * Fx + Tn.k_off * Fy) / mu
        pred_qy = (Tn.k_off * Fx + Tn.k_yy * Fy) / mu
        qn = math.sqrt(rv.q[0] ** 2 + rv.q[1] ** 2)
        err = math.sqrt((rv.q[0] - pred_qx) ** 2 + (rv.q[1] - pred_qy) ** 2) / (qn if qn > 0 else 1)
        print(f"# tensor test at {cfg['validate']:g} deg  (converged {rv.converged}, {rv.steps} steps)")
        print(f"#   predicted q = ({pred_qx:g}, {pred_qy:g})")
        print(f"#   measured  q = ({rv.q[0]:g}, {rv.q[1]:g})")
        print(f"#   relative error {err:g}", flush=True)

    row = T.row2(structure, cfg["ff"], F, mu, porosity, rx, ry, Tn)
    try:
        T.append_csv(resultfile, T.header2(), row)
    except OSError:
        raise Die("cannot open " + resultfile + " for writing") from None
    if not cfg["quiet"]:
        print(f"# K = [ {Tn.k_xx:g} {Tn.k_xy:g} ; {Tn.k_yx:g} {Tn.k_yy:g} ]")
        rel = abs(Tn.k_xy - Tn.k_yx) / abs(2 * Tn.k_off) if Tn.k_off != 0.0 else math.nan
        print(f"# reciprocity residual {Tn.recip:g}   (relative error on k_off: {rel:g})")
        print(f"# k1 {Tn.k1:g}  k2 {Tn.k2:g}  anisotropy {Tn.aniso:g}  theta {Tn.theta:g} deg", flush=True)
    return 0 if (rx.converged and ry.converged) else 3


def write_vel2d(path, uv):
    """exportvelocity (LMB2d/lbm.cpp:634-641): 'U V' per node, y outer, x inner."""
    try:
        with open(path, "w") as fh:
            for row in uv:
                for u, v in row:
                    fh.write(f"{float(u):g} {float(v):g}\n")
    except OSError:
        raise Die("cannot write " + path) from None


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        return run(argv)
    except Die as e:
        sys.stderr.write(f"{PROG}: {e}\n")
        return 2


if __name__ == "__main__":
    sys.exit(main())
