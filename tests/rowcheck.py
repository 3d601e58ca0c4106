"""Row comparison helpers shared by the golden-row tests (CPU oracle and GPU drop-in)."""
import math


def argv_params(argv, defaults):
    p, flags = dict(defaults), set()
    keymap = {"--lag": "lag", "--eps": "eps", "--hold": "hold", "--min-steps": "min_steps",
              "--max-steps": "max_steps", "--avg-steps": "avg_steps", "--avg-sample": "avg_sample",
              "--ff": "ff", "--validate": "validate"}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a == "--validate" and (i + 1 >= len(argv) or argv[i + 1].startswith("--")):
            flags.add("validate"); i += 1; continue
        p[keymap[a]] = float(argv[i + 1]) if a in ("--eps", "--ff", "--validate") else int(argv[i + 1])
        i += 2
    return p, flags


def close_row(mine: str, ref: str, header: str, rtol, skip=()):
    """Field-by-field comparison.  Fluxes and tensor entries: rtol, plus an
    absolute floor of rtol x the largest value of their kind (off-diagonals
    are tiny differences); standard errors and reciprocity residuals are
    roundoff-level by construction and are bounded on the flux / tensor scale.
    Columns in `skip` are not compared (the caller checks them another way)."""
    cols = header.split(",")
    a, b = mine.split(","), ref.split(",")
    assert len(a) == len(b) == len(cols)
    val = {c: y for c, y in zip(cols, b)}
    def fl(c):
        try:
            return abs(float(val[c]))
        except ValueError:
            return 0.0
    qmax = max([fl(c) for c in cols if c.startswith("q")] + [1e-300])
    # principal axes are only defined for distinct principal values
    kk = [fl(c) for c in ("k1", "k2", "k3")] if "k3" in val else []
    degenerate = any(abs(a - b) < 1e-6 * max(kk) for a, b in zip(kk, kk[1:])) if kk else False
    kmax = max([fl(c) for c in cols if c.startswith(("K_", "k_", "k1", "k2", "k3"))] + [1e-300])
    for c, x, y in zip(cols, a, b):
        if c in skip:
            continue
        try:
            fx, fy = float(x), float(y)
        except ValueError:
            assert x == y, c
            continue
        if math.isnan(fy):
            assert math.isnan(fx), c
            continue
        if c.startswith(("steps", "conv", "nx", "ny", "nz")):
            assert fx == fy, c
        elif c.startswith("se_"):
            assert abs(fx - fy) <= 1e-8 * qmax, (c, x, y)
        elif c.startswith("recip") or c.startswith(("fieldres", "alpha", "theta", "aniso")):
            assert abs(fx - fy) <= 1e-6 * max(abs(fy), 1.0) * (1 if not c.startswith("recip") else 1e-2), (c, x, y)
        elif c.startswith(("q",)):
            assert abs(fx - fy) <= rtol * abs(fy) + rtol * qmax, (c, x, y)
        elif c.startswith(("K_", "k_", "k1", "k2", "k3")):
            assert abs(fx - fy) <= rtol * abs(fy) + rtol * kmax, (c, x, y)
        elif c.startswith("v"):
            assert degenerate or abs(fx - fy) <= 1e-6, (c, x, y)
        else:
            assert abs(fx - fy) <= rtol * max(abs(fy), 1e-300), (c, x, y)
