"""CPU restatement of the structure generator — TEST INFRASTRUCTURE ONLY.

Restates the per-voxel parts of scripts/gen_aniso_structures3d.py with numpy
and scipy, in the reference's arithmetic: the trigonometric field summed mode
by mode over outer sums of the per-axis phases (:154-176), the numpy linear
quantile threshold (:179-181) and the 6-connected percolation test on the
3 x 3 x 3 tiling (:184-205).  The random draws reuse the host-side sampling of
flow_anizotropy_b200.gen3d (which the golden fixtures pin through this
module).  Only tests import it, as the checker of the device generator.
"""
from __future__ import annotations

import numpy as np
from scipy.ndimage import generate_binary_structure, label

from flow_anizotropy_b200 import gen3d as G


def field(pts, q, phases):
    """sqrt(2/n) sum_m cos(((2 pi qz) z + (2 pi qy) y) + (2 pi qx) x + phi_m) on [z, y, x]."""
    size = len(pts)
    twopi = 2.0 * np.pi
    acc = np.zeros((size, size, size))
    for (qx, qy, qz), phi in zip(q, phases):
        ph = np.add.outer(np.add.outer(twopi * qz * pts, twopi * qy * pts), twopi * qx * pts)
        ph += phi
        acc += np.cos(ph)
    return np.sqrt(2.0 / len(q)) * acc


def percolates(solid):
    """(x, y, z): a 6-connected pore cluster of the 3 x 3 x 3 tiling touches both faces."""
    lab, n = label(np.tile(~solid.astype(bool), (3, 3, 3)), structure=generate_binary_structure(3, 1))
    if n == 0:
        return False, False, False
    out = []
    for axis in (2, 1, 0):
        lo = set(np.take(lab, 0, axis=axis).ravel())
        hi = set(np.take(lab, -1, axis=axis).ravel())
        out.append(bool((lo & hi) - {0}))
    return tuple(out)


def sample(sample_id, size, **cfg):
    """(solid bool [z, y, x], row) of one sample, or None (gen_aniso_structures3d.py:208-266)."""
    c = {**G.DEFAULTS, **cfg}
    pts = G.axis_points(size)
    rng = np.random.default_rng(c["seed"] + sample_id)
    name, a_lo, a_hi = G.STRATA[sample_id % len(G.STRATA)]
    for attempt in range(c["max_attempts"]):
        a = float(rng.uniform(a_lo, a_hi))
        b = float(rng.uniform(1.0, a)) if a > 1.0 else 1.0
        R = G.rotation(rng)
        k0 = float(rng.uniform(c["k0_min"], c["k0_max"]))
        n_modes = int(rng.integers(c["modes_min"], c["modes_max"] + 1))
        porosity = float(rng.uniform(c["por_min"], c["por_max"]))
        q = G.wavevectors(rng, n_modes, k0, c["dk"], a, b, R)
        if len(q) < 5:
            continue
        phases = rng.uniform(0.0, np.pi, len(q))
        f = field(pts, q, phases)
        t = float(np.quantile(f, porosity))
        solid = f > t
        if not all(percolates(solid)):
            continue
        por = float(1.0 - solid.mean())
        fname = f"sample_{sample_id:06d}_str={name}_A={a:.2f}_B={b:.2f}_k0={k0:.2f}_por={por:.4f}.raw"
        return solid, {"sample_id": sample_id, "filename": fname, "aniso_A": a, "aniso_B": b, "k0": k0,
                       "n_modes": len(q), "porosity": por, "porosity_target": porosity, "threshold": t,
                       "attempts": attempt + 1}
    return None
