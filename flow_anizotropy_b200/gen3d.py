"""3D anisotropic structure sets generated on the GPU.

The dataset generator of scripts/gen_aniso_structures3d.py with its per-voxel
work on the device: for each sample the host draws the random parameters with
numpy's generator in the reference's order (stratum, axis ratios A and B, a
uniformly random rotation, band centre k0, mode count, target porosity,
wavevectors, phases; gen_aniso_structures3d.py:111-152, 208-229), and the
device evaluates the trigonometric field, its exact porosity quantile and the
percolation test (``lbm_trig_structure3d``, ``lbm_percolates3d``).  A sample
whose pore phase does not span x, y and z is redrawn from the same stream,
as the reference does, up to ``max_attempts``.

The output directory has the reference's layout: ``structures/<name>.raw``
(the reference's file names), ``structures.csv`` with its columns, and
``filelist.txt``; ``scripts/solve_permeability3d.py`` and
``flow_anizotropy_b200.batch3d`` take it as it is.

    python -m flow_anizotropy_b200.gen3d --output DATA/aniso3d --n_samples 5000 --size 80
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import sys

import numpy as np

from . import _lib
from .structure_io3d import save_structure

# (name, lowest, highest primary axis ratio), taken by sample_id modulo 3
# (gen_aniso_structures3d.py:84-89)
STRATA = (("iso", 1.0, 1.0), ("mod", 1.5, 2.5), ("strong", 2.5, 4.0))

DEFAULTS = dict(seed=0, k0_min=3.0, k0_max=7.0, dk=1.0, modes_min=20, modes_max=80,
                por_min=0.65, por_max=0.90, max_attempts=200)


def rotation(rng) -> np.ndarray:
    """Uniform rotation from a unit quaternion drawn by Shoemake's method
    (three uniforms; gen_aniso_structures3d.py:111-128)."""
    u1, u2, u3 = rng.random(3)
    s1, s2 = np.sqrt(1.0 - u1), np.sqrt(u1)
    x, y = s1 * np.sin(2 * np.pi * u2), s1 * np.cos(2 * np.pi * u2)
    z, w = s2 * np.sin(2 * np.pi * u3), s2 * np.cos(2 * np.pi * u3)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def wavevectors(rng, n_modes, k0, dk, a, b, R) -> np.ndarray:
    """Integer wavevectors: isotropic directions with magnitudes in a band
    around k0, mapped by the volume-preserving ellipsoid R diag(s) R^T with
    s = (ab)^(1/3) (1/a, 1/b, 1), rounded, zero vectors dropped
    (gen_aniso_structures3d.py:131-151)."""
    v = rng.normal(size=(n_modes, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    q = v * rng.uniform(max(0.5, k0 - dk), k0 + dk, n_modes)[:, None]
    if not (a == 1.0 and b == 1.0):
        s = (a * b) ** (1.0 / 3.0) * np.array([1.0 / a, 1.0 / b, 1.0])
        q = q @ (R @ np.diag(s) @ R.T).T
    q = np.rint(q).astype(int)
    return q[np.any(q != 0, axis=1)]


def axis_points(size) -> np.ndarray:
    """Cell coordinates in [0, 1) of each axis (np.linspace without the end point)."""
    return np.linspace(0.0, 1.0, size, endpoint=False)


class Generator:
    """Draws samples of one configuration on one device."""

    def __init__(self, size=80, device=0, **cfg):
        self.size = size
        self.cfg = {**DEFAULTS, **cfg}
        self.ctx = _lib.context(device)
        self.pts = np.ascontiguousarray(axis_points(size))

    def structure(self, q, phases, porosity):
        """(solid [z, y, x] uint8, threshold) of one drawn mode set."""
        n = self.size
        solid = np.empty((n, n, n), np.uint8)
        t = C.c_double()
        qq = np.ascontiguousarray(q, dtype=np.int32)
        ph = np.ascontiguousarray(phases, dtype=np.float64)
        scale = float(np.sqrt(2.0 / len(qq)))
        self.ctx.check(self.ctx.L.lbm_trig_structure3d(
            self.ctx.h, n, len(qq), qq.ctypes.data_as(C.POINTER(C.c_int32)),
            ph.ctypes.data_as(C.POINTER(C.c_double)), self.pts.ctypes.data_as(C.POINTER(C.c_double)),
            scale, float(porosity), solid.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(t)))
        return solid, t.value

    def percolates(self, solid):
        nz, ny, nx = solid.shape
        p = (C.c_int * 3)()
        arr = np.ascontiguousarray(solid, dtype=np.uint8)
        self.ctx.check(self.ctx.L.lbm_percolates3d(self.ctx.h, arr.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                   nx, ny, nz, p))
        return bool(p[0]), bool(p[1]), bool(p[2])

    def sample(self, sample_id):
        """(solid, row) of one sample, or None when no draw percolates
        (gen_aniso_structures3d.py:208-266)."""
        c = self.cfg
        rng = np.random.default_rng(c["seed"] + sample_id)
        name, a_lo, a_hi = STRATA[sample_id % len(STRATA)]
        for attempt in range(c["max_attempts"]):
            a = float(rng.uniform(a_lo, a_hi))
            b = float(rng.uniform(1.0, a)) if a > 1.0 else 1.0
            R = rotation(rng)
            k0 = float(rng.uniform(c["k0_min"], c["k0_max"]))
            n_modes = int(rng.integers(c["modes_min"], c["modes_max"] + 1))
            porosity = float(rng.uniform(c["por_min"], c["por_max"]))
            q = wavevectors(rng, n_modes, k0, c["dk"], a, b, R)
            if len(q) < 5:
                continue
            phases = rng.uniform(0.0, np.pi, len(q))
            solid, thresh = self.structure(q, phases, porosity)
            if not all(self.percolates(solid)):
                continue
            por = float(1.0 - solid.mean())
            fname = (f"sample_{sample_id:06d}_str={name}_A={a:.2f}"
                     f"_B={b:.2f}_k0={k0:.2f}_por={por:.4f}.raw")
            row = {"sample_id": sample_id, "filename": fname, "stratum": name,
                   "aniso_A": a, "aniso_B": b, "shape": (b - 1.0) / (a - 1.0) if a > 1.0 else 0.0,
                   "e1_x": R[0, 0], "e1_y": R[1, 0], "e1_z": R[2, 0],
                   "e2_x": R[0, 1], "e2_y": R[1, 1], "e2_z": R[2, 1],
                   "k0": k0, "n_modes": len(q), "porosity": por, "porosity_target": porosity,
                   "threshold": thresh, "attempts": attempt + 1}
            return solid.astype(bool), row
        return None


def generate(output, n_samples, size=80, device=0, log=print, **cfg):
    """Write a dataset; returns the structures.csv rows."""
    import pandas as pd
    structures_dir = os.path.join(output, "structures")
    os.makedirs(structures_dir, exist_ok=True)
    gen = Generator(size=size, device=device, **cfg)
    rows = []
    for i in range(n_samples):
        got = gen.sample(i)
        if got is None:
            log(f"sample {i}: no percolating structure in {gen.cfg['max_attempts']} attempts")
            continue
        solid, row = got
        save_structure(os.path.join(structures_dir, row["filename"]), solid)
        rows.append(row)
    df = pd.DataFrame(rows)
    if len(df):
        df = df.sort_values("sample_id").reset_index(drop=True)
    df.to_csv(os.path.join(output, "structures.csv"), index=False)
    with open(os.path.join(output, "filelist.txt"), "w") as fh:
        for n in df.get("filename", []):
            fh.write(os.path.join(structures_dir, n) + "\n")
    log(f"kept {len(df)}/{n_samples} structures")
    return rows


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--output", required=True)
    p.add_argument("--n_samples", type=int, default=5000)
    p.add_argument("--size", type=int, default=80)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--k0_min", type=float, default=3.0)
    p.add_argument("--k0_max", type=float, default=7.0)
    p.add_argument("--dk", type=float, default=1.0)
    p.add_argument("--modes_min", type=int, default=20)
    p.add_argument("--modes_max", type=int, default=80)
    p.add_argument("--porosity_min", type=float, default=0.65)
    p.add_argument("--porosity_max", type=float, default=0.90)
    p.add_argument("--max_attempts", type=int, default=200)
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    generate(a.output, a.n_samples, size=a.size, device=a.device, seed=a.seed, k0_min=a.k0_min,
             k0_max=a.k0_max, dk=a.dk, modes_min=a.modes_min, modes_max=a.modes_max,
             por_min=a.porosity_min, por_max=a.porosity_max, max_attempts=a.max_attempts)
    return 0


if __name__ == "__main__":
    sys.exit(main())
