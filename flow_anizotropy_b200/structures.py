"""Seeded synthetic voxel structures for the benchmark workloads.

All arrays are uint8 ``[z, y, x]``, 1 = solid, periodic in every axis.

* ``sphere_packing``      overlapping spheres at uniform random integer centres,
                          added one at a time until the porosity first drops to
                          the target (the 64^3, r = 6, phi = 0.60 single solve);
* ``ellipsoid_packing``   the same with axis-aligned ellipsoids (the 128^3
                          prolate (4,4,12) precision-study packing);
* ``grf_structure``       FFT-filtered white noise with an anisotropic Gaussian
                          kernel, thresholded at the porosity quantile, keeping
                          the largest pore cluster that spans the chosen axis
                          (the 512^3 low-porosity solve);
* ``batch_mix``           the 256-structure uneven-size mix;
* ``percolates``          6-connected pore percolation per axis.

Percolation follows the intent of scripts/gen_aniso_structures3d.py:184-201
(a pore cluster that crosses the periodic cell): a cluster percolates along an
axis when it connects the two faces normal to that axis, with the cell wrapped
periodically in the other two axes.  Shapes are added in chunks while the
porosity is far above the target and one at a time near it, stopping at the
first addition that brings the porosity to the target or below; every
structure is a deterministic function of its seed.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["sphere_packing", "ellipsoid_packing", "grf_structure", "percolates",
           "largest_spanning_cluster", "batch_mix", "plain_64", "precision_128", "large_grf",
           "serving_request"]


# ------------------------------------------------------------ percolation ---
def _labels(pore):
    from scipy.ndimage import label
    lab, n = label(pore)          # 6-connectivity (the default cross structure)
    return lab, n


class _UF:
    def __init__(self, n):
        self.p = np.arange(n + 1)

    def find(self, a):
        p = self.p
        root = a
        while p[root] != root:
            root = p[root]
        while p[a] != root:
            p[a], a = root, p[a]
        return root

    def union(self, a, b):
        ra, rb = self.find(a), self.find(b)
        if ra != rb:
            self.p[max(ra, rb)] = min(ra, rb)


def _merged_labels(lab, n, wrap_axes):
    """Label map with clusters merged across the periodic faces of wrap_axes."""
    uf = _UF(n)
    for ax in wrap_axes:
        lo = np.take(lab, 0, axis=ax).ravel()
        hi = np.take(lab, -1, axis=ax).ravel()
        both = (lo > 0) & (hi > 0)
        pairs = np.unique(np.stack([lo[both], hi[both]], axis=1), axis=0)
        for a, b in pairs:
            uf.union(int(a), int(b))
    roots = np.array([uf.find(i) for i in range(n + 1)])
    return roots


def percolates(solid):
    """(perc_x, perc_y, perc_z) for the pore phase of a periodic cell."""
    pore = np.asarray(solid) == 0
    lab, n = _labels(pore)
    if n == 0:
        return (False, False, False)
    out = []
    for ax_arr in (2, 1, 0):                         # x, y, z on a [z, y, x] array
        others = [a for a in (0, 1, 2) if a != ax_arr]
        roots = _merged_labels(lab, n, others)
        lo = set(roots[np.unique(np.take(lab, 0, axis=ax_arr))]) - {0}
        hi = set(roots[np.unique(np.take(lab, -1, axis=ax_arr))]) - {0}
        out.append(bool(lo & hi))
    return tuple(out)


def largest_spanning_cluster(solid, axis="z"):
    """Keep only the largest pore cluster spanning `axis`; all other pore becomes solid.

    Returns (new_solid, found)."""
    ax_arr = {"x": 2, "y": 1, "z": 0}[axis]
    pore = np.asarray(solid) == 0
    lab, n = _labels(pore)
    if n == 0:
        return np.ones_like(solid, dtype=np.uint8), False
    others = [a for a in (0, 1, 2) if a != ax_arr]
    roots = _merged_labels(lab, n, others)
    lo = set(roots[np.unique(np.take(lab, 0, axis=ax_arr))]) - {0}
    hi = set(roots[np.unique(np.take(lab, -1, axis=ax_arr))]) - {0}
    span = sorted(lo & hi)
    if not span:
        return np.asarray(solid, dtype=np.uint8), False
    rl = roots[lab]
    sizes = np.bincount(rl.ravel(), minlength=n + 1)
    best = max(span, key=lambda r: sizes[r])
    return (rl != best).astype(np.uint8), True


# ------------------------------------------------------------ packings ------
def _shape_offsets(semi):
    """Integer offsets (dz, dy, dx) inside an axis-aligned ellipsoid with semi-axes (ax, ay, az)."""
    ax, ay, az = semi
    rx, ry, rz = int(math.ceil(ax)), int(math.ceil(ay)), int(math.ceil(az))
    z, y, x = np.mgrid[-rz:rz + 1, -ry:ry + 1, -rx:rx + 1]
    inside = (x / ax) ** 2 + (y / ay) ** 2 + (z / az) ** 2 <= 1.0
    return z[inside].astype(np.int64), y[inside].astype(np.int64), x[inside].astype(np.int64)


def _pack(shape, semi, porosity, rng, max_shapes=10_000_000):
    nz, ny, nx = shape
    N = nz * ny * nx
    dz, dy, dx = _shape_offsets(semi)
    vs = len(dz)
    flat = np.zeros(N, np.uint8)
    nsolid = 0

    def indices(c):                       # c: (m, 3) integer centres (z, y, x)
        zz = (c[:, 0:1] + dz[None, :]) % nz
        yy = (c[:, 1:2] + dy[None, :]) % ny
        xx = (c[:, 2:3] + dx[None, :]) % nx
        return ((zz * ny + yy) * nx + xx).ravel()

    added = 0
    single = False
    while True:
        phi = (N - nsolid) / N
        if phi <= porosity:
            break
        # Boolean-model estimate of the shapes still needed; add half of it at
        # once while that is many, then one at a time
        need = math.log(phi / porosity) * N / vs if porosity > 0 else 1.0
        m = int(need * 0.5)
        if m >= 16 and not single:
            c = np.stack([rng.integers(0, nz, m), rng.integers(0, ny, m), rng.integers(0, nx, m)], axis=1)
            idx = indices(c)
            new = np.count_nonzero(flat[idx] == 0)     # upper bound on newly solid voxels
            if (N - nsolid - new) / N <= porosity:
                before = flat.copy()
                flat[idx] = 1
                if (N - int(flat.sum())) / N < porosity:
                    flat = before                      # overshoot: undo, go one at a time
                    single = True
                    continue
            else:
                flat[idx] = 1
            nsolid = int(flat.sum())
            added += m
        else:
            c = np.array([[rng.integers(0, nz), rng.integers(0, ny), rng.integers(0, nx)]])
            idx = indices(c)
            nsolid += int(np.count_nonzero(flat[np.unique(idx)] == 0))
            flat[idx] = 1
            added += 1
        if added > max_shapes:
            raise RuntimeError("packing did not reach the target porosity")
    return flat.reshape(shape)


def sphere_packing(n, radius, porosity, seed, percolate=(True, False, False), max_tries=50):
    """Overlapping spheres in an n^3 (or (nz,ny,nx)) cell until phi <= porosity; reseeded
    (seed, seed+1000, ...) until it percolates along every axis flagged in `percolate` (x, y, z)."""
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    for t in range(max_tries):
        rng = np.random.default_rng(seed + 1000 * t)
        s = _pack(shape, (radius, radius, radius), porosity, rng)
        p = percolates(s)
        if all(p[i] for i in range(3) if percolate[i]):
            return s
    raise RuntimeError("no percolating sphere packing found")


def ellipsoid_packing(n, semi, porosity, seed, percolate=(True, True, True), max_tries=50):
    """Overlapping axis-aligned ellipsoids, semi-axes (ax, ay, az) in voxels."""
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    for t in range(max_tries):
        rng = np.random.default_rng(seed + 1000 * t)
        s = _pack(shape, semi, porosity, rng)
        p = percolates(s)
        if all(p[i] for i in range(3) if percolate[i]):
            return s
    raise RuntimeError("no percolating ellipsoid packing found")


def grf_structure(n, sigma=(3.0, 3.0, 9.0), porosity=0.15, seed=0, axis="z", max_tries=20):
    """Gaussian random field: white noise convolved (via FFT) with an anisotropic
    Gaussian of std sigma = (sx, sy, sz) voxels, pore where the field is below its
    `porosity` quantile, then only the largest pore cluster spanning `axis` kept."""
    from scipy import fft as sfft
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    nz, ny, nx = shape
    sx, sy, sz = sigma
    for t in range(max_tries):
        rng = np.random.default_rng(seed + 1000 * t)
        noise = rng.standard_normal(shape, dtype=np.float32)
        spec = sfft.rfftn(noise, workers=-1)
        del noise
        kz = (2 * np.pi * sfft.fftfreq(nz)).astype(np.float32)[:, None, None]
        ky = (2 * np.pi * sfft.fftfreq(ny)).astype(np.float32)[None, :, None]
        kx = (2 * np.pi * sfft.rfftfreq(nx)).astype(np.float32)[None, None, :]
        spec *= np.exp(-0.5 * (kx * kx * sx * sx + ky * ky * sy * sy + kz * kz * sz * sz))
        field = sfft.irfftn(spec, s=shape, workers=-1).astype(np.float32)
        del spec
        thr = np.quantile(field[:: max(1, nz // 128)].ravel(), porosity) if field.size > 2**26 \
            else np.quantile(field, porosity)
        solid = (field >= thr).astype(np.uint8)
        del field
        solid, ok = largest_spanning_cluster(solid, axis)
        if ok:
            return solid
    raise RuntimeError("no spanning GRF cluster found")


# --------------------------------------------------------- named workloads --
def plain_64(seed=0):
    """64^3, spheres r = 6 until phi <= 0.60, percolating along x."""
    return sphere_packing(64, 6.0, 0.60, seed, percolate=(True, False, False))


def precision_128(seed=0):
    """128^3 prolate ellipsoids (4, 4, 12) along z, phi = 0.45, percolating in x, y, z."""
    return ellipsoid_packing(128, (4.0, 4.0, 12.0), 0.45, seed, percolate=(True, True, True))


def large_grf(seed=0, n=512):
    """512^3 GRF, sigma = (3, 3, 9), phi = 0.15, largest cluster spanning z."""
    return grf_structure(n, (3.0, 3.0, 9.0), 0.15, seed, axis="z")


def batch_mix(count=256, seed=0, sizes=(48, 64, 96, 128, 160)):
    """Descriptions of the uneven batch: half sphere packings (r in U[3,8],
    phi in U[0.35,0.75]), half ellipsoid packings (axis-aligned stretch U[1,4]
    of a base radius in U[3,8] along a random axis, phi in U[0.35,0.65]).
    Returns a list of dicts; ``make(d)`` builds the array."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(sizes))
        if i % 2 == 0:
            r = float(rng.uniform(3, 8))
            out.append(dict(kind="spheres", n=n, semi=(r, r, r), porosity=float(rng.uniform(0.35, 0.75)),
                            seed=int(rng.integers(0, 2**31 - 1))))
        else:
            r = float(rng.uniform(3, 8))
            stretch = float(rng.uniform(1, 4))
            ax = int(rng.integers(0, 3))
            semi = [r, r, r]
            semi[ax] = r * stretch
            out.append(dict(kind="ellipsoids", n=n, semi=tuple(semi),
                            porosity=float(rng.uniform(0.35, 0.65)),
                            seed=int(rng.integers(0, 2**31 - 1))))
    return out


def disc_packing_2d(seed, solid_fraction, n=256, rmin=4, rmax=12):
    """Periodic 2D cell (the D2Q9 reference's fixed 256 x 256) of overlapping
    discs, radius U{rmin..rmax-1}, added until the solid fraction reaches
    ``solid_fraction``; [y, x] uint8, 1 = solid."""
    rng = np.random.default_rng(seed)
    s = np.zeros((n, n), np.uint8)
    yy, xx = np.mgrid[0:n, 0:n]
    while s.mean() < solid_fraction:
        cx, cy, r = rng.integers(0, n), rng.integers(0, n), rng.integers(rmin, rmax)
        dx = np.minimum(np.abs(xx - cx), n - np.abs(xx - cx))
        dy = np.minimum(np.abs(yy - cy), n - np.abs(yy - cy))
        s[dx * dx + dy * dy <= r * r] = 1
    return s


def make(d):
    """Build one structure from a batch_mix / serving description."""
    if d["kind"] == "grf":
        return grf_structure(d["n"], (3.0, 3.0, 9.0), d["porosity"], d["seed"], axis="z")
    perc = (True, True, True)
    return ellipsoid_packing(d["n"], d["semi"], d["porosity"], d["seed"], percolate=perc)


def serving_request(i, seed=0):
    """Request i of the serving stream: a batch_mix-style structure, and a 256^3
    GRF (phi in U[0.15, 0.35]) for every 20th request."""
    rng = np.random.default_rng(seed * 1_000_003 + i)
    if i % 20 == 19:
        return dict(kind="grf", n=256, porosity=float(rng.uniform(0.15, 0.35)),
                    seed=int(rng.integers(0, 2**31 - 1)))
    return batch_mix(1, seed=int(rng.integers(0, 2**31 - 1)))[0]
