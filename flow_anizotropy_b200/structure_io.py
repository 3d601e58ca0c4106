"""2D structure readers of the D2Q9 solver (LMB2d/lbm.cpp:459-536).

Arrays are indexed ``[y, x]`` (= image ``[row, col]``), 1 = solid:

* GIF: a pixel is pore when its red channel is > 0 (``read_from_gif``,
  LMB2d/lbm.cpp:459-473; mirrored by scripts/structure_io.py:44-54);
* PPM (P3 text, four header lines, R G B per pixel, pore when R != 0):
  ``read_from_ppm``, LMB2d/lbm.cpp:474-501;
* DAT (whitespace-separated integers, y outer, x inner, 0 = pore):
  ``read_from_dat``, LMB2d/lbm.cpp:502-520.

PPM and DAT carry no size: like the reference (whose cell is the compile-time
256 x 256 of LMB2d/lbm.h:24-25) they are read as ``nx`` x ``ny`` = 256 x 256
unless a size is given.  Missing trailing values read as 0 (pore), as the
reference's ``atoi`` of an empty token does.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

DEFAULT_SIZE = 256


def _tokens(path):
    return Path(path).read_text(errors="replace").split()


def load_dat(path, nx: int = DEFAULT_SIZE, ny: int = DEFAULT_SIZE) -> np.ndarray:
    toks = _tokens(path)
    out = np.zeros((ny, nx), np.uint8)
    vals = np.array([_atoi(t) for t in toks[: nx * ny]], dtype=np.int64)
    flat = out.reshape(-1)
    flat[: len(vals)] = (vals != 0).astype(np.uint8)
    return out


def load_ppm(path, nx: int = DEFAULT_SIZE, ny: int = DEFAULT_SIZE) -> np.ndarray:
    lines = Path(path).read_text(errors="replace").splitlines()
    toks = " ".join(lines[4:]).split()
    out = np.ones((ny, nx), np.uint8)
    flat = out.reshape(-1)
    for i in range(nx * ny):
        r = toks[3 * i] if 3 * i < len(toks) else ""
        flat[i] = 0 if _atoi(r) else 1
    return out


def load_gif(path) -> np.ndarray:
    from PIL import Image
    with Image.open(path) as im:
        rgb = np.array(im.convert("RGB"))
    return (rgb[..., 0] == 0).astype(np.uint8)


def load_structure2d(path, nx: int = DEFAULT_SIZE, ny: int = DEFAULT_SIZE) -> np.ndarray:
    """Dispatch on the suffix as ``generate()`` does (LMB2d/lbm.cpp:522-530)."""
    p = str(path)
    if p.endswith(".ppm"):
        return load_ppm(p, nx, ny)
    if p.endswith(".gif"):
        return load_gif(p)
    return load_dat(p, nx, ny)


def save_dat(path, solid) -> Path:
    """Write the text form read_from_dat expects (y outer, x inner, 1 = solid)."""
    solid = np.asarray(solid, dtype=np.uint8)
    with open(path, "w") as fh:
        for row in solid:
            fh.write(" ".join(str(int(v)) for v in row))
            fh.write("\n")
    return Path(path)


def _atoi(tok: str) -> int:
    s = tok.strip()
    i, sign = 0, 1
    if i < len(s) and s[i] in "+-":
        sign = -1 if s[i] == "-" else 1
        i += 1
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    return sign * int(s[i:j]) if j > i else 0
