"""The ``.raw`` voxel format of the 3D solver (scripts/structure_io3d.py:1-72).

    bytes  0..11   three int32, little-endian: nx, ny, nz
    bytes 12..     nx*ny*nz uint8, 1 = solid, 0 = pore, x fastest

Arrays are indexed ``[z, y, x]``.  ``read_raw_checked`` applies the solver's
own validation (LMB3d/lbm3d-perm.cpp:174-193): header present, positive
dimensions, exact payload length, binary values, at least one pore voxel;
its messages are the solver's ``die()`` messages.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

__all__ = ["load_structure", "save_structure", "porosity", "read_raw_checked",
           "StructureError", "MAGIC_HEADER_BYTES"]

MAGIC_HEADER_BYTES = 12


class StructureError(ValueError):
    """Input the reference solver would reject with exit code 2."""


def save_structure(path, solid) -> Path:
    """Write a (nz, ny, nx) {0,1} array as .raw (scripts/structure_io3d.py:40-52)."""
    solid = np.ascontiguousarray(solid).astype(np.uint8)
    if solid.ndim != 3:
        raise ValueError(f"expected a 3D array, got shape {solid.shape}")
    if solid.size and solid.max() > 1:
        raise ValueError("structure must be binary (0 = pore, 1 = solid)")
    nz, ny, nx = solid.shape
    path = Path(path)
    with open(path, "wb") as fh:
        fh.write(np.array([nx, ny, nz], dtype="<i4").tobytes())
        fh.write(solid.tobytes())
    return path


def load_structure(path) -> np.ndarray:
    """Read a .raw as uint8 (nz, ny, nx) (scripts/structure_io3d.py:55-67)."""
    path = Path(path)
    raw = path.read_bytes()
    if len(raw) < MAGIC_HEADER_BYTES:
        raise ValueError(f"{path}: too short to hold a header")
    nx, ny, nz = (int(v) for v in np.frombuffer(raw, dtype="<i4", count=3))
    expect = MAGIC_HEADER_BYTES + nx * ny * nz
    if len(raw) != expect:
        raise ValueError(
            f"{path}: header says {nx}x{ny}x{nz} -> {expect} bytes, file has {len(raw)}")
    return np.frombuffer(raw, dtype=np.uint8, offset=MAGIC_HEADER_BYTES).reshape(nz, ny, nx)


def porosity(solid) -> float:
    return float(1.0 - np.asarray(solid).mean())


def read_raw_checked(path) -> np.ndarray:
    """Read a .raw with the solver's checks; raises StructureError with its messages."""
    path = str(path)
    try:
        raw = Path(path).read_bytes()
    except OSError:
        raise StructureError("cannot open " + path) from None
    if len(raw) < MAGIC_HEADER_BYTES:
        raise StructureError("cannot read header of " + path)
    nx, ny, nz = (int(v) for v in np.frombuffer(raw, dtype="<i4", count=3))
    if nx <= 0 or ny <= 0 or nz <= 0:
        raise StructureError("bad dimensions in " + path)
    n = nx * ny * nz
    if len(raw) < MAGIC_HEADER_BYTES + n:
        raise StructureError("truncated payload in " + path)
    if len(raw) > MAGIC_HEADER_BYTES + n:
        raise StructureError("trailing bytes in " + path)
    arr = np.frombuffer(raw, dtype=np.uint8, offset=MAGIC_HEADER_BYTES).reshape(nz, ny, nx)
    if arr.max() > 1:
        raise StructureError("non-binary voxel")
    if not (arr == 0).any():
        raise StructureError("structure has no pore space")
    return arr
