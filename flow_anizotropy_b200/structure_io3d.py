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


_HDR = np.dtype("<i4")


def _encode(solid) -> bytes:
    """Header + payload bytes of a [z, y, x] array of {0, 1}."""
    vox = np.asarray(solid)
    if vox.ndim != 3:
        raise ValueError(f"a .raw structure is 3D [z, y, x]; got an array of shape {vox.shape}")
    vox = vox.astype(np.uint8, copy=False)
    if vox.size and int(vox.max()) > 1:
        raise ValueError("voxel values must be 0 (pore) or 1 (solid)")
    dims = np.array(vox.shape[::-1], dtype=_HDR)          # nx, ny, nz
    return dims.tobytes() + np.ascontiguousarray(vox).tobytes()


def _decode(buf: bytes, where: str) -> np.ndarray:
    """[z, y, x] view of header + payload; ValueError when the sizes disagree."""
    if len(buf) < MAGIC_HEADER_BYTES:
        raise ValueError(f"{where}: {len(buf)} bytes, fewer than the {MAGIC_HEADER_BYTES}-byte header")
    nx, ny, nz = (int(d) for d in np.frombuffer(buf[:MAGIC_HEADER_BYTES], dtype=_HDR))
    payload = len(buf) - MAGIC_HEADER_BYTES
    if min(nx, ny, nz) < 0 or nx * ny * nz != payload:
        raise ValueError(f"{where}: dimensions {nx} x {ny} x {nz} do not match the "
                         f"{payload}-byte payload")
    return np.frombuffer(buf, dtype=np.uint8, offset=MAGIC_HEADER_BYTES).reshape(nz, ny, nx)


def save_structure(path, solid) -> Path:
    """Write a [z, y, x] array of {0, 1} (1 = solid) as a .raw file; returns the path.

    Same contract as the reference's writer (scripts/structure_io3d.py:40-52):
    ValueError for a non-3D or non-binary array."""
    path = Path(path)
    path.write_bytes(_encode(solid))
    return path


def load_structure(path) -> np.ndarray:
    """Read a .raw file as a read-only uint8 [z, y, x] array (1 = solid).

    Same contract as the reference's reader (scripts/structure_io3d.py:55-67):
    ValueError when the header's shape does not match the file size."""
    path = Path(path)
    return _decode(path.read_bytes(), str(path))


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
