"""Dose .bin files in the reference's layout (src/tests/wrapper_integration_test.cu:
3843-3859): a 36-byte header of int32 dims (x, y, z), float32 spacing (x, y, z)
and float32 origin (x, y, z), then the float32 dose [Z][Y][X] with x fastest.
The header is PbsDoseBinHeader of include/pbs_layouts.h."""
from __future__ import annotations

from pathlib import Path

import numpy as np

HEADER_DTYPE = np.dtype([("dims", "<i4", 3), ("spacing", "<f4", 3), ("origin", "<f4", 3)])
assert HEADER_DTYPE.itemsize == 36


def write_dose_bin(path: str | Path, dose: np.ndarray, spacing, origin) -> None:
    """Write `dose` [Z][Y][X] with its voxel spacing and origin (x, y, z order)."""
    d = np.ascontiguousarray(dose, dtype="<f4")
    if d.ndim != 3:
        raise ValueError("dose must be a [Z][Y][X] array")
    h = np.zeros((), HEADER_DTYPE)
    h["dims"] = (d.shape[2], d.shape[1], d.shape[0])
    h["spacing"] = spacing
    h["origin"] = origin
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(d.tobytes())


def read_dose_bin(path: str | Path):
    """(dose [Z][Y][X] float32, spacing (x, y, z), origin (x, y, z)) of a dose .bin."""
    raw = Path(path).read_bytes()
    if len(raw) < HEADER_DTYPE.itemsize:
        raise ValueError(f"{path}: shorter than the 36-byte header")
    h = np.frombuffer(raw[:HEADER_DTYPE.itemsize], HEADER_DTYPE)[0]
    nx, ny, nz = (int(v) for v in h["dims"])
    n = nx * ny * nz
    if nx <= 0 or ny <= 0 or nz <= 0 or len(raw) != HEADER_DTYPE.itemsize + 4 * n:
        raise ValueError(f"{path}: payload does not match the header's dims {nx}x{ny}x{nz}")
    dose = np.frombuffer(raw[HEADER_DTYPE.itemsize:], "<f4").reshape(nz, ny, nx).copy()
    return dose, tuple(float(v) for v in h["spacing"]), tuple(float(v) for v in h["origin"])
