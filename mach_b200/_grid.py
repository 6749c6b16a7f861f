"""Voxel-grid detection for tiling hints.

Scan grids are usually a flattened ``meshgrid(x, y, z, indexing="ij")`` (z contiguous).
Knowing the (slow, mid, fast) extents lets the multi-frame kernel give each CTA a compact
block of voxels whose sample windows overlap.  The hint only reorders which CTA computes
which voxel; every voxel is still computed from its own coordinates, so a wrong or
missing hint costs speed, never correctness.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from mach_b200 import _dlpack

_cache: dict = {}


def _detect_host(pts: np.ndarray) -> tuple[int, int, int] | None:
    n = pts.shape[0]
    if n < 2 or pts.ndim != 2 or pts.shape[1] != 3:
        return None
    xy = pts[:, :2]
    change = np.nonzero(np.any(xy[1:] != xy[0], axis=1))[0]
    nf = int(change[0]) + 1 if change.size else n
    if n % nf:
        return None
    slab_x = pts[::nf, 0]
    xchange = np.nonzero(slab_x[1:] != slab_x[0])[0]
    nm = int(xchange[0]) + 1 if xchange.size else slab_x.shape[0]
    if n % (nf * nm):
        return None
    # Only shapes the tiler can use: 8 voxels along the contiguous axis, 4 along the middle one.
    if nf < 8 or (nm != 1 and nm < 4):
        return None
    return (n // (nf * nm), nm, nf)


def detect(scan_coords_m: Any) -> tuple[int, int, int] | None:
    """(slow, mid, fast) extents of a meshgrid-ordered scan, or None.  Cached per array version."""
    if _dlpack.is_torch(scan_coords_m):
        key = ("torch", scan_coords_m.data_ptr(), tuple(scan_coords_m.shape), scan_coords_m._version,
               str(scan_coords_m.device))
        if key not in _cache:
            _cache[key] = _detect_host(scan_coords_m.detach().to("cpu", copy=True).numpy())
        return _cache[key]
    if isinstance(scan_coords_m, np.ndarray):
        return _detect_host(scan_coords_m)
    return None
