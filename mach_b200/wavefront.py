"""Transmit-arrival *distances* for plane and spherical waves (mirror of src/mach/wavefront.py).

Divide by the speed of sound to get ``tx_wave_arrivals_s`` for :func:`mach_b200.beamform`.
Evaluated on the host in the caller's precision (float64 for default NumPy arrays); the
beamformer receives them as float32, as mach does (src/mach/kernel.py:231-233).
"""

from __future__ import annotations

from typing import Any

from mach_b200._array_api import array_namespace


def plane(origin_m: Any, points_m: Any, direction: Any) -> Any:
    """Plane-wave distance ``(points - origin) . direction`` (src/mach/wavefront.py:8-50).

    ``direction`` must be a unit vector (tolerance 1e-6), else ``ValueError``.
    Negative distances (points behind the origin) are returned as is.
    """
    xp = array_namespace(origin_m, points_m, direction)
    origin_m, points_m, direction = (xp.asarray(a) for a in (origin_m, points_m, direction))
    norm = xp.vector_norm(direction, axis=-1)
    if not float(xp.abs(norm - 1)) < 1e-6:
        raise ValueError("direction must be a unit vector")
    return xp.vecdot(points_m - origin_m, direction, axis=-1)


def spherical(origin_m: Any, points_m: Any, focus_m: Any) -> Any:
    """Focused or diverging wave distance (src/mach/wavefront.py:53-116).

    ``|origin - focus| * sign(focus_z - origin_z) - |focus - point| * sign(focus_z - point_z)``:
    zero at the transmitting origin; a focus in front of the origin is a focused wave,
    a focus behind it (a virtual source) a diverging wave.
    """
    xp = array_namespace(origin_m, points_m, focus_m)
    origin_m, points_m, focus_m = (xp.asarray(a) for a in (origin_m, points_m, focus_m))
    origin_focus = xp.vector_norm(origin_m - focus_m, axis=-1)
    focus_point = xp.vector_norm(focus_m - points_m, axis=-1)
    origin_sign = xp.sign(focus_m[2] - origin_m[2])
    point_sign = xp.sign(focus_m[2] - points_m[..., 2])
    return origin_focus * origin_sign - focus_point * point_sign
