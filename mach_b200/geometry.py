"""Angle conversions for transmit directions (mirror of src/mach/geometry.py).

``ultrasound_angles_to_cartesian`` follows mach's "ultrasound convention": rotate by
azimuth about y, then by elevation about x (src/mach/geometry.py:31-86);
``spherical_to_cartesian`` is the ISO 80000-2 physics convention
(src/mach/geometry.py:89-132).  Scalars in give a tuple of floats; arrays give
``[..., 3]`` arrays of the same namespace.
"""

from __future__ import annotations

import math
import numbers
from typing import Any

from mach_b200._array_api import array_namespace


def _prepare(*inputs: Any):
    if all(isinstance(x, numbers.Real) for x in inputs):
        return math, inputs
    xp = array_namespace(*[x for x in inputs if hasattr(x, "shape")])
    return xp, tuple(xp.asarray(x) if isinstance(x, numbers.Real) else x for x in inputs)


def _finish(xp, x, y, z):
    if xp is math:
        return (x, y, z)
    return xp.stack((x, y, z), axis=-1)


def ultrasound_angles_to_cartesian(azimuth_rad: Any, elevation_rad: Any, radius_m: Any = 1) -> Any:
    """(azimuth, elevation, radius) -> (x, y, z) = r (sin az, sin el cos az, cos el cos az)."""
    xp, (az, el, r) = _prepare(azimuth_rad, elevation_rad, radius_m)
    x = r * xp.sin(az)
    y = r * xp.sin(el) * xp.cos(az)
    z = r * xp.cos(el) * xp.cos(az)
    return _finish(xp, x, y, z)


def spherical_to_cartesian(theta_rad: Any, phi_rad: Any, radius_m: Any = 1) -> Any:
    """(polar theta, azimuthal phi, radius) -> (r sin t cos p, r sin t sin p, r cos t)."""
    xp, (theta, phi, r) = _prepare(theta_rad, phi_rad, radius_m)
    x = r * xp.sin(theta) * xp.cos(phi)
    y = r * xp.sin(theta) * xp.sin(phi)
    z = r * xp.cos(theta)
    return _finish(xp, x, y, z)
