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


class TransmitWaves:
    """Transmit wavefronts that the beamformer evaluates on the GPU.

    Pass an instance as ``tx_wave_arrivals_s`` of :func:`mach_b200.experimental.beamform`
    (or :func:`mach_b200.doppler.power_doppler`) instead of the ``[n_transmits, n_points]``
    arrivals array: each (point, transmit) arrival is then computed on the GPU from the
    wave's origin and direction or focus, in FP64 and rounded to FP32, the same as
    ``plane(...) / sound_speed`` or ``spherical(...) / sound_speed`` evaluated on the host.
    The array (4 bytes per point and transmit, 79 MB for 75 transmits on 512x512) is formed
    in device memory and never crosses the host link.
    """

    model = 0

    def __init__(self, origin_m: Any, vectors: Any, time_offset_s: Any = 0.0):
        import numpy as np

        origin = np.asarray(origin_m, dtype=np.float64)
        vec = np.atleast_2d(np.asarray(vectors, dtype=np.float64))
        n = vec.shape[0]
        origin = np.broadcast_to(origin, (n, 3))
        offset = np.broadcast_to(np.asarray(time_offset_s, dtype=np.float64), (n,))
        self.table = np.zeros((n, 8), dtype=np.float64)
        self.table[:, 0:3] = origin
        self.table[:, 3:6] = vec
        self.table[:, 6] = offset

    @property
    def n_transmits(self) -> int:
        return int(self.table.shape[0])

    def __len__(self) -> int:
        return self.n_transmits

    def arrivals(self, points_m: Any, sound_speed_m_s: float) -> Any:
        """The ``[n_transmits, n_points]`` float64 arrivals the GPU computes, on the host."""
        import numpy as np

        pts = np.asarray(points_m, dtype=np.float64)
        rows = [self._distance(row[0:3], pts, row[3:6]) / sound_speed_m_s + row[6] for row in self.table]
        return np.stack(rows)


class PlaneWaves(TransmitWaves):
    """Plane waves: ``origin_m`` ``[3]`` or ``[n, 3]``, unit ``directions`` ``[n, 3]``."""

    model = 1

    def __init__(self, origin_m: Any, directions: Any, time_offset_s: Any = 0.0):
        import numpy as np

        d = np.atleast_2d(np.asarray(directions, dtype=np.float64))
        if not np.all(np.abs(np.linalg.norm(d, axis=-1) - 1) < 1e-6):
            raise ValueError("direction must be a unit vector")
        super().__init__(origin_m, d, time_offset_s)

    @staticmethod
    def _distance(origin, points, direction):
        return plane(origin, points, direction)


class SphericalWaves(TransmitWaves):
    """Focused or diverging waves: ``origin_m`` ``[3]`` or ``[n, 3]``, ``foci_m`` ``[n, 3]``."""

    model = 2

    @staticmethod
    def _distance(origin, points, focus):
        return spherical(origin, points, focus)

