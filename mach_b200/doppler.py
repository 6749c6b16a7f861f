"""Power-Doppler imaging fused with the beamformer.

mach's Doppler example beamforms an ensemble and then takes, per scan point, the sum over
frames of the squared magnitude (``np.square(np.abs(result)).sum(axis=-1)``,
examples/doppler.py:252; tests/compare/test_pymust.py:317-318).  :func:`power_doppler`
returns that image directly.  When the ensemble kernel runs the job, the squares are summed
inside the kernel as each frame block finishes, and the ``[n_points, n_frames]`` image is
never written.
"""

from __future__ import annotations

from typing import Any

from mach_b200._cuda_impl import InterpolationType
from mach_b200.experimental import _compound


def power_doppler(
    channel_data: Any,
    rx_coords_m: Any,
    scan_coords_m: Any,
    tx_wave_arrivals_s: Any,
    out: Any = None,
    *,
    rx_start_s: float,
    sampling_freq_hz: float,
    f_number: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float | None = None,
    tukey_alpha: float = 0.5,
    interp_type: InterpolationType = InterpolationType.Linear,
    channel_scale: float = 1.0,
    sync: bool = True,
    grid_shape: Any = None,
    kernel: str = "auto",
    window_rows: int = 0,
    delay: str = "auto",
) -> Any:
    """Power-Doppler image ``sum_f |beamform(...)[:, f]|^2`` as float32 ``[n_points]``.

    Arguments are those of :func:`mach_b200.experimental.beamform`.  A GPU ``out`` is
    accumulated into, a CPU ``out`` is overwritten.  The frame blocks of a scan point are
    added in whatever order they finish, so the last bits can differ between runs
    (relative 1e-7).
    """
    return _compound(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, rx_start_s=rx_start_s,
                     sampling_freq_hz=sampling_freq_hz, f_number=f_number, sound_speed_m_s=sound_speed_m_s,
                     modulation_freq_hz=modulation_freq_hz, tukey_alpha=tukey_alpha, interp_type=interp_type,
                     channel_scale=channel_scale, sync=sync, grid_shape=grid_shape, kernel=kernel,
                     window_rows=window_rows, lanes_per_voxel=0, tx_chunk=0, delay=delay, power=True)
