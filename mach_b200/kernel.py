"""Public single-transmit ``beamform`` (mirror of mach's src/mach/kernel.py:22-292).

Same signature, defaults, dtype promotion, contiguity handling, output allocation
and error types as mach; the work is done by the sm_100a kernels behind
``mach_b200._cuda_impl``.
"""

from __future__ import annotations

from typing import Any

from mach_b200 import _dlpack
from mach_b200._array_api import array_namespace, is_writeable_array
from mach_b200._check import ensure_contiguous, is_contiguous
from mach_b200._cuda_impl import InterpolationType, __nvcc_version__  # noqa: F401
from mach_b200._cuda_impl import beamform as nb_beamform

__all__ = ["InterpolationType", "beamform", "nb_beamform"]


def _describe(x: Any) -> tuple[type, Any]:
    return type(x), getattr(x, "dtype", None)


def _is_array(x: Any) -> bool:
    return hasattr(x, "shape") and hasattr(x, "dtype") and (hasattr(x, "__dlpack__") or hasattr(x, "__array_interface__"))


def _is_numeric(x: Any) -> bool:
    return _is_array(x) and array_namespace(x).is_numeric(x)


def _is_real(x: Any) -> bool:
    return _is_array(x) and array_namespace(x).is_real(x)


def beamform(
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
) -> Any:
    """Delay-and-sum beamforming of one transmit on the GPU.

    Args mirror ``mach.beamform``: ``channel_data[n_rx, n_samples, n_frames]`` (float32 RF
    or complex64 IQ), ``rx_coords_m[n_rx, 3]``, ``scan_coords_m[n_scan, 3]``,
    ``tx_wave_arrivals_s[n_scan]`` (use ``wavefront.plane(...) / c`` or
    ``wavefront.spherical(...) / c``), optional ``out[n_scan, n_frames]``.
    A GPU ``out`` is accumulated into; without ``out`` a zero-filled array of the
    input's namespace is created and returned.
    """
    if not _is_numeric(channel_data):
        t, d = _describe(channel_data)
        raise TypeError(f"channel_data must be array with dtype=numeric, got type={t}, dtype={d}")
    if not _is_real(rx_coords_m):
        t, d = _describe(rx_coords_m)
        raise TypeError(f"rx_coords_m must be array with dtype=Real, got type={t}, dtype={d}")
    if not _is_real(scan_coords_m):
        t, d = _describe(scan_coords_m)
        raise TypeError(f"scan_coords_m must be array with dtype=Real, got type={t}, dtype={d}")
    if not _is_real(tx_wave_arrivals_s):
        t, d = _describe(tx_wave_arrivals_s)
        raise TypeError(f"tx_wave_arrivals_s must be array with dtype=Real, got type={t}, dtype={d}")
    if out is not None and not _is_numeric(out):
        t, d = _describe(out)
        raise TypeError(f"out must be array with dtype=numeric, got type={t}, dtype={d}")

    xp_data = array_namespace(channel_data)
    xp_coords = array_namespace(rx_coords_m)
    xp_grid = array_namespace(scan_coords_m)
    xp_idt = array_namespace(tx_wave_arrivals_s)
    for arr, name in ((channel_data, "channel_data"), (rx_coords_m, "rx_coords_m"),
                      (scan_coords_m, "scan_coords_m"), (tx_wave_arrivals_s, "tx_wave_arrivals_s")):
        try:
            _dlpack.dlpack_device(arr)
        except TypeError:
            raise TypeError(f"Array '{name}' does not support DLPack protocol") from None
    if out is not None:
        try:
            _dlpack.dlpack_device(out)
        except TypeError:
            raise TypeError("Array 'out' does not support DLPack protocol") from None

    rx_coords_m = xp_coords.astype(rx_coords_m, xp_coords.float32, copy=False)
    scan_coords_m = xp_grid.astype(scan_coords_m, xp_grid.float32, copy=False)
    tx_wave_arrivals_s = xp_idt.astype(tx_wave_arrivals_s, xp_idt.float32, copy=False)

    n_frames = channel_data.shape[2]
    n_scan = scan_coords_m.shape[0]

    is_complex = xp_data.is_complex(channel_data)
    if is_complex:
        channel_data = xp_data.astype(channel_data, xp_data.complex64, copy=False)
        output_dtype = xp_data.complex64
        if modulation_freq_hz is None:
            raise ValueError(
                "modulation_freq_hz is required for complex phase-correction. set it to 0 if no demodulation was used."
            )
    else:
        channel_data = xp_data.astype(channel_data, xp_data.float32, copy=False)
        output_dtype = xp_data.float32
        if modulation_freq_hz is None:
            modulation_freq_hz = 0.0

    channel_data = ensure_contiguous(channel_data)
    rx_coords_m = ensure_contiguous(rx_coords_m)
    scan_coords_m = ensure_contiguous(scan_coords_m)
    tx_wave_arrivals_s = ensure_contiguous(tx_wave_arrivals_s)

    if out is None:
        out = xp_data.zeros((n_scan, n_frames), dtype=output_dtype, like=channel_data)
    else:
        expected = xp_data.complex64 if is_complex else xp_data.float32
        if out.dtype != expected:
            raise ValueError(f"Output array dtype {out.dtype} doesn't match expected {expected}")

    if not is_writeable_array(out):
        raise ValueError("Output array `out` is not writable. Try using cupy or pytorch for the output array.")
    if not is_contiguous(out):
        raise ValueError("Output array `out` must be contiguous.")

    nb_beamform(
        channel_data,
        rx_coords_m,
        scan_coords_m,
        tx_wave_arrivals_s,
        out,
        f_number,
        rx_start_s,
        sampling_freq_hz,
        sound_speed_m_s,
        modulation_freq_hz,
        tukey_alpha,
        interp_type,
    )
    return out
