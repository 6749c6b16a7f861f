"""Coherent compounding over transmits (mirror of mach's src/mach/experimental.py:23-108).

mach loops over transmits in Python and launches (and synchronises) its kernel once
per transmit, always with linear interpolation.  Here all transmits go to the GPU in
one launch of ``mach_b200_beamform_compound``: each (voxel, element) receive path is
computed once and reused for every transmit, the sum stays in registers and ``out``
is written once.  ``interp_type`` is honoured, and channel data may be stored as
float32 / complex64 or, for reduced-precision storage, float16, bfloat16 or int16
(real, or complex as a trailing (I, Q) axis; torch ``complex32`` is also accepted).
All arithmetic is FP32.
"""

from __future__ import annotations

import warnings
from typing import Any

from mach_b200 import _cuda_impl, _dlpack, _grid
from mach_b200._array_api import array_namespace, is_writeable_array
from mach_b200._check import ensure_contiguous, is_contiguous
from mach_b200._cuda_impl import InterpolationType


def _current_stream(x: Any) -> int:
    if _dlpack.is_torch(x) and x.device.type == "cuda":
        import torch

        return int(torch.cuda.current_stream(x.device).cuda_stream)
    return 0


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
    channel_scale: float = 1.0,
    sync: bool = True,
    grid_shape: Any = None,
    kernel: str = "auto",
    window_rows: int = 0,
    lanes_per_voxel: int = 0,
    tx_chunk: int = 0,
    delay: str = "auto",
    tile_fast: int = 0,
    frame_slots: int = 0,
    element_block: int = 0,
    tile_order: int = 0,
) -> Any:
    """Beamform and coherently compound ``n_transmits`` transmits.

    Args:
        channel_data: ``[n_transmits, n_rx, n_samples, n_frames]`` (float32, float64,
            complex64, complex128, float16, bfloat16, int16, torch complex32) or
            ``[n_transmits, n_rx, n_samples, n_frames, 2]`` (I, Q) pairs of float16 /
            bfloat16 / int16.
        tx_wave_arrivals_s: ``[n_transmits, n_points]`` seconds.
        channel_scale: multiplier applied to every sample (for int16 storage).
        sync: when False and every array is on the GPU, return without waiting for the
            kernel (it runs on the current torch stream for torch inputs).
        grid_shape: ``(slow, mid, fast)`` extents when ``scan_coords_m`` is a flattened grid
            (fast = contiguous axis); ``None`` detects it, ``False`` disables tiling by grid.
            Only the voxel-to-CTA assignment depends on it, never the result.
        kernel, window_rows, lanes_per_voxel, tx_chunk, tile_fast, frame_slots, element_block,
            tile_order: launch tuning (see ``mach_b200_options`` in include/mach_b200.h); the
            autotuner sets them.
        delay: ``"reference"`` computes delays in FP32 exactly as mach does (bit-identical
            sample positions); ``"split"`` forms each sample position and phase in FP64 per
            receive path and per transmit as an integer base + FP32 fraction (more accurate,
            not bit-identical to mach); ``"auto"`` uses ``"reference"`` for float32/complex64
            storage and ``"split"`` for reduced-precision storage.
        Other arguments as in :func:`mach_b200.kernel.beamform`.

    Returns:
        ``out[n_points, n_frames]``: complex64 for complex storage, float32 otherwise.
        A GPU ``out`` is accumulated into; a CPU ``out`` is overwritten (as in mach).
    """
    return _compound(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, rx_start_s=rx_start_s,
                     sampling_freq_hz=sampling_freq_hz, f_number=f_number, sound_speed_m_s=sound_speed_m_s,
                     modulation_freq_hz=modulation_freq_hz, tukey_alpha=tukey_alpha, interp_type=interp_type,
                     channel_scale=channel_scale, sync=sync, grid_shape=grid_shape, kernel=kernel,
                     window_rows=window_rows, lanes_per_voxel=lanes_per_voxel, tx_chunk=tx_chunk, delay=delay,
                     power=False, tile_fast=tile_fast, frame_slots=frame_slots,
                     element_block=element_block, tile_order=tile_order)


def _tuned(storage, n_tx, n_rx, n_samples, n_frames, n_points, grid, interp_type, delay, channel_data):
    """Cached autotuner knobs for this job on the channel data's (or the current) CUDA device."""
    from mach_b200 import tuning

    index = 0
    if _dlpack.is_torch(channel_data) and channel_data.device.type == "cuda":
        index = channel_data.device.index or 0
    else:
        import torch

        index = torch.cuda.current_device()
    return tuning.lookup(storage, n_tx, n_rx, n_samples, n_frames, n_points, grid, int(interp_type), index, delay)


def _compound(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, *, rx_start_s, sampling_freq_hz,
              f_number, sound_speed_m_s, modulation_freq_hz, tukey_alpha, interp_type, channel_scale, sync, grid_shape,
              kernel, window_rows, lanes_per_voxel, tx_chunk, delay, power, tile_fast=0, frame_slots=0, element_block=0,
              tile_order=0):
    """Shared body of :func:`beamform` and :func:`mach_b200.doppler.power_doppler` (``power``:
    ``out`` is the float32 ``[n_points]`` power image instead of the frames)."""
    xp = array_namespace(channel_data)
    complex_pairs = len(channel_data.shape) == 5
    if complex_pairs and channel_data.shape[-1] != 2:
        raise ValueError("a 5-D channel_data must end in an (I, Q) axis of length 2")
    if not complex_pairs and len(channel_data.shape) != 4:
        raise ValueError("channel_data must be [n_transmits, n_rx, n_samples, n_frames]")
    dtype_name = str(channel_data.dtype).replace("torch.", "")
    if dtype_name == "complex128":
        channel_data = xp.astype(channel_data, xp.complex64, copy=False)
    elif dtype_name == "float64":
        channel_data = xp.astype(channel_data, xp.float32, copy=False)
    channel_data = ensure_contiguous(channel_data)
    ch = _dlpack.view(channel_data)
    storage = _cuda_impl.storage_of(ch, complex_pairs)
    is_complex = bool(_cuda_impl.STORAGE_CODES[storage] & 1)
    if is_complex and modulation_freq_hz is None:
        raise ValueError(
            "modulation_freq_hz is required for complex phase-correction. set it to 0 if no demodulation was used."
        )
    if modulation_freq_hz is None:
        modulation_freq_hz = 0.0

    from mach_b200.wavefront import TransmitWaves

    xpc = array_namespace(rx_coords_m)
    xps = array_namespace(scan_coords_m)
    rx_coords_m = ensure_contiguous(xpc.astype(rx_coords_m, xpc.float32, copy=False))
    scan_coords_m = ensure_contiguous(xps.astype(scan_coords_m, xps.float32, copy=False))
    waves = tx_wave_arrivals_s if isinstance(tx_wave_arrivals_s, TransmitWaves) else None
    if waves is None:
        xpa = array_namespace(tx_wave_arrivals_s)
        tx_wave_arrivals_s = ensure_contiguous(xpa.astype(tx_wave_arrivals_s, xpa.float32, copy=False))
    else:
        if waves.n_transmits != int(channel_data.shape[0]):
            raise RuntimeError(f"{waves.n_transmits} transmit waves for {int(channel_data.shape[0])} transmits")
        # FP64 wave table next to the channel data (device tensor for torch CUDA input)
        if _dlpack.is_torch(channel_data) and channel_data.device.type == "cuda":
            import torch

            tx_wave_arrivals_s = torch.as_tensor(waves.table, device=channel_data.device)
        else:
            import numpy as np

            tx_wave_arrivals_s = np.ascontiguousarray(waves.table)

    n_tx, n_rx, n_samples, n_frames = (int(d) for d in channel_data.shape[:4])
    n_points = int(scan_coords_m.shape[0])
    output_dtype = xp.complex64 if is_complex and not power else xp.float32
    out_shape = (n_points,) if power else (n_points, n_frames)
    if out is None:
        out = xp.zeros(out_shape, dtype=output_dtype, like=channel_data)
    elif out.dtype != output_dtype:
        raise ValueError(f"Output array dtype {out.dtype} doesn't match expected {output_dtype}")
    if not is_writeable_array(out):
        raise ValueError("Output array `out` is not writable. Try using cupy or pytorch for the output array.")
    if not is_contiguous(out):
        raise ValueError("Output array `out` must be contiguous.")

    rx = _dlpack.view(rx_coords_m)
    scan = _dlpack.view(scan_coords_m)
    arr = _dlpack.view(tx_wave_arrivals_s)  # the wave table when `waves` is given
    o = _dlpack.view(out)
    if tuple(rx.shape) != (n_rx, 3):
        raise RuntimeError(f"rx_coords_m.shape {list(rx.shape)} must be [{n_rx}, 3]")
    if tuple(scan.shape) != (n_points, 3):
        raise RuntimeError(f"scan_coords_m.shape {list(scan.shape)} must be [n_points, 3]")
    if waves is None and tuple(arr.shape) != (n_tx, n_points):
        raise RuntimeError(f"tx_wave_arrivals_s.shape {list(arr.shape)} must be [{n_tx}, {n_points}]")
    if tuple(o.shape) != out_shape:
        raise RuntimeError(f"out.shape {list(o.shape)} must be {list(out_shape)}")
    cpu = sum(v.device_type == _dlpack.CPU for v in (ch, rx, scan, arr))
    if cpu:
        warnings.warn(
            f"Found {cpu} input array(s) on CPU. This will add latency due to CPU<->GPU memory transfers. "
            "For optimal performance with CUDA beamforming, move arrays to GPU using cupy, jax, or similar.",
            UserWarning,
            stacklevel=2,
        )
    all_gpu = all(v.on_cuda for v in (ch, rx, scan, arr, o))
    flags = 0 if (sync or not all_gpu) else _cuda_impl.FLAG_ASYNC
    if delay == "auto":
        delay = "reference" if storage in ("f32", "c64") else "split"
    if delay not in ("reference", "split"):
        raise ValueError(f"delay must be 'auto', 'reference' or 'split', got {delay!r}")
    if delay == "split":
        flags |= _cuda_impl.FLAG_SPLIT_DELAY
    if power:
        flags |= _cuda_impl.FLAG_POWER_DOPPLER
    if grid_shape is None:
        grid_shape = _grid.detect(scan_coords_m)
        if (kernel == "auto" and not (window_rows or lanes_per_voxel or tx_chunk or tile_fast or frame_slots
                                      or element_block) and not power):
            # launch knobs the autotuner chose for this job shape, if it has timed one
            tuned = _tuned(storage, n_tx, n_rx, n_samples, n_frames, n_points, grid_shape, interp_type, delay,
                           channel_data)
            if tuned:
                grid_shape = tuned.pop("grid_shape", grid_shape)
                kernel = tuned.get("kernel", kernel)
                window_rows = tuned.get("window_rows", 0)
                lanes_per_voxel = tuned.get("lanes_per_voxel", 0)
                tx_chunk = tuned.get("tx_chunk", 0)
                tile_fast = tuned.get("tile_fast", 0)
                frame_slots = tuned.get("frame_slots", 0)
                element_block = tuned.get("element_block", 0)
    options = _cuda_impl.make_options(
        flags, grid_shape=grid_shape or None, kernel=kernel, tx_chunk=tx_chunk, window_rows=window_rows,
        lanes_per_voxel=lanes_per_voxel, tile_fast=tile_fast, frame_slots=frame_slots, element_block=element_block,
        tile_order=tile_order)
    if waves is not None:
        options.tx_model = waves.model
        options.tx_params = arr.ptr
        arr = _dlpack.NullView()
    _cuda_impl.beamform_compound(
        ch, storage, rx, scan, arr, o, n_tx=n_tx, n_rx=n_rx, n_samples=n_samples, n_vox=n_points,
        n_frames=n_frames, f_number=f_number, rx_start_s=rx_start_s, sampling_freq_hz=sampling_freq_hz,
        sound_speed_m_s=sound_speed_m_s, modulation_freq_hz=modulation_freq_hz, tukey_alpha=tukey_alpha,
        interp_type=int(interp_type), channel_scale=channel_scale, stream=_current_stream(channel_data),
        flags=flags, options=options,
    )
    return out
