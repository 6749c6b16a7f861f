"""ctypes front end for mach's own CUDA kernel built from its unmodified source.

TEST/BASELINE INFRASTRUCTURE ONLY.  ``oracle/_ref/libmachref.so`` is produced by
``oracle/build.py`` from the reference's ``src/mach/kernel.cu``.  This module
drives it exactly the way mach's Python layer does:

* :func:`beamform_device` -- the call ``mach.kernel.nb_beamform`` makes when every
  array is already on the GPU (``_beamform_impl``, src/mach/kernel.cu:1068-1088),
  one call per transmit into the same ``out`` as ``mach.experimental.beamform``
  does (src/mach/experimental.py:80-97).  Each call ends in
  ``cudaDeviceSynchronize`` inside the reference.
* :func:`beamform_host` -- the reference binding with host arrays
  (src/mach/kernel.cu:1090-1208): per call it allocates device buffers, copies the
  host inputs, launches, and copies ``out`` back.
"""

from __future__ import annotations

import ctypes

import numpy as np

from oracle import build as _build

_lib = None
CPU, CUDA = 1, 2


def available() -> bool:
    return _build.REF_LIB.exists()


def _load():
    global _lib
    if _lib is None:
        if not _build.REF_LIB.exists():
            raise FileNotFoundError(f"reference kernel not built: {_build.REF_LIB}")
        lib = ctypes.CDLL(str(_build.REF_LIB))
        common = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32] + [ctypes.c_float] * 6 + [
            ctypes.c_int,
            ctypes.c_char_p,
            ctypes.c_size_t,
        ]
        lib.machref_beamform_impl.restype = ctypes.c_int
        lib.machref_beamform_impl.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5 + common
        lib.machref_beamform_binding.restype = ctypes.c_int
        lib.machref_beamform_binding.argtypes = [
            ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int,
        ] + common
        lib.machref_last_warning.restype = ctypes.c_char_p
        lib.machref_nvcc_version.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def _check(rc: int, err: ctypes.Array) -> None:
    if rc != 0:
        raise RuntimeError(err.value.decode(errors="replace"))


def beamform_device(
    channel_ptrs: list[int],
    rx_ptr: int,
    scan_ptr: int,
    arrival_ptrs: list[int],
    out_ptr: int,
    *,
    is_complex: bool,
    n_rx: int,
    n_samples: int,
    n_vox: int,
    n_frames: int,
    f_number: float,
    rx_start_s: float,
    sampling_freq_hz: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float,
    tukey_alpha: float,
    interp_type: int,
) -> None:
    """One reference launch per transmit, accumulating into the device buffer ``out_ptr``."""
    lib = _load()
    err = ctypes.create_string_buffer(4096)
    for ch, arr in zip(channel_ptrs, arrival_ptrs, strict=True):
        rc = lib.machref_beamform_impl(
            int(is_complex), ch, rx_ptr, scan_ptr, arr, out_ptr, n_rx, n_samples, n_vox, n_frames,
            f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s, modulation_freq_hz,
            tukey_alpha, interp_type, err, len(err),
        )
        _check(rc, err)


def beamform_host(
    channel: np.ndarray,
    rx: np.ndarray,
    scan: np.ndarray,
    arrivals: np.ndarray,
    out: np.ndarray,
    *,
    f_number: float,
    rx_start_s: float,
    sampling_freq_hz: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float,
    tukey_alpha: float,
    interp_type: int,
    out_on_device_ptr: int | None = None,
) -> None:
    """Reference binding with host inputs for every transmit of ``channel[n_tx, n_rx, n_s, n_f]``.

    With ``out_on_device_ptr`` the transmits accumulate into that device buffer (what
    ``mach.experimental.beamform`` does with its GPU temporary); otherwise each call
    overwrites the host ``out`` (the binding zero-fills its staging copy).
    """
    lib = _load()
    err = ctypes.create_string_buffer(4096)
    is_complex = np.iscomplexobj(channel)
    n_tx, n_rx, n_s, n_f = channel.shape
    n_vox = scan.shape[0]
    for t in range(n_tx):
        ch = channel[t]
        arr = arrivals[t]
        if out_on_device_ptr is not None:
            o_ptr, o_dev = out_on_device_ptr, CUDA
        else:
            o_ptr, o_dev = out.ctypes.data, CPU
        rc = lib.machref_beamform_binding(
            int(is_complex), ch.ctypes.data, CPU, rx.ctypes.data, CPU, scan.ctypes.data, CPU,
            arr.ctypes.data, CPU, o_ptr, o_dev, n_rx, n_s, n_vox, n_f, f_number, rx_start_s,
            sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha, interp_type,
            err, len(err),
        )
        _check(rc, err)


def last_warning() -> str:
    return _load().machref_last_warning().decode()
