"""Native binding: the Python face of ``libmach_b200.so``.

Mirrors mach's nanobind module ``mach._cuda_impl`` (src/mach/kernel.cu:1211-1256,
stub src/mach/_cuda_impl.pyi): the same ``beamform`` overloads selected by dtype
without conversion, the same ``InterpolationType`` enum with its exported values,
``__nvcc_version__``, and the same exceptions and warning for bad shapes, unsupported
devices and CPU-resident inputs.  The arrays are passed by pointer (zero copy) to the
C ABI declared in ``include/mach_b200.h``.  There is no fallback: if the CUDA library
is missing, importing this module raises.
"""

from __future__ import annotations

import ctypes
import enum
import os
import warnings
from pathlib import Path
from typing import Any

from mach_b200 import _dlpack

_LIB_PATH = Path(os.environ.get("MACH_B200_LIBRARY", Path(__file__).resolve().parent / "libmach_b200.so"))
if not _LIB_PATH.exists():
    raise ImportError(
        f"mach_b200 CUDA library not found at {_LIB_PATH}; build it with `python -m mach_b200.csrc.build`"
    )
_lib = ctypes.CDLL(str(_LIB_PATH))

_F = ctypes.c_float
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32

_single_args = [_P, _P, _P, _P, _P, _U32, _U32, _U64, _U32, _F, _F, _F, _F, _F, _F, _I32]
for _name in ("mach_b200_beamform_f32", "mach_b200_beamform_c64"):
    getattr(_lib, _name).argtypes = _single_args
    getattr(_lib, _name).restype = ctypes.c_int
_lib.mach_b200_beamform_compound.argtypes = [
    _I32, _P, _P, _P, _P, _P, _U32, _U32, _U32, _U64, _U32, _F, _F, _F, _F, _F, _F, _I32, _F, _P, _U32,
]
_lib.mach_b200_beamform_compound.restype = ctypes.c_int


class Options(ctypes.Structure):
    """``mach_b200_options`` (include/mach_b200.h): launch hints that never change the result."""

    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("grid_shape", ctypes.c_int32 * 3),
        ("kernel", ctypes.c_int32),
        ("tx_chunk", ctypes.c_int32),
        ("window_rows", ctypes.c_int32),
        ("lanes_per_voxel", ctypes.c_int32),
        ("tx_model", ctypes.c_int32),
        ("tile_fast", ctypes.c_int32),
        ("tx_params", ctypes.c_void_p),
        ("frame_slots", ctypes.c_int32),
        ("element_block", ctypes.c_int32),
        ("tile_order", ctypes.c_int32),
    ]


KERNELS = {"auto": 0, "lane_voxel": 1, "staged": 2, "warp": 3, "ensemble": 4, "frame_lane": 5}


def make_options(flags: int = 0, grid_shape=None, kernel: str | int = 0, tx_chunk: int = 0, window_rows: int = 0,
                 lanes_per_voxel: int = 0, tile_fast: int = 0, frame_slots: int = 0,
                 element_block: int = 0, tile_order: int = 0) -> Options:
    o = Options()
    o.struct_size = ctypes.sizeof(Options)
    o.flags = int(flags)
    if grid_shape is not None:
        for i, v in enumerate(grid_shape):
            o.grid_shape[i] = int(v)
    o.kernel = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
    o.tx_chunk = int(tx_chunk)
    o.window_rows = int(window_rows)
    o.lanes_per_voxel = int(lanes_per_voxel)
    o.tile_fast = int(tile_fast)
    o.frame_slots = int(frame_slots)
    o.element_block = int(element_block)
    o.tile_order = int(tile_order)
    return o


_lib.mach_b200_beamform_ex.argtypes = [
    _I32, _P, _P, _P, _P, _P, _U32, _U32, _U32, _U64, _U32, _F, _F, _F, _F, _F, _F, _I32, _F, _P,
    ctypes.POINTER(Options),
]
_lib.mach_b200_beamform_ex.restype = ctypes.c_int
_lib.mach_b200_ingest.argtypes = [_I32, _P, _I32, _P, _U32, _U32, _U32, _U32, _F, _P, _U32]
_lib.mach_b200_ingest.restype = ctypes.c_int
_lib.mach_b200_hilbert.argtypes = [_I32, _P, _I32, _I32, _P, _U32, _U32, _U32, _U32, _F, _P, _U32]
_lib.mach_b200_hilbert.restype = ctypes.c_int
LAYOUT_CHANNEL = 0
LAYOUT_ACQUISITION = 1
_lib.mach_b200_probe_l2_read.argtypes = [_P, _U64, _U32, _P]
_lib.mach_b200_probe_l2_read.restype = ctypes.c_int
_lib.mach_b200_last_error.restype = ctypes.c_char_p
_lib.mach_b200_nvcc_version.restype = ctypes.c_char_p
_lib.mach_b200_version.restype = ctypes.c_char_p
_lib.mach_b200_launch_count.restype = ctypes.c_uint64

__nvcc_version__: str = _lib.mach_b200_nvcc_version().decode()
library_path: str = str(_LIB_PATH)

FLAG_ASYNC = 1
FLAG_OVERWRITE = 2
FLAG_SPLIT_DELAY = 4
FLAG_POWER_DOPPLER = 8

STORAGE_CODES = {"f32": 0, "c64": 1, "f16": 2, "cf16": 3, "bf16": 4, "cbf16": 5, "i16": 6, "ci16": 7}


class InterpolationType(enum.IntEnum):
    """Interpolation of channel samples (src/mach/kernel.cu:25-29, 1221-1225)."""

    NearestNeighbor = 0
    """Use nearest neighbor interpolation (fastest)"""
    Linear = 1
    """Use linear interpolation (default, good balance)"""
    Quadratic = 2
    """Use quadratic interpolation (higher quality)"""


NearestNeighbor = InterpolationType.NearestNeighbor
Linear = InterpolationType.Linear
Quadratic = InterpolationType.Quadratic


def probe_l2_read(ptr: int, nbytes: int, passes: int, stream: int = 0) -> None:
    """Launch the L2 read-bandwidth probe over a device buffer (``mach_b200_probe_l2_read``)."""
    rc = _lib.mach_b200_probe_l2_read(ptr, nbytes, passes, stream)
    if rc != 0:
        raise RuntimeError(f"mach_b200_probe_l2_read failed with code {rc}")


def launch_count() -> int:
    """Kernels launched by the native library since it was loaded."""
    return int(_lib.mach_b200_launch_count())


def _raise_for(rc: int) -> None:
    if rc == 0:
        return
    msg = _lib.mach_b200_last_error().decode(errors="replace")
    raise RuntimeError(msg)


def _shape_str(v: _dlpack.ArrayView) -> str:
    return "[" + ", ".join(str(d) for d in v.shape) + "]"


def _check_dimensions(ch, rx, scan, tx, out, n_rx, n_samples, n_vox, n_frames) -> None:
    """Same checks and messages as mach's check_dimensions (src/mach/kernel.cu:913-951)."""
    if n_rx != ch.shape[0] or n_rx != rx.shape[0]:
        raise RuntimeError(
            "Dimension mismatch in receive elements:\n"
            f"  Expected n_receive_elements: {n_rx}\n"
            f"  channel_data.shape: {_shape_str(ch)}\n"
            f"  rx_coords_m.shape: {_shape_str(rx)}\n"
            "→ channel_data.shape[0] and rx_coords_m.shape[0] must both equal n_receive_elements"
        )
    if n_vox != tx.shape[0] or n_vox != scan.shape[0] or n_vox != out.shape[0]:
        raise RuntimeError(
            "Dimension mismatch in output voxels:\n"
            f"  Expected n_output_voxels: {n_vox}\n"
            f"  scan_coords_m.shape: {_shape_str(scan)}\n"
            f"  tx_wave_arrivals_s.shape: {_shape_str(tx)}\n"
            f"  out.shape: {_shape_str(out)}\n"
            "→ scan_coords_m.shape[0], tx_wave_arrivals_s.shape[0], and out.shape[0] must all equal n_output_voxels"
        )
    if n_frames != ch.shape[2] or n_frames != out.shape[1]:
        raise RuntimeError(
            "Dimension mismatch in frames:\n"
            f"  Expected n_frames: {n_frames}\n"
            f"  channel_data.shape: {_shape_str(ch)}\n"
            f"  out.shape: {_shape_str(out)}\n"
            "→ channel_data.shape[2] and out.shape[1] must both equal n_frames"
        )


def _check_devices(views: list[_dlpack.ArrayView]) -> int:
    """Count CPU arrays; reject devices other than CPU/CUDA (src/mach/kernel.cu:964-987)."""
    cpu = 0
    for v in views:
        if v.device_type == _dlpack.CPU:
            cpu += 1
        elif v.device_type in (_dlpack.CUDA, _dlpack.CUDA_HOST, _dlpack.CUDA_MANAGED):
            pass
        else:
            raise RuntimeError(
                f"Found input array on device: {v.device_type}. Only CPU and CUDA devices are supported."
            )
    return cpu


def _cpu_warning(cpu_count: int) -> None:
    # Same text as src/mach/kernel.cu:1092-1094.
    warnings.warn(
        f"Found {cpu_count} input array(s) on CPU. This will add latency due to CPU<->GPU memory transfers. "
        "For optimal performance with CUDA beamforming, move arrays to GPU using cupy, jax, or similar.",
        UserWarning,
        stacklevel=3,
    )


_SIG = (
    "beamform(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, f_number, rx_start_s, "
    "sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha=0.5, interp_type=Linear)"
)


def _incompatible(reason: str) -> TypeError:
    return TypeError(f"beamform(): incompatible function arguments ({reason}). The following signature is supported:\n    {_SIG}")


def beamform(
    channel_data: Any,
    rx_coords_m: Any,
    scan_coords_m: Any,
    tx_wave_arrivals_s: Any,
    out: Any,
    f_number: float,
    rx_start_s: float,
    sampling_freq_hz: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float | None = None,
    tukey_alpha: float = 0.5,
    interp_type: InterpolationType = InterpolationType.Linear,
) -> None:
    """Single-transmit DAS, accumulating into ``out`` (drop-in for ``mach._cuda_impl.beamform``).

    Overloads (no dtype conversion, C-contiguous arrays only):
    complex64 ``channel_data``/``out`` with a required ``modulation_freq_hz``, or float32
    with ``modulation_freq_hz=0.0`` by default.  A CUDA ``out`` is accumulated into; a CPU
    ``out`` is overwritten.  Synchronous, on the current device.
    """
    try:
        views = [_dlpack.view(a) for a in (channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out)]
    except TypeError as err:
        raise _incompatible(str(err)) from None
    ch, rx, scan, tx, o = views
    if ch.dtype == "complex64" and o.dtype == "complex64":
        fn = _lib.mach_b200_beamform_c64
        if modulation_freq_hz is None:
            raise _incompatible("modulation_freq_hz is required for complex64 channel_data")
    elif ch.dtype == "float32" and o.dtype == "float32":
        fn = _lib.mach_b200_beamform_f32
        if modulation_freq_hz is None:
            modulation_freq_hz = 0.0
    else:
        raise _incompatible(f"channel_data dtype {ch.dtype} / out dtype {o.dtype}")
    for name, v, nd in (("channel_data", ch, 3), ("rx_coords_m", rx, 2), ("scan_coords_m", scan, 2),
                        ("tx_wave_arrivals_s", tx, 1), ("out", o, 2)):
        if name != "channel_data" and name != "out" and v.dtype != "float32":
            raise _incompatible(f"{name} must be float32, got {v.dtype}")
        if len(v.shape) != nd:
            raise _incompatible(f"{name} must have {nd} dimensions, got {len(v.shape)}")
        if not v.c_contiguous:
            raise _incompatible(f"{name} must be C-contiguous")
    if rx.shape[1] != 3 or scan.shape[1] != 3:
        raise _incompatible("coordinate arrays must have shape (n, 3)")
    if not o.writeable:
        raise _incompatible("out must be writable")
    n_rx, n_samples, n_vox, n_frames = rx.shape[0], ch.shape[1], scan.shape[0], o.shape[1]
    _check_dimensions(ch, rx, scan, tx, o, n_rx, n_samples, n_vox, n_frames)
    cpu = _check_devices(views)
    if cpu:
        _cpu_warning(cpu)
    rc = fn(ch.ptr, rx.ptr, scan.ptr, tx.ptr, o.ptr, n_rx, n_samples, n_vox, n_frames, float(f_number),
            float(rx_start_s), float(sampling_freq_hz), float(sound_speed_m_s), float(modulation_freq_hz),
            float(tukey_alpha), int(interp_type))
    _raise_for(rc)


def storage_of(v: _dlpack.ArrayView, complex_pairs: bool) -> str:
    """Storage code name for a channel-data view (trailing (I, Q) axis when ``complex_pairs``)."""
    table = {
        ("float32", False): "f32", ("complex64", False): "c64", ("float16", False): "f16",
        ("float16", True): "cf16", ("complex32", False): "cf16", ("bfloat16", False): "bf16",
        ("bfloat16", True): "cbf16", ("int16", False): "i16", ("int16", True): "ci16",
    }
    key = (v.dtype, complex_pairs)
    if key not in table:
        raise TypeError(f"unsupported channel_data dtype {v.dtype}" + (" with (I, Q) pairs" if complex_pairs else ""))
    return table[key]


def beamform_compound(
    channel: _dlpack.ArrayView,
    storage: str,
    rx: _dlpack.ArrayView,
    scan: _dlpack.ArrayView,
    arrivals: _dlpack.ArrayView,
    out: _dlpack.ArrayView,
    *,
    n_tx: int,
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
    channel_scale: float = 1.0,
    stream: int = 0,
    flags: int = 0,
    options: Options | None = None,
) -> None:
    """Multi-transmit DAS in one launch through ``mach_b200_beamform_ex``."""
    if options is None:
        options = make_options(flags)
    else:
        options.flags = int(options.flags) | int(flags)
    rc = _lib.mach_b200_beamform_ex(
        STORAGE_CODES[storage], channel.ptr, rx.ptr, scan.ptr, arrivals.ptr, out.ptr, n_tx, n_rx, n_samples,
        n_vox, n_frames, float(f_number), float(rx_start_s), float(sampling_freq_hz), float(sound_speed_m_s),
        float(modulation_freq_hz), float(tukey_alpha), int(interp_type), float(channel_scale), stream or None,
        ctypes.byref(options),
    )
    _raise_for(rc)
