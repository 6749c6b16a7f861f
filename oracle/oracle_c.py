"""ctypes front end for the FP64 C oracle (oracle/das_oracle.c).

TEST INFRASTRUCTURE ONLY -- used by tests/, the smoke check and bench.py's
cpu_baseline leg as the checker.  It follows the same reference rules as
oracle/das_fp64.py (see the citations there) and is cross-checked against it.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import build as _build

# storage codes, same numbering as include/mach_b200.h
STORAGE_CODES = {
    "f32": 0,
    "c64": 1,
    "f16": 2,
    "cf16": 3,
    "bf16": 4,
    "cbf16": 5,
    "i16": 6,
    "ci16": 7,
}

_lib = None


def _load():
    global _lib
    if _lib is None:
        path = _build.ORACLE_LIB
        if not path.exists():
            path = _build.build_oracle()
        lib = ctypes.CDLL(str(path))
        f = lib.das_oracle_f64
        f.restype = ctypes.c_int
        f.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_int, ctypes.c_int,
        ]
        lib.das_oracle_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def max_threads() -> int:
    return int(_load().das_oracle_max_threads())


def beamform_c(
    channel_data: np.ndarray,
    rx_coords_m: np.ndarray,
    scan_coords_m: np.ndarray,
    tx_wave_arrivals_s: np.ndarray,
    *,
    storage: str,
    f_number: float,
    rx_start_s: float,
    sampling_freq_hz: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float = 0.0,
    tukey_alpha: float = 0.5,
    interp_type: int = 1,
    channel_scale: float = 1.0,
    voxel_subset: np.ndarray | None = None,
    n_threads: int = 0,
) -> np.ndarray:
    """FP64 DAS over all transmits.

    ``channel_data`` is the raw storage array ``[n_tx, n_rx, n_samples, n_frames(, 2)]``
    as the GPU sees it (complex storage either as numpy complex or with a trailing
    axis of 2 for half/bfloat16/int16 pairs).  Returns ``[n_sel, n_frames]``
    complex128 or float64.
    """
    code = STORAGE_CODES[storage]
    cplx = bool(code & 1)
    ch = np.ascontiguousarray(channel_data)
    arr = np.ascontiguousarray(tx_wave_arrivals_s, dtype=np.float32)
    if arr.ndim == 1:
        arr = arr[None]
    n_tx = arr.shape[0]
    rx = np.ascontiguousarray(rx_coords_m, dtype=np.float32)
    scan = np.ascontiguousarray(scan_coords_m, dtype=np.float32)
    n_rx = rx.shape[0]
    n_vox = scan.shape[0]
    pair_axis = cplx and ch.dtype != np.complex64
    if ch.dtype == np.complex128:
        raise TypeError("complex storage must be complex64 or a trailing (I, Q) axis")
    if ch.ndim == (4 if pair_axis else 3):  # single transmit
        ch = ch.reshape((1,) + ch.shape)
    n_s, n_f = int(ch.shape[2]), int(ch.shape[3])
    if int(ch.shape[0]) != n_tx or int(ch.shape[1]) != n_rx:
        raise ValueError(f"channel_data shape {ch.shape} does not match n_tx={n_tx}, n_rx={n_rx}")
    if voxel_subset is None:
        sel = None
        n_sel = n_vox
    else:
        sel = np.ascontiguousarray(voxel_subset, dtype=np.int64)
        n_sel = sel.shape[0]
    out = np.zeros((n_sel, n_f, 2) if cplx else (n_sel, n_f), dtype=np.float64)
    rc = _load().das_oracle_f64(
        code, ch.ctypes.data, float(channel_scale), rx.ctypes.data, scan.ctypes.data,
        arr.ctypes.data, out.ctypes.data, n_tx, n_rx, n_s, n_f, n_vox,
        None if sel is None else sel.ctypes.data, n_sel, float(f_number), float(rx_start_s),
        float(sampling_freq_hz), float(sound_speed_m_s), float(modulation_freq_hz),
        float(tukey_alpha), int(interp_type), int(n_threads or os.cpu_count() or 1),
    )
    if rc != 0:
        raise ValueError("das_oracle_f64 rejected its arguments")
    if cplx:
        return out[..., 0] + 1j * out[..., 1]
    return out
