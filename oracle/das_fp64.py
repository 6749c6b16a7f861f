"""FP64 NumPy oracle for delay-and-sum (DAS) beamforming.

TEST INFRASTRUCTURE ONLY. Nothing in the ``mach_b200`` product path imports,
links or executes this file; only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` use it, and only as the checker.

This is a float64 restatement of the arithmetic of mach's single CUDA kernel
(mach-beamform 0.1.3).  Each rule below cites the reference file:line it
follows (paths inside the mach repository):

* receive aperture radius ``R = voxel.z / (2 f_number)``  -- src/mach/kernel.cu:583
* aperture test on the *horizontal* distance, ``dx^2 + dy^2 > R^2`` excludes
  the element                                              -- src/mach/kernel.cu:459-465
* delay ``tau = tx_arrival + |rx - voxel| / c`` (physical time, no t0)
                                                           -- src/mach/kernel.cu:467-471
* half-Tukey weight of ``r = sqrt(dx^2 + dy^2) / R``, only when alpha > 0
                                                           -- src/mach/kernel.cu:333-349, 473-482, 749
* skip rule ``tau < 0`` or ``weight == 0``                 -- src/mach/kernel.cu:634
* sample index ``(tau - rx_start) * fs``                   -- src/mach/kernel.cu:637
* nearest / linear / quadratic interpolation with their bounds
                                                           -- src/mach/kernel.cu:106-252
* apodization multiplies the interpolated sample, then IQ data is rotated by
  ``exp(+i 2 pi f_mod tau)`` when ``f_mod != 0``          -- src/mach/kernel.cu:649-669
* coherent compounding is the plain sum over transmits     -- src/mach/experimental.py:80-97

One deliberate deviation, shared with the CUDA kernels: for nearest-neighbour
interpolation the reference accepts ``s == n_samples - 0.5`` and, when
``n_samples`` is even, rounds it to index ``n_samples`` (one past the row,
src/mach/kernel.cu:117-126).  Here that index is treated as out of bounds.

Parity pinning: the reference has no CPU implementation and no value-level
golden vectors.  This oracle is pinned against outputs of the reference CUDA
kernel itself, compiled from its unmodified sources and run on a B200; those
outputs are committed as fixtures under ``tests/golden/`` together with the
script that produced them.
"""

from __future__ import annotations

import numpy as np

NEAREST, LINEAR, QUADRATIC = 0, 1, 2


def tukey_weight(r: np.ndarray, alpha: float) -> np.ndarray:
    """Half-Tukey window of the normalised radius (src/mach/kernel.cu:333-349)."""
    r = np.asarray(r, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        taper = 0.5 - 0.5 * np.cos(np.pi * (1.0 - r) / alpha)
    w = np.where(r <= 1.0 - alpha, 1.0, taper)
    # NaN r (0/0 at z == 0) fails every comparison and keeps the NaN taper, as on the GPU.
    w = np.where((r < 0.0) | (r > 1.0), 0.0, w)
    return w


def interpolate(row: np.ndarray, s: np.ndarray, interp_type: int) -> tuple[np.ndarray, np.ndarray]:
    """Interpolate ``row[n_samples, n_frames]`` at fractional sample ``s[n_vox]``.

    Returns ``(values[n_vox, n_frames], valid[n_vox])`` following the bounds of
    src/mach/kernel.cu:106-252.
    """
    n = row.shape[0]
    s = np.asarray(s, dtype=np.float64)
    with np.errstate(invalid="ignore"):
        if interp_type == NEAREST:
            valid = (s >= -0.5) & (s <= n - 0.5)
            idx = np.rint(np.where(valid, s, 0.0)).astype(np.int64)  # round half to even
            valid &= idx < n
            idx = np.clip(idx, 0, n - 1)
            vals = row[idx]
        elif interp_type == LINEAR:
            valid = (s >= 0.0) & (s <= n - 1)
            ss = np.where(valid, s, 0.0)
            i0 = np.floor(ss).astype(np.int64)
            i1 = np.ceil(ss).astype(np.int64)
            t = (ss - i0)[:, None]
            a = row[i0]
            b = row[i1]
            vals = a + t * (b - a)
        elif interp_type == QUADRATIC:
            valid = (s >= 1.0) & (s <= n - 2.0)
            ss = np.where(valid, s, 1.0)
            c = np.rint(ss).astype(np.int64)
            x = (ss - c)[:, None]
            wm = 0.5 * x * (x - 1.0)
            w0 = (1.0 - x) * (1.0 + x)
            wp = 0.5 * x * (x + 1.0)
            vals = wm * row[c - 1] + w0 * row[c] + wp * row[c + 1]
        else:
            raise ValueError(f"unknown interp_type {interp_type}")
    return vals, valid


def beamform_fp64(
    channel_data: np.ndarray,
    rx_coords_m: np.ndarray,
    scan_coords_m: np.ndarray,
    tx_wave_arrivals_s: np.ndarray,
    *,
    f_number: float,
    rx_start_s: float,
    sampling_freq_hz: float,
    sound_speed_m_s: float,
    modulation_freq_hz: float = 0.0,
    tukey_alpha: float = 0.5,
    interp_type: int = LINEAR,
    channel_scale: float = 1.0,
) -> np.ndarray:
    """Delay-and-sum in float64, compounding over transmits.

    ``channel_data`` is ``[n_rx, n_samples, n_frames]`` (one transmit) or
    ``[n_tx, n_rx, n_samples, n_frames]``; ``tx_wave_arrivals_s`` is
    ``[n_scan]`` or ``[n_tx, n_scan]``.  Integer storage is multiplied by
    ``channel_scale``.  Returns ``[n_scan, n_frames]`` (complex128 for complex
    input, float64 otherwise) -- the sum that mach accumulates into ``out``.
    """
    ch = np.asarray(channel_data)
    arr = np.asarray(tx_wave_arrivals_s, dtype=np.float64)
    if ch.ndim == 3:
        ch = ch[None]
        arr = arr[None]
    is_complex = np.iscomplexobj(ch)
    ch = ch.astype(np.complex128 if is_complex else np.float64) * channel_scale
    rx = np.asarray(rx_coords_m, dtype=np.float64)
    scan = np.asarray(scan_coords_m, dtype=np.float64)
    n_tx, n_rx, _, n_f = ch.shape
    n_vox = scan.shape[0]
    out = np.zeros((n_vox, n_f), dtype=ch.dtype)

    radius = scan[:, 2] / (2.0 * f_number)  # kernel.cu:583
    radius_sq = radius * radius
    rotate = is_complex and modulation_freq_hz != 0.0
    for e in range(n_rx):
        dx = rx[e, 0] - scan[:, 0]
        dy = rx[e, 1] - scan[:, 1]
        dz = rx[e, 2] - scan[:, 2]
        h2 = dx * dx + dy * dy
        in_aperture = ~(h2 > radius_sq)  # kernel.cu:461-464
        dist = np.sqrt(h2 + dz * dz)
        if tukey_alpha > 0.0:
            with np.errstate(invalid="ignore", divide="ignore"):
                weight = tukey_weight(np.sqrt(h2) / radius, tukey_alpha)
        else:
            weight = np.ones(n_vox)
        for t in range(n_tx):
            tau = arr[t] + dist / sound_speed_m_s
            use = in_aperture & ~(tau < 0.0) & ~(weight == 0.0)  # kernel.cu:634
            s = (tau - rx_start_s) * sampling_freq_hz  # kernel.cu:637
            vals, valid = interpolate(ch[t, e], s, interp_type)
            use &= valid
            if not use.any():
                continue
            contrib = vals[use] * weight[use, None]
            if rotate:
                contrib = contrib * np.exp(1j * 2.0 * np.pi * modulation_freq_hz * tau[use])[:, None]
            out[use] += contrib
    return out


def nrms_db(y: np.ndarray, y_ref: np.ndarray) -> float:
    """Normalised RMS error in dB: ``20 log10(||y - y_ref|| / ||y_ref||)``."""
    y = np.asarray(y, dtype=np.complex128).ravel()
    y_ref = np.asarray(y_ref, dtype=np.complex128).ravel()
    num = np.linalg.norm(y - y_ref)
    den = np.linalg.norm(y_ref)
    if den == 0.0:
        return -np.inf if num == 0.0 else np.inf
    if num == 0.0:
        return -np.inf
    return float(20.0 * np.log10(num / den))


def rel_l2(y: np.ndarray, y_ref: np.ndarray) -> float:
    """Relative L2 error ``||y - y_ref|| / ||y_ref||``."""
    y = np.asarray(y, dtype=np.complex128).ravel()
    y_ref = np.asarray(y_ref, dtype=np.complex128).ravel()
    den = np.linalg.norm(y_ref)
    num = np.linalg.norm(y - y_ref)
    return float(num / den) if den > 0 else float(num)
