"""Python API contract checks that fail before any GPU work (mirrors mach's tests/test_nanobind.py)."""

from __future__ import annotations

import numpy as np
import pytest

import mach_b200 as mach
from mach_b200 import _check
from mach_b200.kernel import InterpolationType


def _data(n_rx=4, n_s=100, n_f=2, n_vox=8, seed=0):
    rng = np.random.default_rng(seed)
    rf = rng.normal(size=(n_rx, n_s, n_f)).astype(np.float32)
    iq = (rf + 1j * rng.normal(size=rf.shape)).astype(np.complex64)
    return rf, iq, rng.normal(size=(n_rx, 3)).astype(np.float32), rng.normal(size=(n_vox, 3)).astype(
        np.float32), np.zeros(n_vox, np.float32)


KW = dict(f_number=2.0, rx_start_s=0.0, sampling_freq_hz=1e6, sound_speed_m_s=1500.0)


def test_public_surface():
    for name in ("beamform", "kernel", "experimental", "wavefront", "geometry", "Array", "InterpolationType"):
        assert hasattr(mach, name)
    assert mach.kernel.nb_beamform is mach._cuda_impl.beamform
    assert [int(v) for v in InterpolationType] == [0, 1, 2]
    assert mach._cuda_impl.Linear is InterpolationType.Linear
    major, minor, _ = mach.kernel.__nvcc_version__.split(".")
    assert int(major) >= 12


def test_dimension_mismatch_raises_runtime_error():
    rf, iq, rx, grid, idt = _data()
    with pytest.raises(RuntimeError, match="Dimension mismatch in receive elements"):
        mach.beamform(iq[:2], rx, grid, idt, modulation_freq_hz=5e6, **KW)


def test_bool_channel_data_raises_type_error():
    rf, iq, rx, grid, idt = _data()
    with pytest.raises(TypeError, match="channel_data must be array with dtype=numeric"):
        mach.beamform(iq.astype(bool), rx, grid, idt, modulation_freq_hz=5e6, **KW)


def test_complex_requires_modulation_frequency():
    rf, iq, rx, grid, idt = _data()
    with pytest.raises(ValueError, match="modulation_freq_hz is required"):
        mach.beamform(iq, rx, grid, idt, **KW)


def test_out_dtype_mismatch():
    rf, iq, rx, grid, idt = _data()
    with pytest.raises(ValueError, match="doesn't match expected"):
        mach.beamform(rf, rx, grid, idt, out=np.zeros((8, 2), np.complex64), **KW)


def test_out_must_be_writable_and_contiguous():
    rf, iq, rx, grid, idt = _data()
    out = np.zeros((8, 2), np.float32)
    out.flags.writeable = False
    with pytest.raises(ValueError, match="not writable"):
        mach.beamform(rf, rx, grid, idt, out=out, **KW)
    with pytest.raises(ValueError, match="must be contiguous"):
        mach.beamform(rf, rx, grid, idt, out=np.zeros((2, 8), np.float32).T, **KW)


def test_native_overloads_reject_conversion():
    rf, iq, rx, grid, idt = _data()
    with pytest.raises(TypeError, match="incompatible function arguments"):
        mach.kernel.nb_beamform(rf.astype(np.float64), rx, grid, idt, np.zeros((8, 2), np.float32), 2.0, 0.0, 1e6,
                                1500.0)
    with pytest.raises(TypeError, match="incompatible function arguments"):
        mach.kernel.nb_beamform(iq, rx, grid, idt, np.zeros((8, 2), np.complex64), 2.0, 0.0, 1e6, 1500.0)


def test_contiguity_helpers():
    arr = np.arange(6, dtype=np.float32).reshape(2, 3)
    assert _check.is_contiguous(arr) and _check.ensure_contiguous(arr) is arr
    with pytest.warns(UserWarning, match="array is not contiguous"):
        fixed = _check.ensure_contiguous(arr.T)
    assert fixed.flags["C_CONTIGUOUS"]


def test_grid_hint_detection():
    from mach_b200 import _grid
    from tests import _helpers as H

    w = H.small("doppler", n_x=10, n_z=24)
    assert _grid.detect(w.scan_coords_m) == (10, 1, 24)
    w3 = H.small("volume3d", n_side=8)
    assert _grid.detect(w3.scan_coords_m) == (8, 8, 8)
    assert _grid.detect(np.random.default_rng(0).normal(size=(50, 3)).astype(np.float32)) is None
