"""The FP64 oracles: NumPy and C agree, and both satisfy known answers derived by hand."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import das_fp64, oracle_c
from tests import _helpers as H


@pytest.mark.parametrize("name", ["plain2d", "compound", "doppler", "volume3d"])
def test_numpy_and_c_oracles_agree(name):
    w = H.small(name, **({"n_frames": 5} if name == "doppler" else {}))
    ch = H.channel_numpy(w.channel)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    a = das_fp64.beamform_fp64(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s,
                               channel_scale=w.channel_scale, **p)
    b = H.oracle(w)
    assert np.abs(a).max() > 0
    assert das_fp64.rel_l2(b, a) < 1e-12


@pytest.mark.parametrize("interp", [0, 1, 2])
@pytest.mark.parametrize("alpha", [0.0, 0.3, 1.0])
def test_parameter_grid_agrees(interp, alpha):
    w = H.small("compound", n_x=10, n_z=12, n_tx=2)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    p.update(interp_type=interp, tukey_alpha=alpha)
    ch = H.channel_numpy(w.channel)
    a = das_fp64.beamform_fp64(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, **p)
    b = oracle_c.beamform_c(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, storage="c64", **p)
    assert das_fp64.rel_l2(b, a) < 1e-12


def _single(channel, voxel, element, arrival, **kw):
    params = dict(f_number=0.5, rx_start_s=0.0, sampling_freq_hz=10e6, sound_speed_m_s=1500.0,
                  modulation_freq_hz=0.0, tukey_alpha=0.0, interp_type=1)
    params.update(kw)
    return das_fp64.beamform_fp64(np.asarray(channel)[None], np.array([element]), np.array([voxel]),
                                  np.array([arrival]), **params)


def test_known_answer_linear_ramp():
    # element under the voxel at depth 15 mm: tau = 10 us + 15 mm / 1500 m/s = 20 us -> s = 200.
    ramp = np.arange(512, dtype=np.float64)[:, None]
    out = _single(ramp, [0, 0, 15e-3], [0, 0, 0], 10e-6)
    assert out[0, 0] == pytest.approx(200.0, abs=1e-9)
    out = _single(ramp, [0, 0, 15e-3], [0, 0, 0], 10.025e-6)
    assert out[0, 0] == pytest.approx(200.25, abs=1e-9)


def test_known_answer_quadratic_exact_on_parabola():
    s = np.arange(512, dtype=np.float64)
    parabola = (0.5 * s * s - 3 * s + 1)[:, None]
    out = _single(parabola, [0, 0, 15e-3], [0, 0, 0], 10.037e-6, interp_type=2)
    x = 200.37
    assert out[0, 0] == pytest.approx(0.5 * x * x - 3 * x + 1, rel=1e-12)


def test_known_answer_nearest_rounds_half_to_even():
    # voxel on the element (zero receive path, zero aperture radius still admits it) and fs = 1 Hz,
    # so the sample index equals the arrival time exactly.
    ramp = np.arange(512, dtype=np.float64)[:, None]
    kw = dict(interp_type=0, sampling_freq_hz=1.0)
    assert _single(ramp, [0, 0, 0], [0, 0, 0], 200.5, **kw)[0, 0] == 200.0  # 200.5 -> 200
    assert _single(ramp, [0, 0, 0], [0, 0, 0], 201.5, **kw)[0, 0] == 202.0  # 201.5 -> 202
    assert _single(ramp, [0, 0, 0], [0, 0, 0], -0.5, **kw)[0, 0] == 0.0  # lower bound -0.5 is inside
    assert _single(ramp, [0, 0, 0], [0, 0, 0], -0.25, **kw)[0, 0] == 0.0
    # upper bound n - 0.5 = 511.5 is inside the reference's test but rounds to 512: treated as outside
    assert _single(ramp + 1, [0, 0, 0], [0, 0, 0], 511.5, **kw)[0, 0] == 0.0
    assert _single(ramp + 1, [0, 0, 0], [0, 0, 0], 511.25, **kw)[0, 0] == 512.0


def test_known_answer_aperture_and_tukey():
    ones = np.ones((512, 1))
    # f# 1 at depth 20 mm: radius 10 mm.  Element 4 mm off axis: r = 0.4.
    kw = dict(f_number=1.0, tukey_alpha=1.0)
    w = _single(ones, [0, 0, 20e-3], [4e-3, 0, 0], 0.0, **kw)[0, 0]
    assert w == pytest.approx(0.5 - 0.5 * np.cos(np.pi * 0.6), rel=1e-12)
    # inside the flat part for alpha 0.5
    assert _single(ones, [0, 0, 20e-3], [4e-3, 0, 0], 0.0, f_number=1.0, tukey_alpha=0.5)[0, 0] == 1.0
    # outside the aperture
    assert _single(ones, [0, 0, 20e-3], [10.5e-3, 0, 0], 0.0, f_number=1.0)[0, 0] == 0.0
    # the element's z does not enter the aperture radius, only the range
    assert _single(ones, [0, 0, 20e-3], [9e-3, 0, 5e-3], 0.0, f_number=1.0)[0, 0] == 1.0


def test_known_answer_negative_delay_and_bounds_skipped():
    ones = np.ones((512, 1))
    assert _single(ones, [0, 0, 15e-3], [0, 0, 0], -20e-6)[0, 0] == 0.0  # tau < 0
    assert _single(ones, [0, 0, 15e-3], [0, 0, 0], 50e-6)[0, 0] == 0.0  # s = 600 > 511


def test_known_answer_iq_rotation():
    iq = np.ones((512, 1), dtype=np.complex128)
    f_mod = 3e6
    out = _single(iq, [0, 0, 15e-3], [0, 0, 0], 10e-6, modulation_freq_hz=f_mod)[0, 0]
    assert out == pytest.approx(np.exp(1j * 2 * np.pi * f_mod * 20e-6), abs=1e-12)


def test_compounding_is_sum_over_transmits():
    w = H.small("compound", n_x=8, n_z=10, n_tx=3)
    ch = H.channel_numpy(w.channel)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    total = das_fp64.beamform_fp64(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, **p)
    parts = sum(das_fp64.beamform_fp64(ch[t], w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s[t], **p)
                for t in range(3))
    assert das_fp64.rel_l2(total, parts) < 1e-13


def test_reduced_storage_decoding():
    """The C oracle decodes float16 / bfloat16 / int16 pairs exactly like the float widening."""
    import torch

    from mach_b200 import workloads as W

    w = H.small("compound", n_x=6, n_z=8, n_tx=2)
    for storage in ("cf16", "cbf16"):
        stored = W.to_storage(w, storage)
        widened = torch.view_as_complex(stored.to(torch.float32).contiguous())
        a = H.oracle(w, channel=stored, storage=storage)
        b = H.oracle(w, channel=widened, storage="c64")
        assert das_fp64.rel_l2(a, b) < 1e-12
