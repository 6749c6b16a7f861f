"""Transmit arrivals computed on the device (plane / spherical wave models) give the image
that the host-computed arrivals array gives, on every kernel family."""

from __future__ import annotations

import numpy as np
import pytest

from mach_b200 import geometry, wavefront
from tests import _helpers as H

pytestmark = pytest.mark.gpu


def _plane_waves(angles_deg):
    a = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
    dirs = geometry.ultrasound_angles_to_cartesian(a, np.zeros_like(a))  # [n, 3]
    return wavefront.PlaneWaves(np.zeros(3), dirs)


def _run(w, arrivals, **kw):
    import torch

    from mach_b200 import experimental

    dev = "cuda"
    arr = arrivals if isinstance(arrivals, wavefront.TransmitWaves) else torch.as_tensor(arrivals, device=dev)
    out = experimental.beamform(w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
                                torch.as_tensor(w.scan_coords_m, device=dev), arr, channel_scale=w.channel_scale,
                                **{k: w.params[k] for k in H.PARAM_KEYS}, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name,kw", [("compound", {}), ("doppler", {"kernel": "ensemble"}),
                                     ("doppler", {"kernel": "staged"}), ("doppler", {"kernel": "warp"})])
def test_plane_wave_model_matches_arrays(cuda, name, kw):
    w = H.small(name, n_tx=4) if name == "compound" else H.small("doppler", n_tx=3, n_frames=40)
    angles = np.linspace(-16, 16, w.n_tx) if name == "compound" else np.linspace(-4, 4, w.n_tx)
    waves = _plane_waves(angles)
    c = w.params["sound_speed_m_s"]
    arrays = waves.arrivals(w.scan_coords_m.astype(np.float64), c).astype(np.float32)
    want = _run(w, arrays, **kw)
    got = _run(w, waves, **kw)
    assert np.abs(want).max() > 0
    assert H.rel_l2(got, want) <= 1e-6


def test_spherical_model_matches_arrays(cuda):
    w = H.small("volume3d", n_side=10, n_elem_side=8, n_frames=1)
    foci = np.array([[x, y, -10e-3] for x in (-3e-3, 0, 3e-3) for y in (-3e-3, 0, 3e-3)])
    waves = wavefront.SphericalWaves(np.zeros(3), foci)
    arrays = waves.arrivals(w.scan_coords_m.astype(np.float64), w.params["sound_speed_m_s"]).astype(np.float32)
    want = _run(w, arrays)
    got = _run(w, waves)
    assert H.rel_l2(got, want) <= 1e-6


def test_plane_wave_model_power_doppler_and_host_inputs(cuda):
    import torch

    from mach_b200 import doppler, experimental

    w = H.small("doppler", n_tx=3, n_frames=64)
    waves = _plane_waves(np.linspace(-4, 4, w.n_tx))
    c = w.params["sound_speed_m_s"]
    arrays = waves.arrivals(w.scan_coords_m.astype(np.float64), c).astype(np.float32)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev), torch.as_tensor(w.scan_coords_m, device=dev))
    want = doppler.power_doppler(*args, torch.as_tensor(arrays, device=dev), **p).cpu().numpy()
    got = doppler.power_doppler(*args, waves, **p).cpu().numpy()
    assert want.max() > 0
    assert H.rel_l2(got, want) <= 1e-5  # frame blocks add in any order
    # host inputs: the wave table is staged next to the transmit chunks
    frames = _run(w, arrays)
    with pytest.warns(UserWarning, match="on CPU"):
        host = experimental.beamform(w.channel.numpy(), w.rx_coords_m, w.scan_coords_m, waves, **p)
    assert H.rel_l2(host, frames) <= 1e-6


def test_tx_model_errors(cuda):
    import torch

    from mach_b200 import experimental

    w = H.small("compound", n_tx=4)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev), torch.as_tensor(w.scan_coords_m, device=dev))
    with pytest.raises(RuntimeError, match="transmit waves"):
        experimental.beamform(*args, _plane_waves([0.0, 1.0]), **p)
    bad = _plane_waves(np.linspace(-16, 16, 4))
    bad.model = 7
    with pytest.raises(RuntimeError, match="tx_model"):
        experimental.beamform(*args, bad, **p)
