"""Power-Doppler image (sum over frames of |x|^2) fused into the beamformer: same values as
squaring and summing the beamformed frames, on the fused ensemble path and the general one."""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H
from tests.test_kernels_gpu import _workload

pytestmark = pytest.mark.gpu


def _args(w, dev="cuda"):
    import torch

    return (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
            torch.as_tensor(w.scan_coords_m, device=dev), torch.as_tensor(w.tx_wave_arrivals_s, device=dev))


@pytest.mark.parametrize("storage,n_frames", [("c64", 64), ("c64", 200), ("cf16", 32), ("ci16", 64), ("i16", 128),
                                              ("f32", 64)])
@pytest.mark.parametrize("kernel", ["auto", "ensemble", "warp"])
def test_power_matches_frames(cuda, storage, n_frames, kernel):
    import torch

    from mach_b200 import doppler, experimental

    w = _workload(storage, n_frames, 1)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    args = _args(w)
    frames = experimental.beamform(*args, channel_scale=w.channel_scale, kernel=kernel, **p)
    want = (frames.abs() ** 2).sum(dim=-1) if frames.is_complex() else (frames ** 2).sum(dim=-1)
    got = doppler.power_doppler(*args, channel_scale=w.channel_scale, kernel=kernel, **p)
    torch.cuda.synchronize()
    assert got.shape == (w.n_vox,) and got.dtype == torch.float32
    assert float(want.max()) > 0
    assert H.rel_l2(got.cpu().numpy(), want.cpu().numpy()) <= 1e-5


def test_power_accumulates_on_gpu_and_overwrites_on_cpu(cuda):
    import torch

    from mach_b200 import doppler

    w = _workload("c64", 64, 1)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    args = _args(w)
    once = doppler.power_doppler(*args, **p)
    out = once.clone()
    doppler.power_doppler(*args, out, **p)
    torch.cuda.synchronize()
    assert torch.allclose(out, 2 * once, rtol=1e-6)
    host = [np.asarray(a.cpu()) for a in args]
    out_h = np.full(w.n_vox, 5.0, dtype=np.float32)
    with pytest.warns(UserWarning):
        doppler.power_doppler(*host, out_h, **p)
    assert H.rel_l2(out_h, once.cpu().numpy()) <= 1e-5


@pytest.mark.parametrize("storage,kernel", [("c64", "auto"), ("c64", "ensemble"), ("cf16", "auto"),
                                            ("ci16", "ensemble")])
def test_power_vs_fp64_oracle(cuda, storage, kernel):
    """The power image against sum |x|^2 of the FP64 oracle's frames on the same stored samples
    (not against the library's own frames): -60 dB, the project's bar against the oracle."""
    import torch

    from mach_b200 import doppler

    w = _workload(storage, 64, 1)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    got = doppler.power_doppler(*_args(w), channel_scale=w.channel_scale, kernel=kernel, **p)
    torch.cuda.synchronize()
    frames = H.oracle(w, storage=storage)
    want = (np.abs(frames) ** 2).sum(axis=1)
    assert want.max() > 0
    assert H.nrms_db(got.cpu().numpy(), want) <= -60.0
