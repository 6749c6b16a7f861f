"""The autotuner picks a launch that computes the same image and caches its choice."""

from __future__ import annotations

import json

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,storage", [("doppler", "c64"), ("doppler", "cf16"), ("compound", "c64")])
def test_tuned_launch_matches_default(cuda, tmp_path, monkeypatch, name, storage):
    import torch

    from mach_b200 import tuning
    from mach_b200 import workloads as W

    monkeypatch.setenv("MACH_B200_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setattr(tuning, "_MEMO", {})
    w = H.small(name, **({"n_frames": 32, "n_tx": 2} if name == "doppler" else {"n_tx": 4}))
    ch, scale = W.as_storage(w, storage)
    w.channel, w.channel_scale, w.storage = ch.contiguous(), scale, storage
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
            torch.as_tensor(w.scan_coords_m, device=dev), torch.as_tensor(w.tx_wave_arrivals_s, device=dev))
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    best = tuning.tune(*args, channel_scale=w.channel_scale, **p)
    assert best["kernel"] in ("lane_voxel", "staged", "ensemble", "warp")
    cached = json.loads((tmp_path / "tuning.json").read_text())
    assert len(cached) == 1 and list(cached.values())[0]["kernel"] == best["kernel"]
    assert tuning.tune(*args, channel_scale=w.channel_scale, **p) == best  # served from the cache
    tuned = H.gpu_compound(w, **best)
    default = H.gpu_compound(w)
    assert H.rel_l2(tuned, default) < 1e-5
    assert H.nrms_db(tuned, H.oracle(w)) < -60
