"""The ensemble kernel (lanes = frames, sample windows in tensor memory) computes the same
sums as the other kernel families, for every storage type, tap kind, frame count, window
size and tiling, and matches mach's kernel and the FP64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H
from tests.test_kernels_gpu import STORAGES, _run, _workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("interp", [0, 1])
def test_ensemble_matches_warp_kernel_and_oracle(cuda, storage, interp):
    n_frames = 64 if storage in ("c64", "cf16", "cbf16", "ci16") else 128
    w = _workload(storage, n_frames, interp)
    ens = _run(w, kernel="ensemble")
    warp = _run(w, kernel="warp")
    assert np.abs(ens).max() > 0
    assert H.rel_l2(ens, warp) <= 2e-6
    db = H.nrms_db(ens, H.oracle(w, storage=storage))
    assert db <= -60.0, f"{storage}: {db:.1f} dB vs the oracle on the stored samples"


@pytest.mark.parametrize("n_frames", [32, 40, 72, 100, 200])
def test_ensemble_frame_blocks(cuda, n_frames):
    w = _workload("c64", n_frames, 1)
    assert H.rel_l2(_run(w, kernel="ensemble"), _run(w, kernel="warp")) <= 2e-6


@pytest.mark.parametrize("n_frames", [64, 72, 136])
def test_ensemble_real_frame_pairs(cuda, n_frames):
    w = _workload("i16", n_frames, 1)
    assert H.rel_l2(_run(w, kernel="ensemble"), _run(w, kernel="warp")) <= 2e-6


@pytest.mark.parametrize("window_rows", [16, 32, 48, 64])
@pytest.mark.parametrize("grid", [None, False])
def test_ensemble_windows_and_tiling(cuda, window_rows, grid):
    """Small windows send most steps down the direct-load path; 1-D tiles have wide windows."""
    w = _workload("cf16", 64, 1)
    base = _run(w, kernel="warp")
    got = _run(w, kernel="ensemble", window_rows=window_rows, grid_shape=grid)
    assert H.rel_l2(got, base) <= 2e-6


def test_ensemble_many_transmits(cuda):
    """More transmits than are staged per tile: arrivals come from global memory."""
    w = H.small("doppler", n_x=12, n_z=20, n_tx=20, n_frames=32, n_elements=32)
    assert H.rel_l2(_run(w, kernel="ensemble"), _run(w, kernel="warp")) <= 2e-6


def test_ensemble_matches_reference_kernel(cuda):
    """FP32 storage with mach's FP32 delays: within 1e-5 of mach's own kernel."""
    w = H.small("doppler", n_frames=64)
    got = _run(w, kernel="ensemble", delay="reference")
    ref = H.reference_compound(w)
    assert H.rel_l2(got, ref) <= 1e-5


def test_ensemble_accumulates_into_gpu_out(cuda):
    import torch

    from mach_b200 import experimental

    w = _workload("c64", 64, 1)
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
            torch.as_tensor(w.scan_coords_m, device=dev), torch.as_tensor(w.tx_wave_arrivals_s, device=dev))
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    once = experimental.beamform(*args, kernel="ensemble", **p)
    out = once.clone()
    experimental.beamform(*args, out, kernel="ensemble", **p)
    torch.cuda.synchronize()
    assert torch.allclose(out, 2 * once, rtol=1e-6, atol=0)
