"""The frame-lane kernel (lanes = frames, sample rows kept in registers along voxel runs)
computes the same sums as the other kernel families for every storage type, tap kind, frame
count, run length, row span and tiling, matches mach's kernel and the FP64 oracle,
accumulates into a GPU `out`, and fuses the power-Doppler epilogue."""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H
from tests.test_kernels_gpu import STORAGES, _run, _workload

pytestmark = pytest.mark.gpu

CPLX = ("c64", "cf16", "cbf16", "ci16")


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("interp", [0, 1])
def test_frame_lane_matches_warp_kernel_and_oracle(cuda, storage, interp):
    n_frames = 64 if storage in CPLX else 128
    w = _workload(storage, n_frames, interp)
    got = _run(w, kernel="frame_lane")
    warp = _run(w, kernel="warp")
    assert np.abs(got).max() > 0
    assert H.rel_l2(got, warp) <= 2e-6
    db = H.nrms_db(got, H.oracle(w, storage=storage))
    assert db <= -60.0, f"{storage}: {db:.1f} dB vs the oracle on the stored samples"


@pytest.mark.parametrize("n_frames", [32, 33, 40, 64, 72, 100, 129, 200])
@pytest.mark.parametrize("slots", [1, 2, 4])
def test_frame_lane_frame_chunks(cuda, n_frames, slots):
    """Partial lane-word columns and several frame chunks per run, for every run length."""
    w = _workload("c64", n_frames, 1)
    got = _run(w, kernel="frame_lane", frame_slots=slots)
    assert H.rel_l2(got, _run(w, kernel="warp")) <= 2e-6


@pytest.mark.parametrize("n_frames", [64, 66, 130])
def test_frame_lane_real_frame_pairs(cuda, n_frames):
    w = _workload("i16", n_frames, 1)
    assert H.rel_l2(_run(w, kernel="frame_lane"), _run(w, kernel="warp")) <= 2e-6


@pytest.mark.parametrize("grid", [None, False])
def test_frame_lane_tiling(cuda, grid):
    """Runs along the grid's lateral axis, or of consecutive voxels without a grid."""
    w = _workload("cf16", 64, 1)
    base = _run(w, kernel="warp")
    got = _run(w, kernel="frame_lane", grid_shape=grid)
    assert H.rel_l2(got, base) <= 2e-6


def test_frame_lane_wide_row_spans(cuda):
    """A coarse lateral grid: the rows of one element's voxels span more than the four held at
    once, so points load their rows one voxel at a time."""
    w = H.small("doppler", n_x=9, n_z=16, n_tx=2, n_frames=64, n_elements=40)  # 4 mm lateral steps
    assert H.rel_l2(_run(w, kernel="frame_lane"), _run(w, kernel="warp")) <= 2e-6


def test_frame_lane_ragged_grid(cuda):
    """Grid extents that are not multiples of the run length (runs end early)."""
    w = H.small("doppler", n_x=13, n_z=7, n_tx=3, n_frames=48, n_elements=40)
    for slots in (1, 2, 4):
        got = _run(w, kernel="frame_lane", frame_slots=slots)
        assert H.rel_l2(got, _run(w, kernel="warp")) <= 2e-6


def test_frame_lane_3d_grid(cuda):
    """Runs along the mid axis of a 3-D grid, real storage with many frames."""
    w = _workload("f16", 64, 1)
    assert w.grid_shape and len(w.grid_shape) == 3
    assert H.rel_l2(_run(w, kernel="frame_lane"), _run(w, kernel="warp")) <= 2e-6


def test_frame_lane_matches_reference_kernel(cuda):
    """FP32 storage with mach's FP32 delays: within 1e-5 of mach's own kernel."""
    from oracle import machref

    if not machref.available():
        pytest.skip("reference kernel library not built")
    w = H.small("doppler", n_frames=64)
    got = _run(w, kernel="frame_lane", delay="reference")
    ref = H.reference_compound(w)
    assert H.rel_l2(got, ref) <= 1e-5


def test_frame_lane_accumulates_into_gpu_out(cuda):
    import torch

    from mach_b200 import experimental

    w = _workload("c64", 64, 1)
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
            torch.as_tensor(w.scan_coords_m, device=dev), torch.as_tensor(w.tx_wave_arrivals_s, device=dev))
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    once = experimental.beamform(*args, kernel="frame_lane", **p)
    out = once.clone()
    experimental.beamform(*args, out, kernel="frame_lane", **p)
    torch.cuda.synchronize()
    assert torch.allclose(out, 2 * once, rtol=1e-6, atol=0)


@pytest.mark.parametrize("storage", ["c64", "cf16"])
def test_frame_lane_power_doppler_vs_oracle(cuda, storage):
    """The fused power-Doppler epilogue against sum |x|^2 of the FP64 oracle's frames."""
    import torch

    from mach_b200 import doppler

    w = _workload(storage, 72, 1)
    dev = "cuda"
    args = (w.channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev),
            torch.as_tensor(w.scan_coords_m, device=dev), torch.as_tensor(w.tx_wave_arrivals_s, device=dev))
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    got = doppler.power_doppler(*args, channel_scale=w.channel_scale, kernel="frame_lane", **p)
    torch.cuda.synchronize()
    frames = H.oracle(w, storage=storage)
    want = (np.abs(frames) ** 2).sum(axis=1)
    err = np.linalg.norm(got.cpu().numpy() - want) / np.linalg.norm(want)
    # -60 dB on the power image, the project's bar against the oracle (FP32 frames are
    # about -85 dB from it, and squaring doubles the relative error)
    assert err <= 1e-3, f"power Doppler rel L2 {err:.2e} vs the FP64 oracle"
