"""Every kernel family computes the same sums: staged-window (TMA and direct loads),
warp-per-voxel and voxel-per-lane, for every storage type and interpolation, with and
without a voxel-grid tiling hint; each is also checked against the FP64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu

STORAGES = ["f32", "c64", "f16", "cf16", "bf16", "cbf16", "i16", "ci16"]


def _workload(storage: str, n_frames: int, interp: int):
    """Small multi-frame job in the requested storage (complex ones from the Doppler physics)."""
    import torch

    if storage in ("c64", "cf16", "cbf16", "ci16"):
        w = H.small("doppler", n_x=10, n_z=24, n_tx=2, n_frames=n_frames, n_elements=48)
        ch = w.channel
        if storage == "cf16":
            ch = torch.view_as_real(ch).to(torch.float16).contiguous()
        elif storage == "cbf16":
            ch = torch.view_as_real(ch).to(torch.bfloat16).contiguous()
        elif storage == "ci16":
            scale = float(torch.view_as_real(ch).abs().max()) / 20000.0
            ch = (torch.view_as_real(ch) / scale).round().to(torch.int16).contiguous()
            w.channel_scale = scale
    else:
        w = H.small("volume3d", n_side=6, n_elem_side=8, n_frames=n_frames, n_samples=1400)
        ch = w.channel
        if storage == "f32":
            ch = ch.to(torch.float32) * w.channel_scale
            w.channel_scale = 1.0
        elif storage in ("f16", "bf16"):
            ch = (ch.to(torch.float32) * w.channel_scale).to(torch.float16 if storage == "f16" else torch.bfloat16)
            w.channel_scale = 1.0
    w.channel = ch.contiguous()
    w.storage = storage
    w.params["interp_type"] = interp
    return w


def _run(w, **kw):
    return H.gpu_compound(w, **kw)


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("interp", [0, 1, 2])
def test_staged_matches_warp_kernel_and_oracle(cuda, storage, interp):
    w = _workload(storage, 16, interp)
    staged = _run(w, kernel="staged")
    warp = _run(w, kernel="warp")
    direct = _run(w, kernel="staged", window_rows=4)  # windows never fit: taps from global memory
    flat = _run(w, kernel="staged", grid_shape=False)  # 1-D tiles
    assert np.abs(staged).max() > 0
    for other in (warp, direct, flat):
        assert H.rel_l2(staged, other) <= 2e-6
    db = H.nrms_db(staged, H.oracle(w, storage=storage))
    assert db <= -60.0, f"{storage}: {db:.1f} dB vs the oracle on the stored samples"


@pytest.mark.parametrize("n_frames", [9, 12, 16, 24, 32, 40, 64, 72])
def test_staged_frame_chunks(cuda, n_frames):
    w = _workload("c64", n_frames, 1)
    staged = _run(w, kernel="staged")
    warp = _run(w, kernel="warp")
    assert H.rel_l2(staged, warp) <= 2e-6


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
@pytest.mark.parametrize("window_rows", [16, 64, 256])
def test_staged_tuning_knobs_do_not_change_results(cuda, lanes, window_rows):
    w = _workload("cf16", 32, 2)
    base = _run(w, kernel="warp")
    got = _run(w, kernel="staged", lanes_per_voxel=lanes, window_rows=window_rows)
    assert H.rel_l2(got, base) <= 2e-6


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("n_frames", [1, 3])
def test_lane_voxel_storage(cuda, storage, n_frames):
    w = _workload(storage, n_frames, 2)
    got = _run(w)
    tuned = _run(w, tx_chunk=1)  # transmit-major summation order: FP32 rounding only
    assert H.rel_l2(got, tuned) <= 1e-5
    assert H.nrms_db(got, H.oracle(w, storage=storage)) <= -60.0


@pytest.mark.parametrize("interp", [0, 1, 2])
@pytest.mark.parametrize("kernel", ["lane_voxel", "staged"])
def test_split_delay_is_more_accurate(cuda, interp, kernel):
    """Split delays (FP64 per path, integer base + FP32 fraction) beat mach's FP32 delays
    against the FP64 oracle, on both kernel families."""
    w = H.small("compound") if kernel == "lane_voxel" else _workload("c64", 16, interp)
    w.params["interp_type"] = interp
    want = H.oracle(w)
    ref_db = H.nrms_db(_run(w, kernel=kernel, delay="reference"), want)
    split_db = H.nrms_db(_run(w, kernel=kernel, delay="split"), want)
    print(f"{kernel} interp {interp}: reference delays {ref_db:.1f} dB, split delays {split_db:.1f} dB")
    assert split_db <= ref_db + 0.5
    assert split_db <= -75.0


@pytest.mark.parametrize("storage", ["cf16", "ci16", "f16", "i16"])
def test_split_delay_reduced_storage(cuda, storage):
    w = _workload(storage, 16, 1)
    got = _run(w)  # delay="auto" selects split delays for reduced storage
    assert H.nrms_db(got, H.oracle(w, storage=storage)) <= -75.0


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("interp", [0, 1, 2])
def test_lane_voxel_sixteen_frames(cuda, storage, interp):
    """16-frame jobs take the vectorised voxel-per-lane path; it matches the other families."""
    w = _workload(storage, 16, interp)
    lane = _run(w, kernel="lane_voxel")
    warp = _run(w, kernel="warp")
    assert H.rel_l2(lane, warp) <= 2e-6
    assert H.nrms_db(lane, H.oracle(w, storage=storage)) <= -60.0


@pytest.mark.parametrize("name,n_frames", [("compound", 1), ("volume3d", 16), ("volume3d", 3)])
def test_lane_voxel_grid_tiles_are_bit_identical(cuda, name, n_frames):
    """The voxel-to-warp assignment on a grid (4 x 8, 2 x 16, ... neighbours, edge tiles
    partly empty) and the order in which CTAs take the tiles change which thread sums a voxel,
    never the sum."""
    if name == "compound":
        w = H.small("compound", n_x=37, n_z=45, n_tx=3)  # extents not multiples of the tiles
    else:
        w = H.small("volume3d", n_side=7, n_elem_side=8, n_frames=n_frames, n_samples=1400)
    base = _run(w, kernel="lane_voxel", grid_shape=False)
    for tile_order in (0, 1, 2):  # automatic, far end of the contiguous axis first, grid order
        for tile_fast in (0, 1, 2, 4, 8, 16):
            got = _run(w, kernel="lane_voxel", tile_fast=tile_fast, tile_order=tile_order)
            np.testing.assert_array_equal(got, base)
    assert np.abs(base).max() > 0


@pytest.mark.parametrize("name,storage", [("compound", "c64"), ("compound", "cf16"), ("plain2d", "f32"),
                                          ("volume3d", "i16")])
def test_lane_voxel_lanes_per_voxel(cuda, name, storage):
    """One-frame jobs summed by 1, 2 or 4 lanes per voxel (each lane every 2nd / 4th element,
    partial sums added by warp shuffles) agree to FP32 rounding and with the oracle."""
    import torch

    if name == "compound":
        w = H.small("compound", n_tx=5)
    elif name == "plain2d":
        w = H.small("plain2d")
    else:
        w = H.small("volume3d", n_side=10, n_elem_side=8, n_frames=1)
    if storage == "cf16":
        w.channel = torch.view_as_real(w.channel).to(torch.float16).contiguous()
        w.storage = "cf16"
    results = [_run(w, kernel="lane_voxel", lanes_per_voxel=lanes) for lanes in (1, 2, 4)]
    assert np.abs(results[0]).max() > 0
    for r in results[1:]:
        assert H.rel_l2(r, results[0]) <= 1e-6
    assert H.nrms_db(results[2], H.oracle(w, storage=storage)) <= -60.0


@pytest.mark.parametrize("storage", ["c64", "cf16", "cbf16", "ci16", "f16", "i16", "f32"])
@pytest.mark.parametrize("n_frames", [24, 40])
def test_lane_voxel_frame_chunks(cuda, storage, n_frames):
    """Ensembles longer than 16 frames in chunks of 8 frames per CTA row (the automatic kernel
    for 4-byte complex storage) give the ensemble / warp kernels' sums."""
    w = _workload(storage, n_frames, 1)
    chunks = _run(w, kernel="lane_voxel")
    other = _run(w, kernel="warp")
    assert np.abs(chunks).max() > 0
    assert H.rel_l2(chunks, other) <= 2e-6
    for tile_order in (1, 2):  # the order in which CTAs take the tiles never changes a sum
        np.testing.assert_array_equal(_run(w, kernel="lane_voxel", tile_order=tile_order), chunks)
    assert H.nrms_db(chunks, H.oracle(w, storage=storage)) <= -60.0
    if storage in ("cf16", "cbf16", "ci16"):
        np.testing.assert_array_equal(_run(w), chunks)  # the automatic choice


@pytest.mark.parametrize("block", [32, 64, -1])
def test_lane_voxel_element_blocks(cuda, block):
    """A job run as one launch per block of elements (accumulating) gives the one-launch sums
    to FP32 rounding, and the oracle's."""
    w = H.small("volume3d", n_side=8, n_elem_side=12, n_frames=16, n_samples=1400)  # 144 elements
    one = _run(w, kernel="lane_voxel", element_block=-1)
    got = _run(w, kernel="lane_voxel", element_block=block)
    assert np.abs(one).max() > 0
    assert H.rel_l2(got, one) <= 1e-6
    assert H.nrms_db(got, H.oracle(w)) <= -60.0


@pytest.mark.parametrize("block", [32, 50])
def test_element_blocks_from_host_memory(cuda, block):
    """Host channel data of an element-block job is copied block by block (one 2-D copy of the
    block's rows of every transmit) while earlier blocks run: the sums are bit-identical to the
    same blocks on device inputs, for pageable and pinned memory, int16 and FP32 storage."""
    import torch

    from mach_b200 import experimental

    w = H.small("volume3d", n_side=8, n_elem_side=12, n_frames=16, n_samples=1400)  # 144 elements
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    for storage in ("i16", "f32"):
        ch, scale = H.W.as_storage(w, storage)
        ch = ch.cpu().contiguous()
        dev_out = torch.zeros((w.n_vox, w.n_frames), dtype=torch.float32, device="cuda")
        experimental.beamform(ch.cuda(), torch.as_tensor(w.rx_coords_m, device="cuda"),
                              torch.as_tensor(w.scan_coords_m, device="cuda"),
                              torch.as_tensor(w.tx_wave_arrivals_s, device="cuda"), dev_out, channel_scale=scale,
                              kernel="lane_voxel", element_block=block, **p)
        want = dev_out.cpu().numpy()
        assert np.abs(want).max() > 0
        for pin in (False, True):
            host_ch = ch.pin_memory() if pin else ch
            out = torch.full((w.n_vox, w.n_frames), 3.0, dtype=torch.float32)  # a CPU out is overwritten
            with pytest.warns(UserWarning, match="latency"):
                experimental.beamform(host_ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, out,
                                      channel_scale=scale, kernel="lane_voxel", element_block=block, **p)
            np.testing.assert_array_equal(out.numpy(), want)
