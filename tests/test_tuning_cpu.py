"""Autotuner candidate lists (host logic only)."""

from mach_b200 import tuning


def test_candidates_cover_the_families():
    kinds = {c["kernel"] for c in tuning.candidates("c64", 64, (1, 256, 256))}
    assert kinds == {"staged", "ensemble", "warp", "lane_voxel", "frame_lane"}
    kinds = {c["kernel"] for c in tuning.candidates("cf16", 16, None)}
    assert kinds == {"lane_voxel", "staged", "warp"}
    assert {c["kernel"] for c in tuning.candidates("f32", 1, None)} == {"lane_voxel"}
    # long ensembles: 8-frame chunks of the voxel-per-lane kernel next to the ensemble kernel
    kinds = {c["kernel"] for c in tuning.candidates("cf16", 200, (1, 256, 256))}
    assert {"lane_voxel", "ensemble", "staged", "warp", "frame_lane"} <= kinds


def test_frame_lane_knobs():
    """Frame columns per warp that would leave whole columns empty are not tried."""
    def knobs(storage, n_frames):
        return {c["frame_slots"] for c in tuning.candidates(storage, n_frames, (256, 1, 256))
                if c["kernel"] == "frame_lane"}

    assert knobs("c64", 200) == {1, 2, 4}
    assert knobs("c64", 32) == {1}
    assert knobs("c64", 64) == {1, 2}
    assert knobs("i16", 128) == {1, 2}  # 64 lane words of two frames
    assert knobs("c64", 16) == set()
    assert knobs("i16", 33) == set()  # odd real frame counts have no lane words of two frames


def test_lane_voxel_knobs():
    one = [c for c in tuning.candidates("c64", 1, (1, 512, 512)) if c["kernel"] == "lane_voxel"]
    assert {c["lanes_per_voxel"] for c in one} == {1, 2, 4}
    assert {c["tile_fast"] for c in one} == {2, 4, 8}
    assert {c["tx_chunk"] for c in one} == {8, 16, 32, 40}
    no_grid = [c for c in tuning.candidates("c64", 1, None) if c["kernel"] == "lane_voxel"]
    assert {c["tile_fast"] for c in no_grid} == {0}


def test_staged_lanes_respect_storage_limits():
    for c in tuning.candidates("cbf16", 200, (1, 64, 64)):
        if c["kernel"] == "staged":
            assert c["lanes_per_voxel"] <= 16
    lanes = {c["lanes_per_voxel"] for c in tuning.candidates("c64", 200, None) if c["kernel"] == "staged"}
    assert lanes == {4, 8, 16, 32}
    # no lane count that leaves half the lanes idle
    lanes = {c["lanes_per_voxel"] for c in tuning.candidates("c64", 8, None) if c["kernel"] == "staged"}
    assert lanes == {4, 8}


def test_lookup_reads_the_cache_written_by_the_tuner(tmp_path, monkeypatch):
    """Automatic calls find the knobs the tuner stored for the same job shape, device and
    delay mode (auto resolved as the call resolves it), and nothing for other shapes."""
    monkeypatch.setenv("MACH_B200_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setattr(tuning, "_MEMO", {})
    monkeypatch.setattr(tuning, "_LOADED", False)
    monkeypatch.setitem(tuning._DEVICE_NAMES, 0, "NVIDIA B200")
    grid = (128, 128, 128)
    key = tuning._key("i16", 9, 1024, 2048, 16, 128 ** 3, grid, 1, "NVIDIA B200", tuning.resolve_delay("i16", "auto"))
    tuning._store(key, {"kernel": "lane_voxel", "element_block": 64, "ms": 70.0})
    assert tuning.resolve_delay("i16", "auto") == "split" and tuning.resolve_delay("c64", "auto") == "reference"
    hit = tuning.lookup("i16", 9, 1024, 2048, 16, 128 ** 3, grid, 1, 0, "split")
    assert hit == {"kernel": "lane_voxel", "element_block": 64}
    assert tuning.lookup("i16", 9, 1024, 2048, 16, 128 ** 3, grid, 1, 0, "reference") is None
    assert tuning.lookup("i16", 9, 1024, 2048, 1, 128 ** 3, grid, 1, 0, "auto") is None
