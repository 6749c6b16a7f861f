"""Autotuner candidate lists (host logic only)."""

from mach_b200 import tuning


def test_candidates_cover_the_families():
    kinds = {c["kernel"] for c in tuning.candidates("c64", 64, (1, 256, 256))}
    assert kinds == {"staged", "ensemble", "warp"}
    kinds = {c["kernel"] for c in tuning.candidates("cf16", 16, None)}
    assert kinds == {"lane_voxel", "staged", "warp"}
    assert {c["kernel"] for c in tuning.candidates("f32", 1, None)} == {"lane_voxel"}


def test_staged_lanes_respect_storage_limits():
    for c in tuning.candidates("cbf16", 200, (1, 64, 64)):
        if c["kernel"] == "staged":
            assert c["lanes_per_voxel"] <= 16
    lanes = {c["lanes_per_voxel"] for c in tuning.candidates("c64", 200, None) if c["kernel"] == "staged"}
    assert lanes == {4, 8, 16, 32}
    # no lane count that leaves half the lanes idle
    lanes = {c["lanes_per_voxel"] for c in tuning.candidates("c64", 8, None) if c["kernel"] == "staged"}
    assert lanes == {4, 8}
