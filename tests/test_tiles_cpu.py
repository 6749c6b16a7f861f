"""Voxel-to-CTA assignment of the voxel-per-lane kernels on a known grid, restated on the CPU.

A CTA of `vpc` voxels (128 / lanes per voxel) takes a tile of wf voxels along the contiguous
(fast) axis times vpc / wf along the next one.  In grid order tiles run outer-major; with
`tile_rev` they run fast-axis-major from the far end of the fast axis (the deepest tiles of a
depth-fastest scan first).  Whatever the order and shape, every voxel of the grid belongs to
exactly one (tile, thread) and the launch has exactly the planner's number of tiles
(mach_b200_capi.cu, plan_launch; das_lane_voxel.cuh, lane_voxel_index).
"""

from __future__ import annotations

import numpy as np
import pytest


def tiles(n_outer: int, n_fast: int, vpc: int, wf: int) -> int:
    per_outer = vpc // wf
    return -(-n_outer // per_outer) * -(-n_fast // wf)


def voxel(tile: int, j: int, n_outer: int, n_fast: int, vpc: int, wf: int, rev: bool) -> int:
    """Voxel of thread j of `tile` (n_outer * n_fast for none): the device function's arithmetic."""
    lw = wf.bit_length() - 1
    tiles_fast = (n_fast + wf - 1) >> lw
    per_outer = vpc >> lw
    if rev:
        tiles_outer = (n_outer + per_outer - 1) // per_outer
        q = tile // tiles_outer
        to, tf = tile - q * tiles_outer, tiles_fast - 1 - q
    else:
        to = tile // tiles_fast
        tf = tile - to * tiles_fast
    o = to * per_outer + (j >> lw)
    f = (tf << lw) + (j & (wf - 1))
    return o * n_fast + f if (o < n_outer and f < n_fast) else n_outer * n_fast


@pytest.mark.parametrize("rev", [False, True])
@pytest.mark.parametrize("vpc", [128, 64, 32])
@pytest.mark.parametrize("wf", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("shape", [(37, 45), (512, 512), (1, 300), (129, 7), (64, 1)])
def test_every_voxel_in_exactly_one_tile(rev, vpc, wf, shape):
    n_outer, n_fast = shape
    if wf > n_fast:  # the planner falls back to runs of consecutive voxels
        return
    n_vox = n_outer * n_fast
    seen = np.zeros(n_vox + 1, dtype=np.int64)
    for t in range(tiles(n_outer, n_fast, vpc, wf)):
        for j in range(vpc):
            seen[voxel(t, j, n_outer, n_fast, vpc, wf, rev)] += 1
    assert (seen[:n_vox] == 1).all()


def test_deepest_tiles_first():
    """With tile_rev the first tiles hold the last fast-axis (deepest) voxels, the last tiles
    the first ones, and consecutive tiles sit side by side along the outer axis."""
    n_outer, n_fast, vpc, wf = 512, 512, 64, 4
    first = [voxel(0, j, n_outer, n_fast, vpc, wf, True) % n_fast for j in range(vpc)]
    last = [voxel(tiles(n_outer, n_fast, vpc, wf) - 1, j, n_outer, n_fast, vpc, wf, True) % n_fast
            for j in range(vpc)]
    assert min(first) == n_fast - wf and max(last) == wf - 1
    a = voxel(0, 0, n_outer, n_fast, vpc, wf, True)
    b = voxel(1, 0, n_outer, n_fast, vpc, wf, True)
    assert a % n_fast == b % n_fast and b // n_fast - a // n_fast == vpc // wf
