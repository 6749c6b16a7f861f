"""Voxel sharding across ranks: world_size-2 gloo processes on CPU.

The per-rank compute here is the FP64 oracle (no GPU on this machine); the sharding,
slicing and image assembly are the same code the GPU path uses.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from mach_b200.distributed import shard_range


@pytest.mark.parametrize("n_vox", [1, 127, 128, 1000, 65536, 65537])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_cover_exactly_once(n_vox, world):
    covered = np.zeros(n_vox, dtype=int)
    for r in range(world):
        a, b = shard_range(n_vox, world, r)
        assert a % 128 == 0 or a == n_vox
        covered[a:b] += 1
    assert (covered == 1).all()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, result_path: str) -> None:
    import torch
    import torch.distributed as dist

    from mach_b200.distributed import all_gather_image, beamform_shard
    from oracle import oracle_c
    from tests import _helpers as H

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = H.small("compound", n_x=20, n_z=26, n_tx=3)
        ch = H.channel_numpy(w.channel)
        p = {k: w.params[k] for k in H.PARAM_KEYS}

        def cpu_beamform(ch_, rx, scan, arr, grid_shape=None):
            return oracle_c.beamform_c(ch_, rx, scan, arr, storage="c64", n_threads=2, **p)

        out, (a, b) = beamform_shard(cpu_beamform, ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s,
                                     world=world, rank=rank)
        full = all_gather_image(torch.as_tensor(out), w.n_vox, world)
        if rank == 0:
            np.save(result_path, full.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_matches_single_process(tmp_path):
    import torch.multiprocessing as mp

    from tests import _helpers as H

    world = 2
    path = str(tmp_path / "img.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), path), nprocs=world, start_method="spawn", join=True)
    got = np.load(path)
    w = H.small("compound", n_x=20, n_z=26, n_tx=3)
    want = H.oracle(w)
    assert got.shape == want.shape
    assert H.rel_l2(got, want) < 1e-12
