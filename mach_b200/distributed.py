"""Multi-GPU beamforming by voxel sharding (one process per GPU).

Voxels are independent: every output voxel is a sum over its own elements, transmits
and frames.  A job therefore shards across ranks by voxel ranges with no exchange in
the data path -- each rank holds the full channel data for its job and computes a
contiguous slice of the scan (aligned to the kernels' 128-voxel tiles).  The only
optional collective is the final assembly of the image on every rank
(``torch.distributed.all_gather`` over NCCL, or gloo on CPU), used when a caller wants
the whole image in one place.  mach itself has no multi-GPU support; this is the
B200-native extension of its single-GPU call.
"""

from __future__ import annotations

from typing import Any, Callable

TILE = 128


def shard_range(n_vox: int, world: int, rank: int, align: int = TILE) -> tuple[int, int]:
    """Voxel range [start, stop) of ``rank``: near-equal, ``align``-aligned slices covering [0, n_vox)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    units = -(-n_vox // align)
    lo = units * rank // world
    hi = units * (rank + 1) // world
    return min(lo * align, n_vox), min(hi * align, n_vox)


def beamform_shard(beamform: Callable[..., Any], channel_data: Any, rx_coords_m: Any, scan_coords_m: Any,
                   tx_wave_arrivals_s: Any, *, world: int, rank: int, **kwargs) -> tuple[Any, tuple[int, int]]:
    """Run ``beamform`` (e.g. :func:`mach_b200.experimental.beamform`) on this rank's voxel slice.

    ``tx_wave_arrivals_s`` is ``[n_tx, n_vox]``; the slice is taken along the voxel axis.
    Returns ``(out_slice, (start, stop))``.
    """
    n_vox = int(scan_coords_m.shape[0])
    start, stop = shard_range(n_vox, world, rank)
    kwargs.setdefault("grid_shape", False)  # a slice of a grid is not a grid
    out = beamform(channel_data, rx_coords_m, scan_coords_m[start:stop],
                   tx_wave_arrivals_s[:, start:stop], **kwargs)
    return out, (start, stop)


def all_gather_image(out_slice: Any, n_vox: int, world: int, group=None) -> Any:
    """Assemble the full ``[n_vox, n_frames]`` image on every rank from per-rank slices.

    Slices are padded to a common length for the collective and trimmed afterwards.
    """
    import torch
    import torch.distributed as dist

    t = out_slice if isinstance(out_slice, torch.Tensor) else torch.as_tensor(out_slice)
    per = max(shard_range(n_vox, world, r)[1] - shard_range(n_vox, world, r)[0] for r in range(world))
    padded = torch.zeros((per,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    padded[: t.shape[0]] = t
    if padded.is_complex():
        parts = [torch.zeros_like(torch.view_as_real(padded)) for _ in range(world)]
        dist.all_gather(parts, torch.view_as_real(padded).contiguous(), group=group)
        parts = [torch.view_as_complex(p) for p in parts]
    else:
        parts = [torch.zeros_like(padded) for _ in range(world)]
        dist.all_gather(parts, padded, group=group)
    pieces = []
    for r in range(world):
        a, b = shard_range(n_vox, world, r)
        pieces.append(parts[r][: b - a])
    return torch.cat(pieces, dim=0)
