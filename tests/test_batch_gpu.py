"""Batched persistent launches give the same images as one call per job.

A mixed batch (several storage types, frame counts, grid sizes and kernel families)
runs through ``mach_b200_batch_run``; every job's image must equal, bit for bit, what
``experimental.beamform`` gives for that job alone (same tile function, same summation
order), and both must agree with the FP64 oracle.  A captured CUDA graph replays the
batch and picks up new channel data written into the same buffers.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu


def _jobs_and_workloads():
    import torch

    from mach_b200 import workloads as W
    from mach_b200.batch import Job

    specs = [
        (H.small("compound", n_x=40, n_z=48, n_tx=6), "c64"),
        (H.small("compound", n_x=24, n_z=20, n_tx=3), "c64"),
        (H.small("plain2d", n_x=32, n_z=40), "f32"),
        (H.small("doppler", n_x=16, n_z=24, n_tx=2, n_frames=40), "c64"),
        (H.small("doppler", n_x=12, n_z=16, n_tx=2, n_frames=16), "cf16"),
        (H.small("doppler", n_x=12, n_z=20, n_tx=2, n_frames=32), "cf16"),
        (H.small("volume3d", n_side=8, n_elem_side=8, n_frames=4), "i16"),
        (H.small("volume3d", n_side=6, n_elem_side=8, n_frames=1), "i16"),
    ]
    out = []
    for w, storage in specs:
        ch, scale = W.as_storage(w, storage)
        w.channel, w.channel_scale, w.storage = ch.contiguous(), scale, storage
        dev = "cuda"
        job = Job(
            channel=w.channel.to(dev), rx_coords_m=torch.as_tensor(w.rx_coords_m, device=dev),
            scan_coords_m=torch.as_tensor(w.scan_coords_m, device=dev),
            arrivals=torch.as_tensor(w.tx_wave_arrivals_s, device=dev), channel_scale=w.channel_scale,
            **{k: w.params[k] for k in H.PARAM_KEYS})
        out.append((w, job))
    return out


def test_mixed_batch_matches_single_calls_and_oracle(cuda):
    import torch

    from mach_b200.batch import Batch

    pairs = _jobs_and_workloads()
    batch = Batch([j for _, j in pairs])
    try:
        batch.run()
        torch.cuda.synchronize()
        for w, job in pairs:
            got = job.out.cpu().numpy()
            alone = H.gpu_compound(w)
            assert np.array_equal(got, alone), (w.name, w.storage, H.rel_l2(got, alone))
            want = H.oracle(w)
            assert H.nrms_db(got, want) < -60, (w.name, w.storage)
    finally:
        batch.close()


def test_batch_overwrites_and_reruns_identically(cuda):
    import torch

    from mach_b200.batch import Batch

    pairs = _jobs_and_workloads()[:4]
    batch = Batch([j for _, j in pairs])
    try:
        batch.run()
        first = [j.out.clone() for _, j in pairs]
        for _, j in pairs:
            j.out.fill_(123.0)
        batch.run()
        torch.cuda.synchronize()
        for (_, j), f in zip(pairs, first):
            assert torch.equal(j.out, f)
    finally:
        batch.close()


def test_captured_batch_replays_with_new_channel_data(cuda):
    import torch

    from mach_b200.batch import Batch

    pairs = [p for p in _jobs_and_workloads() if p[0].storage in ("c64", "f32")]
    batch = Batch([j for _, j in pairs])
    try:
        batch.capture()
        batch.replay()
        torch.cuda.synchronize()
        base = [j.out.clone() for _, j in pairs]
        for (w, j), b in zip(pairs, base):
            assert np.array_equal(b.cpu().numpy(), H.gpu_compound(w))
        for _, j in pairs:
            j.channel.mul_(2)  # exact in binary floating point
        batch.replay()
        torch.cuda.synchronize()
        for (_, j), b in zip(pairs, base):
            assert torch.equal(j.out, 2 * b)
    finally:
        batch.close()


def test_batch_accumulate_flag_adds(cuda):
    import torch

    from mach_b200.batch import Batch

    (w, job), = _jobs_and_workloads()[:1]
    job.accumulate = True
    batch = Batch([job])
    try:
        batch.run()
        once = job.out.clone()
        batch.run()
        torch.cuda.synchronize()
        assert torch.allclose(job.out, 2 * once, rtol=1e-6, atol=0)
    finally:
        batch.close()


def test_batch_rejects_host_buffers_and_too_many_jobs(cuda):
    import torch

    from mach_b200.batch import Batch, Job

    (w, job), = _jobs_and_workloads()[:1]
    batch = Batch([job, job], max_jobs=1)
    try:
        with pytest.raises(RuntimeError, match="exceed"):
            batch.run()
    finally:
        batch.close()
    host = Job(channel=job.channel, rx_coords_m=job.rx_coords_m.cpu(), scan_coords_m=job.scan_coords_m,
               arrivals=job.arrivals, **{k: w.params[k] for k in H.PARAM_KEYS})
    batch = Batch([host])
    try:
        with pytest.raises(ValueError, match="contiguous CUDA tensor"):
            batch.run()
    finally:
        batch.close()
    empty = Batch([])
    try:
        empty.run()
    finally:
        empty.close()
    assert torch.cuda.is_available()
