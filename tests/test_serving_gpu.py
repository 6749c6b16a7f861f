"""Serving on the GPU: a mixed stream of requests (reduced sizes of the serving mix) runs
through continuous batching, two banks and graph replays; every request's image is the
same, bit for bit, as that job beamformed alone, and agrees with the FP64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu


def test_results_are_the_same_alone_and_in_the_mix(cuda):
    import torch

    from mach_b200 import serving
    from mach_b200.batch import Batch, Job
    from oracle import oracle_c

    classes = serving.c4_classes(small=True)
    results = {}

    def keep(r, wave):
        results[(pass_no[0], r.rid)] = engine.executor.out_of(r, wave.bank).clone()

    pass_no = [0]
    engine = serving.ServingEngine(classes, slots_per_class=4, on_done=keep)
    weights = [c.weight for c in classes]
    reqs = serving.poisson_arrivals(20000.0, 48, weights, seed=4)
    engine.serve(reqs)
    pass_no[0] = 1
    reqs2 = serving.poisson_arrivals(20000.0, 48, weights, seed=4)
    engine.serve(reqs2)  # same stream again: slot sets repeat, so graphs are replayed
    assert all(r.done_s is not None and r.done_s >= r.arrival_s for r in reqs + reqs2)
    assert max(len(w.requests) for w in engine.scheduler.waves) > 1  # requests were batched together
    assert engine.executor.graph_hits > 0

    params = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
              "interp_type")
    alone = {}
    for ci, c in enumerate(classes):
        t = c.tensors
        job = Job(channel=t["channel"], rx_coords_m=t["rx"], scan_coords_m=t["scan"], arrivals=t["arr"],
                  channel_scale=t["scale"], **{k: c.workload.params[k] for k in params})
        b = Batch([job])
        b.run(sync=True)
        alone[ci] = job.out.clone()
        b.close()
        w = c.workload
        want = oracle_c.beamform_c(H.channel_numpy(t["channel"].cpu()), w.rx_coords_m, w.scan_coords_m,
                                   w.tx_wave_arrivals_s, storage=c.storage, channel_scale=t["scale"],
                                   **{k: w.params[k] for k in H.PARAM_KEYS})
        assert H.nrms_db(alone[ci].cpu().numpy(), want) <= -60.0, c.name
    for (p, rid), out in results.items():
        r = (reqs if p == 0 else reqs2)[rid]
        assert torch.equal(out, alone[r.cls]), (p, rid, classes[r.cls].name)
    lat = serving.latency_summary(reqs)
    assert lat["p50"] > 0


def test_uploaded_requests_match_their_acquisition_alone(cuda):
    """Upload mode: every request carries its own acquisition from pinned host memory (two per
    class here), uploaded on a copy stream while the other bank's wave runs; its image comes
    back to pinned host memory and equals, bit for bit, that acquisition beamformed alone."""
    import torch

    from mach_b200 import serving
    from mach_b200.batch import Batch, Job

    classes = serving.c4_classes(small=True)
    results = {}

    def keep(r, wave):
        results[r.rid] = (r.cls, r.acq, engine.executor.out_of(r, wave.bank).clone())

    engine = serving.ServingEngine(classes, slots_per_class=4, on_done=keep, upload=True, n_acquisitions=2)
    reqs = serving.poisson_arrivals(20000.0, 48, [c.weight for c in classes], seed=5)
    engine.serve(reqs)
    engine.serve(serving.poisson_arrivals(20000.0, 48, [c.weight for c in classes], seed=5))  # graph replays
    assert engine.executor.graph_hits > 0
    assert len(results) == 48 and all(not out.is_cuda for _, _, out in results.values())
    assert {acq for _, acq, _ in results.values()} == {0, 1}
    # admission counts the input buffer as well as the image
    assert all(b > c.workload.n_vox * c.workload.n_frames * 4 for b, c in zip(engine.bytes_of, classes))
    params = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
              "interp_type")
    alone = {}
    for ci, c in enumerate(classes):
        t = c.tensors
        for k, acq in enumerate(c.acquisitions):
            job = Job(channel=acq.to("cuda"), rx_coords_m=t["rx"], scan_coords_m=t["scan"], arrivals=t["arr"],
                      channel_scale=t["scale"], **{p: c.workload.params[p] for p in params})
            b = Batch([job])
            b.run(sync=True)
            alone[(ci, k)] = job.out.cpu()
            b.close()
        assert not torch.equal(alone[(ci, 0)], alone[(ci, 1)])  # the acquisitions differ
    for rid, (cls, acq, out) in results.items():
        assert torch.equal(out, alone[(cls, acq)]), (rid, classes[cls].name, acq)
