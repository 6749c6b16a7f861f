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
