"""Serving scheduler on CPU with a simulated GPU: admission by memory budget and free
slots, continuous batching across two banks, Poisson arrivals, latency bookkeeping."""

from __future__ import annotations

import numpy as np

from mach_b200 import serving


class SimExecutor:
    """One simulated GPU: waves run back to back, each taking the sum of its jobs' times."""

    def __init__(self, service_s):
        self.t = 0.0
        self.gpu_free = 0.0
        self.service_s = service_s
        self.waves = []

    def now(self):
        return self.t

    def launch(self, wave):
        start = max(self.t, self.gpu_free)
        end = start + sum(self.service_s[r.cls] for r in wave.requests)
        self.gpu_free = end
        self.waves.append(wave)
        return end

    def done(self, handle):
        return handle if self.t >= handle else None

    def wait(self, seconds):
        self.t += min(seconds, 1e-4) if seconds else 1e-4


def test_poisson_arrivals_rate_and_mix():
    reqs = serving.poisson_arrivals(2000.0, 20000, [0.5, 0.3, 0.15, 0.05], seed=4)
    t = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(t) >= 0)
    assert abs(np.mean(np.diff(t)) - 1 / 2000.0) < 0.05 / 2000.0
    frac = np.bincount([r.cls for r in reqs], minlength=4) / len(reqs)
    assert np.allclose(frac, [0.5, 0.3, 0.15, 0.05], atol=0.02)
    again = serving.poisson_arrivals(2000.0, 20000, [0.5, 0.3, 0.15, 0.05], seed=4)
    assert [r.arrival_s for r in again] == [r.arrival_s for r in reqs]


def test_every_request_completes_after_it_arrives():
    ex = SimExecutor([1e-4, 1e-3, 8e-4, 2e-3])
    reqs = serving.poisson_arrivals(500.0, 300, [0.5, 0.3, 0.15, 0.05], seed=1)
    sch = serving.Scheduler(ex, [4, 4, 4, 4], [1, 1, 1, 1], budget=1 << 30)
    sch.serve(reqs)
    assert all(r.done_s is not None and r.done_s >= r.arrival_s for r in reqs)
    # every wave ran on one bank with distinct slots of each class
    for w in ex.waves:
        keys = [(r.cls, r.slot) for r in w.requests]
        assert len(keys) == len(set(keys))
    lat = serving.latency_summary(reqs)
    assert lat["p50"] <= lat["p99"] <= lat["max"]


def test_memory_budget_limits_what_is_in_flight():
    ex = SimExecutor([1e-3] * 2)
    reqs = serving.poisson_arrivals(5000.0, 100, [0.5, 0.5], seed=2)
    sch = serving.Scheduler(ex, [8, 8], [300, 500], budget=1000)
    sch.serve(reqs)
    assert sch.peak_in_flight_bytes <= 1000
    assert all(r.done_s is not None for r in reqs)
    for w in ex.waves:
        assert sum(300 if r.cls == 0 else 500 for r in w.requests) <= 1000


def test_requests_arriving_during_a_wave_join_the_next_one():
    ex = SimExecutor([5e-3])
    reqs = [serving.Request(i, 1e-4 * i, 0) for i in range(10)]
    sch = serving.Scheduler(ex, [16], [1], budget=100, banks=1)
    sch.serve(reqs)
    assert [r.rid for r in ex.waves[0].requests] == [0]
    assert len(ex.waves) == 2 and len(ex.waves[1].requests) == 9  # all batched while wave 0 ran


def test_two_banks_keep_a_second_wave_queued_on_the_gpu():
    ex = SimExecutor([5e-3])
    reqs = [serving.Request(i, 1e-4 * i, 0) for i in range(10)]
    sch = serving.Scheduler(ex, [16], [1], budget=100, banks=2)
    sch.serve(reqs)
    assert ex.waves[0].bank != ex.waves[1].bank
    assert sum(len(w.requests) for w in ex.waves) == 10
    assert len(ex.waves) < 10  # later arrivals were batched


def test_serial_reference_queue():
    reqs = [serving.Request(0, 0.0, 0), serving.Request(1, 0.001, 0), serving.Request(2, 0.010, 0)]
    out = serving.serial_reference_latencies(reqs, lambda r: 0.004)
    assert [r.done_s for r in out] == [0.004, 0.008, 0.014]
