"""Serving loop: continuous batching of beamforming requests of mixed sizes on one GPU.

Requests arrive over time (seeded Poisson arrivals) and belong to request classes: a
beamforming configuration whose geometry (element positions, scan grid, transmit arrival
times) stays resident on the device.  The engine keeps two banks of slots per class; a
*wave* is a set of admitted requests that runs as one :class:`mach_b200.batch.Batch` (one
persistent launch per kernel signature) on its bank's stream.  While one wave runs, requests
that arrived meanwhile are admitted into the next wave on the other bank, so the two waves
overlap on the GPU.  A request is admitted when its class has a free slot in that bank and
the device bytes in flight stay within the HBM budget (a fraction of the free device memory
measured at start-up).  Waves with the same slot set are recorded once as a CUDA graph and
replayed afterwards.

Two modes:
* resident (``upload=False``): every request of a class beamforms the class's acquisition,
  already on the device; a request holds its output slot (output bytes in flight);
* upload (``upload=True``): every request carries its own acquisition in pinned host memory.
  Its channel data is copied into the slot's device input buffer on the bank's copy stream
  (overlapping the other bank's running wave), beamformed, and its image copied back to a
  pinned host buffer; a request holds input and output bytes while in flight.

Latency of a request = device completion time of its wave (CUDA event, measured from a
start event recorded when serving begins; in upload mode after the image is back in host
memory) minus its arrival time.

mach has no serving layer; its closest equivalent is one synchronous call per transmit of
each job, in arrival order (``serial_reference_latencies`` gives the queue of that baseline
from measured service times).

The scheduling logic (:class:`Scheduler`) is independent of the GPU: an executor object
launches waves and reports completions, so the host logic is tested on CPU with a
simulated executor.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np


# ----------------------------------------------------------------------------- requests


@dataclass
class Request:
    rid: int
    arrival_s: float
    cls: int
    done_s: float | None = None  # completion time on the serving clock
    wave: int = -1
    slot: int = -1
    acq: int = 0  # upload mode: which of the class's acquisitions the request carries


def poisson_arrivals(rate_hz: float, n: int, weights: list[float], seed: int) -> list[Request]:
    """``n`` requests with exponential inter-arrival gaps (mean 1/rate) and classes drawn by weight."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=n)
    times = np.cumsum(gaps) - gaps[0]
    p = np.asarray(weights, dtype=np.float64)
    cls = rng.choice(len(p), size=n, p=p / p.sum())
    return [Request(i, float(t), int(c)) for i, (t, c) in enumerate(zip(times, cls))]


def latency_summary(requests: list[Request]) -> dict:
    lat = np.array([(r.done_s - r.arrival_s) * 1e3 for r in requests if r.done_s is not None])
    if lat.size == 0:
        return {"p50": None, "p99": None, "mean": None, "max": None}
    return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "mean": float(lat.mean()), "max": float(lat.max())}


def serial_reference_latencies(requests: list[Request], service_s: Callable[[Request], float]) -> list[Request]:
    """Single-server FIFO: each request starts when it has arrived and the previous one is done."""
    free_at = 0.0
    out = []
    for r in sorted(requests, key=lambda q: q.arrival_s):
        start = max(free_at, r.arrival_s)
        free_at = start + service_s(r)
        out.append(Request(r.rid, r.arrival_s, r.cls, done_s=free_at))
    return out


# ----------------------------------------------------------------------------- scheduler


@dataclass
class Wave:
    wid: int
    bank: int
    requests: list[Request]
    handle: Any = None


class Scheduler:
    """Admission and continuous batching.

    ``slots[c]``: output slots of class ``c`` per bank; ``bytes_of[c]``: device bytes a
    request of class ``c`` holds while in flight; ``budget``: bytes that may be in flight.
    ``executor`` provides ``now()``, ``launch(wave) -> handle``, ``done(handle) -> float | None``
    (completion time on the serving clock, or None while running) and ``wait(seconds)``.
    """

    def __init__(self, executor, slots: list[int], bytes_of: list[int], budget: int, *, banks: int = 2,
                 max_wave_jobs: int = 32, on_done: Callable[[Request, Wave], None] | None = None):
        self.ex = executor
        self.slots = list(slots)
        self.bytes_of = list(bytes_of)
        self.budget = int(budget)
        self.banks = banks
        self.max_wave_jobs = max_wave_jobs
        self.on_done = on_done
        self.free = [[list(range(n)) for n in self.slots] for _ in range(banks)]
        self.bank_busy = [False] * banks
        self.in_flight_bytes = 0
        self.waves: list[Wave] = []
        self.peak_in_flight_bytes = 0

    def _admit(self, queue: deque, bank: int) -> list[Request]:
        wave: list[Request] = []
        kept: deque = deque()
        while queue and len(wave) < self.max_wave_jobs:
            r = queue.popleft()
            fits = self.in_flight_bytes + self.bytes_of[r.cls] <= self.budget
            if fits and self.free[bank][r.cls]:
                r.slot = self.free[bank][r.cls].pop(0)
                self.in_flight_bytes += self.bytes_of[r.cls]
                wave.append(r)
            else:
                kept.append(r)
        kept.extend(queue)
        queue.clear()
        queue.extend(kept)
        self.peak_in_flight_bytes = max(self.peak_in_flight_bytes, self.in_flight_bytes)
        return wave

    def _retire(self, w: Wave, t_done: float) -> None:
        for r in w.requests:
            r.done_s = t_done
            if self.on_done is not None:
                self.on_done(r, w)
            self.free[w.bank][r.cls].append(r.slot)
            self.free[w.bank][r.cls].sort()
            self.in_flight_bytes -= self.bytes_of[r.cls]
        self.bank_busy[w.bank] = False

    def serve(self, requests: list[Request]) -> list[Request]:
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        queue: deque = deque()
        running: list[Wave] = []
        n_done = 0
        total = len(pending)
        while n_done < total:
            now = self.ex.now()
            while pending and pending[0].arrival_s <= now:
                queue.append(pending.popleft())
            for w in list(running):
                t = self.ex.done(w.handle)
                if t is not None:
                    running.remove(w)
                    self._retire(w, t)
                    n_done += len(w.requests)
            launched = False
            if queue:
                for bank in range(self.banks):
                    if self.bank_busy[bank]:
                        continue
                    reqs = self._admit(queue, bank)
                    if reqs:
                        w = Wave(len(self.waves), bank, reqs)
                        for r in reqs:
                            r.wave = w.wid
                        self.bank_busy[bank] = True
                        w.handle = self.ex.launch(w)
                        self.waves.append(w)
                        running.append(w)
                        launched = True
                    break
            if not launched:
                nxt = pending[0].arrival_s - now if pending else None
                self.ex.wait(nxt)
        return requests


# ----------------------------------------------------------------------------- GPU engine


@dataclass
class RequestClass:
    """A beamforming configuration served from resident device memory.

    ``workload`` is a :class:`mach_b200.workloads.Workload` whose channel data is on the
    device; ``storage`` the channel storage the requests use.
    """

    name: str
    weight: float
    workload: Any
    storage: str
    tensors: dict = field(default_factory=dict)
    acquisitions: list = field(default_factory=list)  # upload mode: pinned host channel data

    @property
    def points(self) -> int:
        return self.workload.points


class GpuExecutor:
    """Runs waves as persistent batch launches on one stream per bank; replays CUDA graphs
    for slot sets seen before (``use_graphs``)."""

    def __init__(self, classes: list[RequestClass], slots: list[int], banks: int = 2, use_graphs: bool = True,
                 upload: bool = False, n_acquisitions: int = 2):
        import torch

        from mach_b200 import workloads as W
        from mach_b200.batch import Job

        self.torch = torch
        self.classes = classes
        self.use_graphs = use_graphs
        self.upload = upload
        self.streams = [torch.cuda.Stream() for _ in range(banks)]
        self.copy_streams = [torch.cuda.Stream() for _ in range(banks)] if upload else []
        self.jobs: list[list[list[Any]]] = []  # [bank][class][slot]
        self.host_out: list[list[list[Any]]] = []  # upload mode: [bank][class][slot] pinned images
        for c in classes:
            w = c.workload
            ch, scale = W.as_storage(w, c.storage)
            c.tensors = {
                "channel": ch.contiguous().to("cuda"),
                "rx": torch.as_tensor(w.rx_coords_m, device="cuda").contiguous(),
                "scan": torch.as_tensor(w.scan_coords_m, device="cuda").contiguous(),
                "arr": torch.as_tensor(w.tx_wave_arrivals_s, device="cuda").contiguous(),
                "scale": scale,
            }
            if upload:
                c.acquisitions = make_acquisitions(c.tensors["channel"], n_acquisitions)
        params = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
                  "interp_type")
        knobs = [class_tuning(c) for c in classes]
        for _ in range(banks):
            per_class, per_class_out = [], []
            for c, n, tuned in zip(classes, slots, knobs):
                t = c.tensors
                jobs = []
                for _ in range(n):
                    channel = torch.empty_like(t["channel"]) if upload else t["channel"]
                    jobs.append(Job(channel=channel, rx_coords_m=t["rx"], scan_coords_m=t["scan"], arrivals=t["arr"],
                                    channel_scale=t["scale"], tuning=dict(tuned),
                                    **{k: c.workload.params[k] for k in params}))
                per_class.append(jobs)
                if upload:
                    per_class_out.append([torch.empty(j.out.shape, dtype=j.out.dtype, pin_memory=True) for j in jobs])
            self.jobs.append(per_class)
            self.host_out.append(per_class_out)
        self.graphs: dict[tuple, Any] = {}
        self.graph_hits = 0
        self.graph_misses = 0
        self.replayed_kernels = 0  # kernels launched by graph replays (the library counts direct launches)
        self.captured_kernels = 0  # launches the library counted while recording graphs (never run)
        self.t0_event = None
        self.t0 = 0.0

    def start(self) -> None:
        torch = self.torch
        torch.cuda.synchronize()
        self.t0_event = torch.cuda.Event(enable_timing=True)
        self.t0_event.record(torch.cuda.current_stream())
        self.t0_event.synchronize()
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def out_of(self, r: Request, bank: int):
        """The request's image: the pinned host copy in upload mode, else the device slot."""
        if self.upload:
            return self.host_out[bank][r.cls][r.slot]
        return self.jobs[bank][r.cls][r.slot].out

    def bytes_per_request(self, cls: int) -> tuple[int, int]:
        """(host-to-device, device-to-host) bytes one request of class ``cls`` moves in upload mode."""
        job = self.jobs[0][cls][0]
        if not self.upload:
            return 0, 0
        ch = job.channel
        return ch.numel() * ch.element_size(), job.out.numel() * job.out.element_size()

    def launch(self, wave: Wave):
        from mach_b200.batch import Batch

        torch = self.torch
        stream = self.streams[wave.bank]
        order = sorted(wave.requests, key=lambda r: (r.cls, r.slot))
        key = (wave.bank, tuple((r.cls, r.slot) for r in order))
        jobs = [self.jobs[wave.bank][r.cls][r.slot] for r in order]
        if self.upload:  # each request's acquisition into its slot, on this bank's copy stream
            copy = self.copy_streams[wave.bank]
            with torch.cuda.stream(copy):
                for r, j in zip(order, jobs):
                    acq = self.classes[r.cls].acquisitions
                    j.channel.copy_(acq[r.acq % len(acq)], non_blocking=True)
                uploaded = torch.cuda.Event()
                uploaded.record(copy)
            stream.wait_event(uploaded)
        with torch.cuda.stream(stream):
            entry = self.graphs.get(key) if self.use_graphs else None
            if entry is not None:
                self.graph_hits += 1
                entry.replay()
                self.replayed_kernels += entry.kernels
            else:
                from mach_b200 import _cuda_impl

                self.graph_misses += 1
                batch = Batch(jobs)
                before = _cuda_impl.launch_count()
                batch.run(sync=False, stream=stream)
                batch.kernels = _cuda_impl.launch_count() - before
                if self.use_graphs:
                    batch.capture(warmup=False)
                    self.captured_kernels += batch.kernels
                    self.graphs[key] = batch
            if self.upload:  # images back to pinned host memory
                for r, j in zip(order, jobs):
                    self.host_out[wave.bank][r.cls][r.slot].copy_(j.out, non_blocking=True)
            done = torch.cuda.Event(enable_timing=True)
            done.record(stream)
        return done

    def done(self, handle) -> float | None:
        if not handle.query():
            return None
        return self.t0_event.elapsed_time(handle) / 1e3

    def wait(self, seconds: float | None) -> None:
        if seconds is None or seconds > 2e-4:
            time.sleep(5e-5)


class ServingEngine:
    """Request classes + scheduler + GPU executor (resident or upload mode)."""

    def __init__(self, classes: list[RequestClass], *, slots_per_class: int = 8, hbm_fraction: float = 0.5,
                 max_wave_jobs: int = 32, use_graphs: bool = True, on_done=None, upload: bool = False,
                 n_acquisitions: int = 2):
        import torch

        self.classes = classes
        self.executor = GpuExecutor(classes, [slots_per_class] * len(classes), use_graphs=use_graphs, upload=upload,
                                    n_acquisitions=n_acquisitions)
        # device bytes a request holds in flight: its output, plus its input buffer in upload mode
        self.bytes_of = []
        for c in classes:
            w = c.workload
            cplx = c.storage in ("c64", "cf16", "cbf16", "ci16")
            held = w.n_vox * w.n_frames * (8 if cplx else 4)
            if upload:
                ch = c.tensors["channel"]
                held += ch.numel() * ch.element_size()
            self.bytes_of.append(held)
        free, _total = torch.cuda.mem_get_info()
        self.budget = int(hbm_fraction * free)
        self.scheduler = Scheduler(self.executor, [slots_per_class] * len(classes), self.bytes_of, self.budget,
                                   max_wave_jobs=max_wave_jobs, on_done=on_done)

    def serve(self, requests: list[Request]) -> list[Request]:
        for r in requests:  # upload mode: the request's acquisition (the same stream gives the same data)
            n = max(1, len(self.classes[r.cls].acquisitions))
            r.acq = r.rid % n
        self.executor.start()
        self.scheduler.serve(requests)
        self.torch_sync()
        return requests

    @staticmethod
    def torch_sync():
        import torch

        torch.cuda.synchronize()


def class_tuning(c: RequestClass) -> dict:
    """Autotuner knobs cached for the class's job shape (empty when it has not been timed)."""
    import torch

    from mach_b200 import _grid, tuning

    ch = c.tensors["channel"]
    n_tx, n_rx, n_s, n_f = (int(d) for d in ch.shape[:4])
    hit = tuning.lookup(c.storage, n_tx, n_rx, n_s, n_f, c.workload.n_vox, _grid.detect(c.tensors["scan"]),
                        int(c.workload.params["interp_type"]), torch.cuda.current_device(), "auto")
    return hit or {}


def make_acquisitions(channel, n: int) -> list:
    """``n`` distinct acquisitions in pinned host memory with the statistics of ``channel``
    ([n_tx, n_rx, n_samples, n_frames(, 2)]): the data itself, then copies delayed by 17 k
    samples (rolled along the sample axis)."""
    import torch

    out = []
    for k in range(n):
        x = channel if k == 0 else torch.roll(channel, shifts=17 * k, dims=2)
        host = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
        host.copy_(x)
        out.append(host)
    return out


def c4_classes(device: str = "cuda", small: bool = False) -> list[RequestClass]:
    """The serving mix: 50% plain 2-D (256^2, 128 el, 1 frame), 30% 75-transmit compounding on
    384^2, 15% 32-frame Doppler, 5% 3-D 1024-channel 96^3; FP16 storage (real RF as float16,
    IQ as complex float16).  ``small`` gives reduced sizes of the same physics for tests."""
    from mach_b200 import workloads as W

    if small:
        return [
            RequestClass("plain2d", 0.5, W.plain2d(n_x=32, n_z=40, n_elements=32, n_samples=600, device=device), "f16"),
            RequestClass("compound", 0.3, W.compound(n_x=24, n_z=32, n_tx=6, n_elements=32, n_samples=1500,
                                                     n_speckle=300, device=device), "cf16"),
            RequestClass("doppler", 0.15, W.doppler(n_x=16, n_z=24, n_tx=2, n_frames=32, n_elements=32,
                                                    n_samples=1024, n_scatterers=200, device=device), "cf16"),
            RequestClass("volume3d", 0.05, W.volume3d(n_side=8, n_elem_side=8, n_frames=1, n_samples=1400,
                                                      n_scatterers=20, device=device), "f16"),
        ]
    return [
        RequestClass("plain2d", 0.5, W.plain2d(device=device), "f16"),
        RequestClass("compound", 0.3, W.compound(n_x=384, n_z=384, device=device), "cf16"),
        RequestClass("doppler", 0.15, W.doppler(n_frames=32, device=device), "cf16"),
        RequestClass("volume3d", 0.05, W.volume3d(n_side=96, n_frames=1, device=device), "f16"),
    ]
