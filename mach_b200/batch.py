"""Batched beamforming: many jobs in one persistent launch per kernel signature.

A :class:`Batch` holds device-resident jobs (channel data, geometry, outputs) of any mix
of grid sizes, transmit counts, frame counts and storage types.  :meth:`Batch.run`
hands them to ``mach_b200_batch_run``: jobs are grouped by kernel signature and each
group runs as one persistent launch whose CTAs pull (job, tile) work items from a device
counter.  :meth:`Batch.capture` records the whole batch -- job-table copy, counter
reset, persistent launches -- in a CUDA graph; :meth:`Batch.replay` re-runs it with a
single graph launch (the buffers stay the same; new channel data written into them is
picked up).  mach has no batching; its closest equivalent is one call per transmit and
per job.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Any

from mach_b200 import _cuda_impl, _dlpack, _grid

_lib = _cuda_impl._lib


class _Job(ctypes.Structure):
    """``mach_b200_job`` (include/mach_b200.h)."""

    _fields_ = [
        ("storage", ctypes.c_int32),
        ("interp_type", ctypes.c_int32),
        ("channel_data", ctypes.c_void_p),
        ("rx_coords_m", ctypes.c_void_p),
        ("scan_coords_m", ctypes.c_void_p),
        ("tx_wave_arrivals_s", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n_tx", ctypes.c_uint32),
        ("n_rx", ctypes.c_uint32),
        ("n_samples", ctypes.c_uint32),
        ("n_frames", ctypes.c_uint32),
        ("n_scan", ctypes.c_uint64),
        ("f_number", ctypes.c_float),
        ("rx_start_s", ctypes.c_float),
        ("sampling_freq_hz", ctypes.c_float),
        ("sound_speed_m_s", ctypes.c_float),
        ("modulation_freq_hz", ctypes.c_float),
        ("tukey_alpha", ctypes.c_float),
        ("channel_scale", ctypes.c_float),
        ("flags", ctypes.c_uint32),
        ("grid_shape", ctypes.c_int32 * 3),
        ("kernel", ctypes.c_int32),
        ("tx_chunk", ctypes.c_int32),
        ("window_rows", ctypes.c_int32),
        ("lanes_per_voxel", ctypes.c_int32),
    ]


_lib.mach_b200_batch_create.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]
_lib.mach_b200_batch_create.restype = ctypes.c_int
_lib.mach_b200_batch_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Job), ctypes.c_uint32, ctypes.c_void_p,
                                     ctypes.c_uint32]
_lib.mach_b200_batch_run.restype = ctypes.c_int
_lib.mach_b200_batch_destroy.argtypes = [ctypes.c_void_p]
_lib.mach_b200_batch_destroy.restype = None


@dataclass
class Job:
    """One beamforming job with device-resident torch tensors.

    ``channel`` is ``[n_tx, n_rx, n_samples, n_frames]`` (or ``[..., 2]`` (I, Q) pairs of a
    16-bit type), ``arrivals`` ``[n_tx, n_scan]``; ``out`` is allocated when omitted and is
    overwritten (``accumulate=True`` adds into it instead).
    """

    channel: Any
    rx_coords_m: Any
    scan_coords_m: Any
    arrivals: Any
    f_number: float
    rx_start_s: float
    sampling_freq_hz: float
    sound_speed_m_s: float
    modulation_freq_hz: float = 0.0
    tukey_alpha: float = 0.5
    interp_type: int = 1
    channel_scale: float = 1.0
    out: Any = None
    accumulate: bool = False
    delay: str = "auto"
    grid_shape: Any = None
    tuning: dict = field(default_factory=dict)

    def __post_init__(self):
        import torch

        pairs = self.channel.dim() == 5
        self._view = _dlpack.view(self.channel)
        self.storage = _cuda_impl.storage_of(self._view, pairs)
        cplx = bool(_cuda_impl.STORAGE_CODES[self.storage] & 1)
        n_frames = int(self.channel.shape[3])
        if self.out is None:
            self.out = torch.zeros((int(self.scan_coords_m.shape[0]), n_frames),
                                   dtype=torch.complex64 if cplx else torch.float32, device=self.channel.device)
        if self.grid_shape is None:
            self.grid_shape = _grid.detect(self.scan_coords_m)

    @property
    def points(self) -> int:
        n_tx, n_rx, _, n_f = (int(d) for d in self.channel.shape[:4])
        return int(self.scan_coords_m.shape[0]) * n_rx * n_tx * n_f

    def as_struct(self) -> _Job:
        for name in ("channel", "rx_coords_m", "scan_coords_m", "arrivals", "out"):
            t = getattr(self, name)
            if not (t.is_cuda and t.is_contiguous()):
                raise ValueError(f"Job.{name} must be a contiguous CUDA tensor")
        n_tx, n_rx, n_s, n_f = (int(d) for d in self.channel.shape[:4])
        j = _Job()
        j.storage = _cuda_impl.STORAGE_CODES[self.storage]
        j.interp_type = int(self.interp_type)
        j.channel_data = self.channel.data_ptr()
        j.rx_coords_m = self.rx_coords_m.data_ptr()
        j.scan_coords_m = self.scan_coords_m.data_ptr()
        j.tx_wave_arrivals_s = self.arrivals.data_ptr()
        j.out = self.out.data_ptr()
        j.n_tx, j.n_rx, j.n_samples, j.n_frames = n_tx, n_rx, n_s, n_f
        j.n_scan = int(self.scan_coords_m.shape[0])
        j.f_number, j.rx_start_s = float(self.f_number), float(self.rx_start_s)
        j.sampling_freq_hz, j.sound_speed_m_s = float(self.sampling_freq_hz), float(self.sound_speed_m_s)
        j.modulation_freq_hz, j.tukey_alpha = float(self.modulation_freq_hz), float(self.tukey_alpha)
        j.channel_scale = float(self.channel_scale)
        delay = self.delay
        if delay == "auto":
            delay = "reference" if self.storage in ("f32", "c64") else "split"
        j.flags = (0 if self.accumulate else _cuda_impl.FLAG_OVERWRITE) | (
            _cuda_impl.FLAG_SPLIT_DELAY if delay == "split" else 0)
        t = self.tuning or {}
        grid = t.get("grid_shape")
        grid = self.grid_shape if grid is None else grid
        if grid:
            for i, v in enumerate(grid):
                j.grid_shape[i] = int(v)
        kernel = t.get("kernel", 0)
        j.kernel = _cuda_impl.KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        j.tx_chunk = int(t.get("tx_chunk", 0))
        j.window_rows = int(t.get("window_rows", 0))
        j.lanes_per_voxel = int(t.get("lanes_per_voxel", 0))
        return j


class Batch:
    """A set of device-resident jobs run by persistent launches (optionally as a CUDA graph)."""

    def __init__(self, jobs: list[Job], max_jobs: int | None = None):
        self.jobs = list(jobs)
        self.max_jobs = max(1, max_jobs or len(self.jobs))
        handle = ctypes.c_void_p()
        _cuda_impl._raise_for(_lib.mach_b200_batch_create(self.max_jobs, ctypes.byref(handle)))
        self._handle = handle
        self._graph = None
        self._table = None

    def _structs(self):
        arr = (_Job * max(1, len(self.jobs)))()
        for i, j in enumerate(self.jobs):
            arr[i] = j.as_struct()
        self._table = arr  # keep alive while the stream may read it
        return arr

    @property
    def points(self) -> int:
        return sum(j.points for j in self.jobs)

    def run(self, sync: bool = True, stream: Any = None) -> None:
        import torch

        if stream is None:
            stream = torch.cuda.current_stream()
        flags = 0 if sync else _cuda_impl.FLAG_ASYNC
        arr = self._structs()
        _cuda_impl._raise_for(_lib.mach_b200_batch_run(self._handle, arr, len(self.jobs), stream.cuda_stream, flags))

    def capture(self, warmup: bool = True) -> None:
        """Record the batch once in a CUDA graph (jobs and buffers fixed from now on).

        ``warmup`` first runs the batch synchronously, so lazy module loading happens
        outside the capture; a batch that has already run once can skip it.  Capturing
        only records: nothing runs until :meth:`replay`.
        """
        import torch

        if warmup:
            self.run(sync=True)
        side = torch.cuda.Stream()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            graph.capture_begin(capture_error_mode="relaxed")
            try:
                self.run(sync=False, stream=side)
            finally:
                graph.capture_end()
        self._graph = graph

    def replay(self) -> None:
        if self._graph is None:
            raise RuntimeError("Batch.capture() first")
        self._graph.replay()

    def close(self) -> None:
        if self._handle:
            self._graph = None
            _lib.mach_b200_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
