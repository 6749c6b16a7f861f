"""Launch autotuner: time the kernel variants for one job shape and keep the fastest.

The candidates are the launch knobs of ``mach_b200_options`` (include/mach_b200.h):
kernel family, transmits staged per pass (voxel-per-lane), lanes per voxel and window
rows (staged windows), frame columns per warp (frame-lane), and whether to tile by the voxel
grid.  None of them changes the
result beyond summation order; every candidate is timed with CUDA events on the current
stream over a few repetitions on the caller's own device-resident data, and the winner
is cached per job shape and device in a JSON file (``MACH_B200_TUNING_CACHE``, default
``~/.cache/mach_b200/tuning.json``).  Automatic calls of :func:`mach_b200.experimental.beamform`
and the serving engine's batch jobs look the cache up (:func:`lookup`) and run the tuned
knobs when an entry exists.  mach itself has a fixed launch shape.
"""

from __future__ import annotations

import json
import os
import threading
from typing import Any

from mach_b200 import _grid

_LOCK = threading.Lock()
_MEMO: dict[str, dict] = {}

_STORAGE_BYTES = {"f32": 4, "c64": 8, "f16": 2, "cf16": 4, "bf16": 2, "cbf16": 4, "i16": 2, "ci16": 4}


def cache_path() -> str:
    return os.environ.get("MACH_B200_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mach_b200", "tuning.json"))


def candidates(storage: str, n_frames: int, grid: Any) -> list[dict]:
    """Launch settings worth timing for this storage type and frame count."""
    esz = _STORAGE_BYTES[storage]
    vf = 8 // esz
    out: list[dict] = []
    grids = [None, False] if grid else [False]
    if n_frames > 16 and n_frames % 8 == 0:  # the voxel-per-lane kernel in 8-frame chunks
        for tile_fast in ((2, 4) if grid else (0,)):
            out.append({"kernel": "lane_voxel", "tile_fast": tile_fast})
    if n_frames <= 8 or n_frames == 16:
        for tx_chunk in (8, 16, 32, 40):
            for tile_fast in ((2, 4, 8) if grid else (0,)):
                for lanes in ((1, 2, 4) if n_frames == 1 else (0,)):
                    out.append({"kernel": "lane_voxel", "tx_chunk": tx_chunk, "tile_fast": tile_fast,
                                "lanes_per_voxel": lanes})
    if n_frames == 16:  # elements per launch (L2-resident channel data per launch)
        for block in (-1, 64, 128, 256):
            out.append({"kernel": "lane_voxel", "element_block": block})
    if n_frames % vf == 0 and n_frames > 1:
        lv_max = 32 if storage in ("f32", "c64") else 16
        needed = -(-n_frames // vf)
        for lv in (4, 8, 16, 32):
            if lv > lv_max or (lv > 4 and lv // 2 >= needed):
                continue
            for rows in (32, 64, 128):
                for g in grids:
                    out.append({"kernel": "staged", "lanes_per_voxel": lv, "window_rows": rows, "grid_shape": g})
    cplx = storage in ("c64", "cf16", "cbf16", "ci16")
    words = n_frames if cplx else (n_frames // 2 if n_frames % 2 == 0 else 0)
    if words >= 32:  # lanes = frames, each element's rows loaded once for runs of 16 / 8 / 4 voxels
        for slots in (1, 2, 4):
            if slots > 1 and words <= 32 * (slots // 2):
                continue
            out.append({"kernel": "frame_lane", "frame_slots": slots})
    if n_frames >= (32 if cplx else 64) and (n_frames * esz) % 16 == 0:
        for rows in (32, 48, 64):
            for g in grids:
                out.append({"kernel": "ensemble", "window_rows": rows, "grid_shape": g})
    if n_frames > 1:
        out.append({"kernel": "warp"})
    return out


_DEVICE_NAMES: dict[int, str] = {}
_LOADED = False

KNOBS = ("kernel", "tx_chunk", "window_rows", "lanes_per_voxel", "tile_fast", "frame_slots", "element_block",
         "grid_shape")


def resolve_delay(storage: str, delay: str) -> str:
    """The delay mode a call runs with ("auto": mach's FP32 arithmetic for float32 / complex64
    storage, split delays otherwise)."""
    if delay == "auto":
        return "reference" if storage in ("f32", "c64") else "split"
    return delay


def _device_name(index: int) -> str:
    name = _DEVICE_NAMES.get(index)
    if name is None:
        import torch

        name = _DEVICE_NAMES[index] = torch.cuda.get_device_name(index)
    return name


def lookup(storage, n_tx, n_rx, n_samples, n_frames, n_vox, grid, interp, device_index, delay) -> dict | None:
    """Launch knobs the autotuner chose for this job shape, or None if it has not timed one.
    Reads the cache file once per process; called by every automatic beamforming call."""
    global _LOADED
    key = _key(storage, n_tx, n_rx, n_samples, n_frames, n_vox, grid, interp, _device_name(device_index),
               resolve_delay(storage, delay))
    with _LOCK:
        if key not in _MEMO and not _LOADED:
            _MEMO.update({k: v for k, v in _load().items() if k not in _MEMO})
            _LOADED = True
        hit = _MEMO.get(key)
    return _restore(hit) if hit is not None else None


def _key(storage, n_tx, n_rx, n_samples, n_frames, n_vox, grid, interp, device_name, delay="auto") -> str:
    return (f"{device_name}|{storage}|tx{n_tx}|rx{n_rx}|s{n_samples}|f{n_frames}|v{n_vox}|g{grid}|i{int(interp)}"
            f"|d{delay}")


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load()
        data[key] = value
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the cache


def tune(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, *, reps: int = 3, use_cache: bool = True,
         **params) -> dict:
    """Fastest launch settings for this job; returns keyword arguments for
    :func:`mach_b200.experimental.beamform` (and ``Job.tuning``).

    All arrays must be torch CUDA tensors; ``params`` are the beamforming parameters
    (``f_number``, ``rx_start_s``, ...).  The job runs ``reps`` times per candidate into a
    scratch output, so the caller's buffers are untouched.
    """
    import torch

    from mach_b200 import _cuda_impl, _dlpack, experimental

    pairs = channel_data.dim() == 5
    storage = _cuda_impl.storage_of(_dlpack.view(channel_data), pairs)
    n_tx, n_rx, n_samples, n_frames = (int(d) for d in channel_data.shape[:4])
    n_vox = int(scan_coords_m.shape[0])
    grid = _grid.detect(scan_coords_m)
    key = _key(storage, n_tx, n_rx, n_samples, n_frames, n_vox, grid, params.get("interp_type", 1),
               _device_name(channel_data.device.index or 0), resolve_delay(storage, params.get("delay", "auto")))
    if use_cache:
        with _LOCK:
            if key in _MEMO:
                return _restore(_MEMO[key])
            hit = _load().get(key)
        if hit is not None:
            _MEMO[key] = hit
            return _restore(hit)

    cplx = bool(_cuda_impl.STORAGE_CODES[storage] & 1)
    scratch = torch.zeros((n_vox, n_frames), dtype=torch.complex64 if cplx else torch.float32,
                          device=channel_data.device)
    stream = torch.cuda.current_stream()
    best, best_ms, timings = None, float("inf"), []
    for cand in candidates(storage, n_frames, grid):
        kw = dict(cand)

        def run():
            experimental.beamform(channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, scratch, sync=False,
                                  **params, **kw)

        try:
            run()  # warm-up (module load, occupancy queries)
        except (RuntimeError, ValueError):
            continue
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            run()
        stop.record(stream)
        stop.synchronize()
        ms = start.elapsed_time(stop) / reps
        timings.append((ms, cand))
        if ms < best_ms:
            best, best_ms = cand, ms
    if best is None:
        raise RuntimeError("no launch candidate ran for this job")
    entry = dict(best)
    entry["ms"] = best_ms
    with _LOCK:
        _MEMO[key] = entry
    if use_cache:
        _store(key, entry)
    return _restore(entry)


def _restore(entry: dict) -> dict:
    return {k: v for k, v in entry.items() if k != "ms"}
