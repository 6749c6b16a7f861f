#!/usr/bin/env python
"""Benchmark: delay-and-sum throughput in points/s (voxel x channel x transmit x frame).

One step = one complete beamforming job of the chosen workload with every input already in
HBM.  The default workload is the largest single-GPU configuration: 3-D DAS, 9 diverging
waves, 32 x 32 matrix array (1024 elements), 128^3 voxels, 2048 int16 RF samples x 16
frames, linear interpolation, f# 1.0.  The same JSON line also carries, under "workloads",
the Doppler ensemble (5 plane waves x 200 frames, 256^2, complex64 and FP16 IQ storage) and
the 75-transmit compounding job measured the same way in the same process, and on one GPU,
under "serving", the serving stream (`--workload serving`).  Prints ONE JSON line on rank 0.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload compound|doppler|plain2d|volume3d|volume3d16|serving|rf2iq|ingest]
                  [--storage c64|cf16|...] [--also doppler:c64,doppler:cf16,compound:c64 | --also none]

rf2iq and ingest time the front end before the beamformer (RF -> IQ by the analytic signal,
and the acquisition-order rearrange) in channel samples/s.

--impl reference times mach's own CUDA kernel (built from its unmodified source into
oracle/_ref) on the same inputs, driven as mach drives it: one launch and one
cudaDeviceSynchronize per transmit into a zeroed output, float32 / complex64 input (int16
and FP16 storage are widened for it, as mach only takes those two types).  That process
imports nothing of mach_b200 that opens its CUDA library.

Multi-GPU (torchrun): every rank runs its own full job on its own GPU (voxels and jobs are
independent; there is no data exchange), so scaling is weak; the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings
from datetime import timedelta
from pathlib import Path

import numpy as np
import torch

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "points/s (voxel*channel*transmit*frame)"

WORKLOAD_DESC = {
    "compound": "75 plane waves -16..16 deg, 128-el linear array, 512x512 grid (40x50 mm), 3328 IQ samples, "
    "quadratic interpolation, f# 1.75, Tukey 0.5",
    "doppler": "5 plane waves x 200 frames, 128 el, 256x256 grid, 1024 IQ samples, linear, f# 1.0",
    "plain2d": "single 0 deg plane wave, 128 el, 256x256 grid, 2048 float32 RF samples, linear, Hann f# 1.5",
    "volume3d": "9 diverging waves, 32x32 matrix array, 128^3 grid, 2048 int16 RF samples, 1 frame, linear, f# 1.0",
    "volume3d16": "9 diverging waves, 32x32 matrix array, 128^3 grid, 2048 int16 RF samples, 16 frames, linear, f# 1.0",
    "rf2iq": "RF -> IQ front end (src/mach/io/uff.py:70-105 at modulation 0): float32 RF in acquisition order "
             "[3328 samples, 128 elements, 75 waves] -> analytic signal, complex64 in the beamformer's layout",
    "ingest": "Doppler channel-data ingest (examples/doppler.py:193-195): complex64 IQ in acquisition order "
              "[1024 samples, 128 elements, 5 waves, 200 frames] -> the beamformer's layout",
    "serving": "Poisson 2000 req/s (seed 4): 50% plain 2-D 256^2, 30% 75-tx compounding 384^2, 15% 32-frame Doppler "
               "256^2, 5% 3-D 1024-ch 96^3; FP16 storage, FP32 accumulation; resident data, continuous batching",
}

FRONTEND_SHAPES = {"rf2iq": (3328, 128, 75, 1), "ingest": (1024, 128, 5, 200)}  # acquisition order
FRONTEND_METRIC = "samples/s (channel samples through the front-end step)"

SERVING_RATE_HZ = 2000.0
SERVING_REQUESTS_PER_STEP = 100  # one step = 100 requests of the stream (50 ms of arrivals)


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=sorted(WORKLOAD_DESC), default="volume3d16")
    p.add_argument("--storage", default=None, help="channel storage (default: the workload's own)")
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU time of the cpu_baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--frames", type=int, default=None, help="override the workload's frame count (profiling)")
    p.add_argument("--side", type=int, default=None, help="override the 3-D grid side (profiling)")
    p.add_argument("--also", default=None,
                   help="extra workload:storage lines measured in the same run (default with the default "
                        "workload: doppler:c64,doppler:cf16; 'none' for none)")
    p.add_argument("--delay", choices=["reference", "split", "auto"], default="reference",
                   help="delay arithmetic: mach's FP32 (default), FP64-split, or the library default per storage")
    p.add_argument("--no-tune", dest="tune", action="store_false",
                   help="skip the autotuner pass in warm-up (run the planner's automatic choice)")
    p.add_argument("--launch", default="",
                   help="launch options for the headline job, e.g. kernel=frame_lane,frame_slots=4 (profiling)")
    return p.parse_args()


# ----------------------------------------------------------------------------- plumbing


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=180), device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        """Start sampling; returns once the first sample is in (at most 3 s), so that even a
        short timed region is bracketed by samples."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        t0 = time.perf_counter()
        while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        seen = len(self.lines)  # one more sample after the timed region (at most 1 s)
        t0 = time.perf_counter()
        while len(self.lines) == seen and time.perf_counter() - t0 < 1.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(key: str) -> dict:
    """DRAM and L2 bytes per launch of the dominant kernel of a workload, from one ncu capture
    summarised in profiles/ncu_traffic.json (not measured in this run)."""
    path = REPO / "profiles" / "ncu_traffic.json"
    if path.exists():
        entry = json.loads(path.read_text()).get(key)
        if entry:
            return entry
    return {}


_L2_PEAK = None


def l2_peak_gbs() -> float | None:
    """L2 read bandwidth of this GPU, measured now with the library's probe kernel: 16-byte
    L1-bypassing loads over a 32 MB and a 64 MB buffer (both well inside the 126 MB L2), the
    best of 5 timed launches of 8 passes each after one untimed launch; the larger of the two."""
    global _L2_PEAK
    if _L2_PEAK is not None:
        return _L2_PEAK
    from mach_b200 import _cuda_impl

    best = 0.0
    stream = torch.cuda.current_stream()
    for mb in (32, 64):
        buf = torch.ones(mb << 18, dtype=torch.float32, device="cuda")
        nbytes = buf.numel() * 4
        _cuda_impl.probe_l2_read(buf.data_ptr(), nbytes, 1, stream.cuda_stream)
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _cuda_impl.probe_l2_read(buf.data_ptr(), nbytes, 8, stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            best = max(best, nbytes * 8 / (a.elapsed_time(b) * 1e-3) / 1e9)
        del buf
    _L2_PEAK = best
    return best


def roofline(w, storage, kernel_s, key, sm_mhz=None) -> dict:
    """HBM roofline of the dominant kernel (algorithmic bytes / CUDA-event time) with the DRAM
    and L2 bytes of its ncu capture beside it (L2 against the probed L2 read bandwidth), and
    its instruction-issue floor: the capture's warp instructions per step at one warp
    instruction per SM sub-partition per clock (4 per SM), at the SM clock sampled in this
    run."""
    peak, peak_kind = measured_peak_hbm()
    alg = algorithmic_bytes(w, storage)
    achieved = alg / kernel_s / 1e9
    prof = profiled_traffic(key)
    r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
         "traffic": prof.get("dram_bytes"), "algorithmic_bytes_per_launch": alg, "kernel_ms": kernel_s * 1e3,
         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)" if peak_kind == "measured"
         else "fallback 6650 GB/s"}
    if prof:
        r["traffic_source"] = f"ncu capture, not this run: {prof.get('source', '')}"
    l2_peak = l2_peak_gbs()
    lts = prof.get("lts_bytes")
    if lts:
        r["l2_bytes_per_launch"] = lts
        r["l2_achieved"] = lts / kernel_s / 1e9
    if l2_peak:
        r["l2_peak"] = l2_peak
        r["l2_peak_source"] = "mach_b200_probe_l2_read in this run (ld.global.cg over 32/64 MB)"
        if lts:
            r["l2_frac"] = r["l2_achieved"] / l2_peak
    inst = prof.get("warp_inst")
    if inst and sm_mhz:
        n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        floor_s = inst / (4.0 * n_sm * sm_mhz * 1e6)
        r["issue"] = {"warp_inst_per_step": inst, "floor_ms": floor_s * 1e3, "frac": floor_s / kernel_s,
                      "sm_mhz": sm_mhz, "sms": n_sm, "source": prof.get("inst_source", "")}
    if prof.get("l1_wavefront_pct") is not None:
        r["l1_wavefront_pct_of_peak"] = prof["l1_wavefront_pct"]
    if prof.get("binding"):
        r["binding_limit"] = prof["binding"]
    return r


# ----------------------------------------------------------------------------- workloads


def make_workload(name: str, frames: int | None = None, side: int | None = None):
    from mach_b200 import workloads as W

    grid = {"n_side": side} if side else {}
    if name == "volume3d":
        w = W.volume3d(n_frames=frames or 1, device="cuda", **grid)
    elif name == "volume3d16":
        w = W.volume3d(n_frames=frames or 16, device="cuda", **grid)
    elif name == "doppler" and frames:
        w = W.doppler(n_frames=frames, device="cuda")
    else:
        w = W.CONFIGS[name](device="cuda")
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # drop the synthesis temporaries
    return w


def storage_channel(w, storage):
    """Channel data in the requested storage; sets ``w.storage_scale`` for int16."""
    from mach_b200 import workloads as W

    ch, scale = W.as_storage(w, storage)
    w.storage_scale = scale
    return ch.contiguous()


def algorithmic_bytes(w, storage) -> int:
    esz = {"f32": 4, "c64": 8, "f16": 2, "cf16": 4, "bf16": 2, "cbf16": 4, "i16": 2, "ci16": 4}[storage]
    out_esz = 8 if storage in ("c64", "cf16", "cbf16", "ci16") else 4
    return (w.n_tx * w.n_rx * w.n_samples * w.n_frames * esz + w.n_tx * w.n_vox * 4 + w.n_vox * 12 + w.n_rx * 12
            + w.n_vox * w.n_frames * out_esz)


# ----------------------------------------------------------------------------- our arm


def workload_config(name, w, storage, world) -> dict:
    """The `config` of a line: identical in both arms for the same workload."""
    return {
        "workload": f"{name}: {WORKLOAD_DESC[name]}",
        "storage": storage,
        "n_tx": w.n_tx, "n_rx": w.n_rx, "n_samples": w.n_samples, "n_frames": w.n_frames, "n_vox": w.n_vox,
        "points_per_step": w.points,
        "l2": f"inputs larger than L2 ({algorithmic_bytes(w, storage) / 1e6:.0f} MB per step > 126 MB), no flush",
        "parallelism": f"replicas x{world} (one job per GPU, no exchange)",
    }


DELAY_CHOICE = "reference"


def delay_mode(storage: str) -> str:
    """Delay arithmetic of the measured lines: mach's FP32 delays by default (the reference
    kernel's own arithmetic); `--delay split` forms sample positions in FP64 split form, and
    `--delay auto` takes the library's default (split for 16-bit floating-point storage)."""
    if DELAY_CHOICE == "auto":
        return "split" if storage in ("f16", "cf16", "bf16", "cbf16") else "reference"
    return DELAY_CHOICE


def default_line(args) -> bool:
    """The default run (no workload, frame or grid override): it also measures the Doppler and
    compounding lines and, on one GPU, the serving stream."""
    return args.workload == "volume3d16" and not args.frames and not args.side and args.also is None


def with_serving(line: dict, runner, args, world, rank, local) -> dict:
    """Attach the serving stream's line to the default line (one GPU only); a failure there is
    recorded in the line instead of losing the headline."""
    if not default_line(args) or world != 1:
        return line
    try:
        line["serving"] = runner(args, world, rank, local)
    except Exception as exc:  # noqa: BLE001 - reported in the JSON line
        line["serving"] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    return line


def parse_also(args) -> list[tuple[str, str | None]]:
    spec = args.also
    if spec is None:
        spec = "doppler:c64,doppler:cf16,compound:c64" if default_line(args) else "none"
    if spec.strip().lower() in ("", "none"):
        return []
    out = []
    for item in spec.split(","):
        name, _, storage = item.strip().partition(":")
        if name not in WORKLOAD_DESC or name in ("serving", "rf2iq", "ingest"):
            raise SystemExit(f"--also: unknown beamforming workload {name!r}")
        out.append((name, storage or None))
    return out


def run_ours(args, world, rank, local):
    line = measure_ours(args, args.workload, args.storage, world, rank, local, headline=True)
    also = parse_also(args)
    if also:
        line["workloads"] = [measure_ours(args, name, storage, world, rank, local, headline=False)
                             for name, storage in also]
    return with_serving(line, run_serving, args, world, rank, local)


def measure_ours(args, name, storage, world, rank, local, headline):
    """One workload through the C ABI (kernel-only `value`, device-resident inputs), its e2e
    through the public API, and on rank 0 its accuracy (and, for the headline, the CPU baseline)."""
    from mach_b200 import _cuda_impl, _dlpack, _grid

    frames, side = (args.frames, args.side) if headline else (None, None)
    w = make_workload(name, frames, side)
    storage = storage or w.storage
    ch = storage_channel(w, storage)
    dev = torch.device("cuda", local)
    rx = torch.as_tensor(w.rx_coords_m, device=dev)
    scan = torch.as_tensor(w.scan_coords_m, device=dev)
    arr = torch.as_tensor(w.tx_wave_arrivals_s, device=dev)
    is_c = storage in ("c64", "cf16", "cbf16", "ci16")
    out = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if is_c else torch.float32, device=dev)
    v_ch, v_rx, v_scan, v_arr, v_out = (_dlpack.view(t) for t in (ch, rx, scan, arr, out))
    stream = torch.cuda.current_stream(dev)
    p = w.params
    common = dict(n_tx=w.n_tx, n_rx=w.n_rx, n_samples=w.n_samples, n_vox=w.n_vox, n_frames=w.n_frames,
                  f_number=p["f_number"], rx_start_s=p["rx_start_s"], sampling_freq_hz=p["sampling_freq_hz"],
                  sound_speed_m_s=p["sound_speed_m_s"], modulation_freq_hz=p["modulation_freq_hz"],
                  tukey_alpha=p["tukey_alpha"], interp_type=p["interp_type"], channel_scale=w.storage_scale)
    grid_shape = _grid.detect(w.scan_coords_m)
    knobs = {}
    if headline and args.launch:
        for item in args.launch.split(","):
            key, _, val = item.partition("=")
            knobs[key.strip()] = val.strip() if key.strip() == "kernel" else int(val)
    if args.tune and not knobs:
        from mach_b200 import tuning

        knobs = tuning.tune(ch, rx, scan, arr, channel_scale=w.storage_scale, delay=delay_mode(storage), **p)
        grid_shape = knobs.pop("grid_shape", grid_shape)
        if grid_shape is False:
            grid_shape = None
    options = _cuda_impl.make_options(grid_shape=grid_shape, **knobs)
    flags = _cuda_impl.FLAG_ASYNC | _cuda_impl.FLAG_OVERWRITE
    # Storage whose samples are exact in FP32 (float32, complex64, int16 x scale) uses mach's
    # FP32 delay arithmetic (bit-identical sample positions); FP16 / BF16 storage uses split
    # delays, the API's default for it.
    delay = delay_mode(storage)
    if delay == "split":
        flags |= _cuda_impl.FLAG_SPLIT_DELAY

    def step():
        _cuda_impl.beamform_compound(v_ch, storage, v_rx, v_scan, v_arr, v_out, stream=stream.cuda_stream,
                                     flags=flags, options=options, **common)

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = _cuda_impl.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches = _cuda_impl.launch_count() - launches0
    clock_info = clocks.stop()
    per_step = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = starts[0].elapsed_time(ends[-1])
    total_ms = max_over_ranks(total_ms, world)
    result = out.clone()

    line = {
        "metric": METRIC,
        "value": world * w.points * args.steps / (total_ms / 1e3),
        "unit": "points/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded simulation of the configuration; no public dataset offline)",
        "config": workload_config(name, w, storage, world),
        "latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99))},
        "gpu_launches": int(launches),
        "launch": {"delay": delay,
                   "grid_shape": list(grid_shape) if grid_shape else None, "knobs": knobs or None,
                   "tuned": bool(args.tune and not (headline and args.launch))},
    }
    kernel_s = statistics.mean(per_step) / 1e3
    line["roofline"] = roofline(w, storage, kernel_s, f"{name}:{storage}", sm_mhz=clock_info.get("sm_mhz"))
    line["clocks"] = clock_info
    if not args.no_e2e:
        line["e2e"] = run_e2e(args, w, storage, ch, world, local, dict(knobs, grid_shape=grid_shape or False))
    if rank == 0 and world == 1:
        line.update(accuracy_and_baselines(args, w, storage, result, cpu_baseline=headline))
    del ch, rx, scan, arr, out, result, v_ch, v_out
    w.channel = None
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return line


def accuracy_and_baselines(args, w, storage, result, cpu_baseline=True):
    """nRMS against the FP64 oracle on a voxel sample (which also gives the CPU baseline rate),
    and relative L2 against mach's kernel on the whole job."""
    from oracle import das_fp64, machref, oracle_c

    extra = {}
    ch_np = storage_numpy(w, storage)
    src_np = storage_numpy(w, w.storage)
    keys = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
            "interp_type")
    p = {k: w.params[k] for k in keys}
    cores = os.cpu_count() or 1

    def oracle_on(n_sub, data, st, scale):
        sel = np.unique(np.linspace(0, w.n_vox - 1, n_sub).astype(np.int64))
        t = time.perf_counter()
        y = oracle_c.beamform_c(data, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, storage=st,
                                channel_scale=scale, voxel_subset=sel, n_threads=cores, **p)
        return sel, y, time.perf_counter() - t

    n_sub = 256
    sel, y, dt = oracle_on(n_sub, ch_np, storage, w.storage_scale)
    if cpu_baseline and not args.no_cpu_baseline:
        while dt < 0.25 * args.cpu_seconds and n_sub < w.n_vox:
            n_sub = int(min(w.n_vox, n_sub * max(2.0, 0.5 * args.cpu_seconds / max(dt, 1e-3))))
            sel, y, dt = oracle_on(n_sub, ch_np, storage, w.storage_scale)
        reps = 1
        if dt < 0.25 * args.cpu_seconds:  # the whole job is quick on the CPU: time repeated passes
            reps = int(min(1000, np.ceil(0.5 * args.cpu_seconds / max(dt, 1e-4))))
            t_rep = time.perf_counter()
            for _ in range(reps):
                oracle_on(n_sub, ch_np, storage, w.storage_scale)
            dt = time.perf_counter() - t_rep
        pts = len(sel) * w.n_rx * w.n_tx * w.n_frames * reps
        extra["cpu_baseline"] = {
            "value": pts / dt, "unit": "points/s", "cores": cores, "kind": "port",
            "sample": f"{len(sel)} of {w.n_vox} voxels (evenly spaced) x all elements/transmits/frames"
                      f"{f', {reps} passes' if reps > 1 else ''}; FP64 C restatement (oracle/das_oracle.c), "
                      f"OpenMP, {dt:.1f} s",
        }
    got = result.cpu().numpy()[sel]
    acc = {"nrms_db_vs_fp64_oracle_on_stored_samples": das_fp64.nrms_db(got, y), "oracle_voxels": int(len(sel))}
    if storage != w.storage:
        _, y_src, _ = oracle_on(len(sel), src_np, w.storage, w.channel_scale)
        acc["nrms_db_vs_fp64_oracle_on_source_data"] = das_fp64.nrms_db(got, y_src)
    if machref.available() and w.storage in ("c64", "f32", "i16"):
        ref = reference_once(w)
        # mach takes float32 / complex64 only: int16 is widened exactly, so the same samples;
        # FP16 / BF16 storage is compared against mach on the unrounded source data.
        key = "rel_l2_vs_reference_kernel" if storage == w.storage else "rel_l2_vs_reference_kernel_on_source_data"
        acc[key] = das_fp64.rel_l2(result.cpu().numpy(), ref)
    extra["accuracy"] = acc
    return extra


def storage_numpy(w, storage):
    from mach_b200 import workloads as W

    ch, _ = W.as_storage(w, storage)
    if ch.dtype == torch.bfloat16:
        return ch.view(torch.int16).cpu().numpy().view(np.uint16)
    return ch.cpu().numpy()


def reference_once(w):
    from oracle import machref

    ch = w.channel
    if ch.dtype == torch.int16:
        ch = ch.to(torch.float32) * w.channel_scale
    ch = ch.cuda().contiguous()
    rx = torch.as_tensor(w.rx_coords_m, device="cuda")
    scan = torch.as_tensor(w.scan_coords_m, device="cuda")
    arr = torch.as_tensor(w.tx_wave_arrivals_s, device="cuda")
    out = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if ch.is_complex() else torch.float32,
                      device="cuda")
    machref.beamform_device([ch[t].data_ptr() for t in range(w.n_tx)], rx.data_ptr(), scan.data_ptr(),
                            [arr[t].data_ptr() for t in range(w.n_tx)], out.data_ptr(), is_complex=ch.is_complex(),
                            n_rx=w.n_rx, n_samples=w.n_samples, n_vox=w.n_vox, n_frames=w.n_frames,
                            **{k: w.params[k] for k in ("f_number", "rx_start_s", "sampling_freq_hz",
                                                        "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
                                                        "interp_type")})
    torch.cuda.synchronize()
    return out.cpu().numpy()


def run_e2e(args, w, storage, ch_dev, world, local, knobs=None):
    """Same job through the public API with pinned host buffers: H2D + kernel + D2H per step."""
    from mach_b200 import experimental

    ch_h = ch_dev.cpu().pin_memory()
    rx_h = torch.as_tensor(w.rx_coords_m).pin_memory()
    scan_h = torch.as_tensor(w.scan_coords_m).pin_memory()
    arr_h = torch.as_tensor(w.tx_wave_arrivals_s).pin_memory()
    is_c = storage in ("c64", "cf16", "cbf16", "ci16")
    out_h = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if is_c else torch.float32).pin_memory()

    def step():
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", UserWarning)
            experimental.beamform(ch_h, rx_h, scan_h, arr_h, out=out_h, channel_scale=w.storage_scale, **w.params,
                                  delay=delay_mode(storage), **(knobs or {}))

    for _ in range(max(1, min(args.warmup, 3))):
        step()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, world)
    h2d = ch_h.numel() * ch_h.element_size() + rx_h.numel() * 4 + scan_h.numel() * 4 + arr_h.numel() * 4
    d2h = out_h.numel() * out_h.element_size()
    return {"value": world * w.points * args.steps / dt, "unit": "points/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": dt / args.steps * 1e3,
            "api": "mach_b200.experimental.beamform with pinned host tensors"}


# ----------------------------------------------------------------------------- serving


def _serving_stream(args, classes, seed=4):
    from mach_b200 import serving

    n = max(1, args.steps) * SERVING_REQUESTS_PER_STEP
    return serving.poisson_arrivals(SERVING_RATE_HZ, n, [c.weight for c in classes], seed=seed)


def _serving_config(args, classes, n):
    return {
        "workload": f"serving: {WORKLOAD_DESC['serving']}",
        "requests": n, "rate_hz": SERVING_RATE_HZ,
        "classes": {c.name: {"storage": c.storage, "n_tx": c.workload.n_tx, "n_rx": c.workload.n_rx,
                             "n_samples": c.workload.n_samples, "n_frames": c.workload.n_frames,
                             "n_vox": c.workload.n_vox, "points": c.workload.points} for c in classes},
        "l2": "working set of the resident classes > 126 MB (compounding channel data alone 128 MB), no flush",
    }


SERVING_SWEEP_HZ = (200.0, 400.0, 600.0, 800.0, 1000.0)
SERVING_SWEEP_REQUESTS = 300


def _serve_once(engine, classes, rate, n, seed):
    """One stream through an engine; returns (requests, makespan_s, waves, graph replays)."""
    from mach_b200 import serving

    reqs = serving.poisson_arrivals(rate, n, [c.weight for c in classes], seed=seed)
    waves0, hits0 = len(engine.scheduler.waves), engine.executor.graph_hits
    engine.serve(reqs)
    waves = engine.scheduler.waves[waves0:]
    return reqs, max(r.done_s for r in reqs), waves, engine.executor.graph_hits - hits0


def run_serving(args, world, rank, local):
    """The serving stream through mach_b200.serving (continuous batching, graph replays):
    `value` with each class's acquisition resident in HBM, `e2e` with every request's own
    acquisition uploaded from pinned host memory and its image read back, and a rate sweep
    of the upload mode."""
    from mach_b200 import _cuda_impl, serving
    from mach_b200.batch import Batch, Job
    from oracle import das_fp64, oracle_c

    classes = serving.c4_classes()
    if args.tune:  # one autotuner pass per class; the engine's batch jobs run the tuned knobs
        from mach_b200 import tuning, workloads as W

        for c in classes:
            w = c.workload
            ch, scale = W.as_storage(w, c.storage)
            tuning.tune(ch.contiguous().cuda(), torch.as_tensor(w.rx_coords_m, device="cuda"),
                        torch.as_tensor(w.scan_coords_m, device="cuda"),
                        torch.as_tensor(w.tx_wave_arrivals_s, device="cuda"), channel_scale=scale, **w.params)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    engine = serving.ServingEngine(classes, slots_per_class=8)
    engine.serve(serving.poisson_arrivals(SERVING_RATE_HZ, max(100, args.warmup * SERVING_REQUESTS_PER_STEP),
                                          [c.weight for c in classes], seed=104))
    reqs = _serving_stream(args, classes)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = _cuda_impl.launch_count()
    replayed0 = engine.executor.replayed_kernels
    captured0 = engine.executor.captured_kernels
    waves0 = len(engine.scheduler.waves)
    hits0 = engine.executor.graph_hits
    engine.serve(reqs)
    launches = ((_cuda_impl.launch_count() - launches0) + (engine.executor.replayed_kernels - replayed0)
                - (engine.executor.captured_kernels - captured0))
    clock_info = clocks.stop()
    makespan = max_over_ranks(max(r.done_s for r in reqs), world)
    points = sum(classes[r.cls].points for r in reqs)
    waves = engine.scheduler.waves[waves0:]
    alg = sum(algorithmic_bytes(classes[r.cls].workload, classes[r.cls].storage) for r in reqs)
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / makespan / 1e9
    line = {
        "metric": METRIC, "value": world * points / makespan, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": makespan * 1e3 / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16 storage, f32 math",
        "data": "synthetic (seeded simulation of the configurations; no public dataset offline)",
        "config": _serving_config(args, classes, len(reqs)) | {
            "parallelism": f"replicas x{world} (one request stream per GPU, no exchange)"},
        "latency_ms": serving.latency_summary(reqs),
        "requests_per_s": len(reqs) / makespan,
        "tuned": {c.name: serving.class_tuning(c) for c in classes} if args.tune else None,
        "waves": {"count": len(waves), "mean_requests": float(np.mean([len(w.requests) for w in waves])),
                  "graph_replays": engine.executor.graph_hits - hits0},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "algorithmic_bytes_per_launch": None,
                     "note": "algorithmic bytes of all requests / makespan", "peak_source": peak_kind},
        "clocks": clock_info,
        "mode": "value: each class's acquisition resident in HBM (output slots only)",
    }
    if rank == 0 and world == 1:
        params = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz",
                  "tukey_alpha", "interp_type")
        acc = {}
        for c in classes:
            t = c.tensors
            job = Job(channel=t["channel"], rx_coords_m=t["rx"], scan_coords_m=t["scan"], arrivals=t["arr"],
                      channel_scale=t["scale"], **{k: c.workload.params[k] for k in params})
            b = Batch([job])
            b.run(sync=True)
            w = c.workload
            sel = np.unique(np.linspace(0, w.n_vox - 1, 128).astype(np.int64))
            y = oracle_c.beamform_c(storage_numpy(w, c.storage), w.rx_coords_m, w.scan_coords_m,
                                    w.tx_wave_arrivals_s, storage=c.storage, channel_scale=t["scale"],
                                    voxel_subset=sel, **{k: w.params[k] for k in params})
            acc[c.name] = das_fp64.nrms_db(job.out.cpu().numpy()[sel], y)
            b.close()
        line["accuracy"] = {"nrms_db_vs_fp64_oracle_on_stored_samples": acc, "oracle_voxels_per_class": 128}
        if not args.no_cpu_baseline:
            w = classes[0].workload
            w.storage_scale = classes[0].tensors["scale"]
            cpu = accuracy_and_baselines(args, w, classes[0].storage, _alone_result(classes[0]))
            line["cpu_baseline"] = cpu.get("cpu_baseline")
            if line["cpu_baseline"]:
                line["cpu_baseline"]["sample"] = "plain 2-D class: " + line["cpu_baseline"]["sample"]
    del engine
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # ---- upload mode: the same stream, every request's acquisition from pinned host memory
    if not args.no_e2e:
        up = serving.ServingEngine(classes, slots_per_class=8, upload=True)
        _serve_once(up, classes, SERVING_RATE_HZ, max(100, args.warmup * SERVING_REQUESTS_PER_STEP), 104)
        reqs_u, span_u, waves_u, _ = _serve_once(up, classes, SERVING_RATE_HZ, len(reqs), 4)
        span_u = max_over_ranks(span_u, world)
        h2d = sum(up.executor.bytes_per_request(r.cls)[0] for r in reqs_u)
        d2h = sum(up.executor.bytes_per_request(r.cls)[1] for r in reqs_u)
        steps = max(1, args.steps)
        line["e2e"] = {"value": world * sum(classes[r.cls].points for r in reqs_u) / span_u, "unit": "points/s",
                       "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": int(d2h / steps),
                       "ms_per_step": span_u * 1e3 / steps, "requests_per_s": len(reqs_u) / span_u,
                       "latency_ms": serving.latency_summary(reqs_u),
                       "api": "mach_b200.serving upload mode: per-request H2D of its own acquisition from pinned "
                              "host memory on a copy stream, D2H of its image"}
        sweep = []
        for i, rate in enumerate(SERVING_SWEEP_HZ):
            rq, span, _, _ = _serve_once(up, classes, rate, SERVING_SWEEP_REQUESTS, 200 + i)
            served = len(rq) / span
            lat = serving.latency_summary(rq)
            sweep.append({"rate_hz": rate, "requests_per_s": served, "latency_ms": lat,
                          "sustained": bool(served >= 0.95 * rate * (1 - 1.0 / len(rq)))})
        ok = [x for x in sweep if x["sustained"]]
        line["rate_sweep"] = {"mode": "upload", "requests_per_rate": SERVING_SWEEP_REQUESTS, "points": sweep,
                              "highest_sustained_hz": max((x["rate_hz"] for x in ok), default=None),
                              "rule": "sustained: served >= 95% of the offered rate over the stream"}
        del up
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return line


def _alone_result(c):
    from mach_b200.batch import Batch, Job

    t = c.tensors
    params = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
              "interp_type")
    job = Job(channel=t["channel"], rx_coords_m=t["rx"], scan_coords_m=t["scan"], arrivals=t["arr"],
              channel_scale=t["scale"], **{k: c.workload.params[k] for k in params})
    b = Batch([job])
    b.run(sync=True)
    out = job.out.clone()
    b.close()
    return out


SERVING_REFERENCE_SECONDS = 15.0


def run_serving_reference(args, world, rank, local):
    """mach's kernel served serially over the same arrival stream, in real time: each request
    starts when it has arrived and the previous one is done, and runs mach's path for one job
    (one launch + cudaDeviceSynchronize per transmit, float32 / complex64 input as mach
    requires, the request's own acquisition).  `value`: inputs already on the device; `e2e`:
    host inputs through mach's binding (its CPU staging path) and the image read back.  Each
    run stops after SERVING_REFERENCE_SECONDS of serving; the requests served by then count."""
    from mach_b200 import serving, workloads as W
    from oracle import machref

    if not machref.available():
        return {"impl": "reference", "unavailable": "mach's kernel was not built into oracle/_ref (no reference checkout)"}
    classes = serving.c4_classes()
    keys = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
            "interp_type")
    prep = []
    for c in classes:
        w = c.workload
        src = "c64" if c.storage in ("cf16", "cbf16", "ci16", "c64") else "f32"
        ch, scale = W.as_storage(w, src)
        ch = (ch * scale).contiguous().cuda() if scale != 1.0 else ch.contiguous().cuda()
        acqs = serving.make_acquisitions(ch, 2)  # the two acquisitions our upload mode serves
        d = {"acq_dev": [a.cuda() for a in acqs], "acq_host": [a.numpy() for a in acqs],
             "rx": torch.as_tensor(w.rx_coords_m, device="cuda"), "scan": torch.as_tensor(w.scan_coords_m, device="cuda"),
             "arr": torch.as_tensor(w.tx_wave_arrivals_s, device="cuda"),
             "rx_h": w.rx_coords_m, "scan_h": w.scan_coords_m, "arr_h": np.ascontiguousarray(w.tx_wave_arrivals_s),
             "p": {k: w.params[k] for k in keys}, "w": w, "cplx": ch.is_complex()}
        d["out"] = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if d["cplx"] else torch.float32,
                               device="cuda")
        d["out_h"] = torch.zeros(d["out"].shape, dtype=d["out"].dtype).pin_memory()
        prep.append(d)
        del ch

    def job(d, acq, host):
        w = d["w"]
        d["out"].zero_()
        if host:
            machref.beamform_host(d["acq_host"][acq], d["rx_h"], d["scan_h"], d["arr_h"], None,
                                  out_on_device_ptr=d["out"].data_ptr(), **d["p"])
            d["out_h"].copy_(d["out"])
        else:
            ch, arr = d["acq_dev"][acq], d["arr"]
            machref.beamform_device([ch[t].data_ptr() for t in range(w.n_tx)], d["rx"].data_ptr(),
                                    d["scan"].data_ptr(), [arr[t].data_ptr() for t in range(w.n_tx)],
                                    d["out"].data_ptr(), is_complex=d["cplx"], n_rx=w.n_rx, n_samples=w.n_samples,
                                    n_vox=w.n_vox, n_frames=w.n_frames, **d["p"])
        torch.cuda.synchronize()

    def serve(host, rate, n, seed, seconds):
        reqs = serving.poisson_arrivals(rate, n, [c.weight for c in classes], seed=seed)
        for d in prep:  # warm-up of every class
            job(d, 0, host)
        done = []
        t0 = time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t0
            if now > seconds:
                break
            if now < r.arrival_s:
                time.sleep(r.arrival_s - now)
            job(prep[r.cls], r.rid % 2, host)
            r.done_s = time.perf_counter() - t0
            done.append(r)
        return reqs, done, max(r.done_s for r in done)

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    reqs, done, span = serve(False, SERVING_RATE_HZ, max(1, args.steps) * SERVING_REQUESTS_PER_STEP, 4,
                             SERVING_REFERENCE_SECONDS)
    clock_info = clocks.stop()
    points = sum(classes[r.cls].points for r in done)
    line = {
        "metric": METRIC, "value": points / span, "unit": "points/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": span * 1e3 / max(1, len(done)) *
        SERVING_REQUESTS_PER_STEP,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded simulation of the configurations; no public dataset offline)",
        "config": _serving_config(args, classes, len(reqs)) | {
            "parallelism": f"replicas x{world} (one request stream per GPU, no exchange)"},
        "reference": "mach's kernel (src/mach/kernel.cu, unmodified, sm_100a) serving the same arrival stream serially "
                     "in real time, one launch + cudaDeviceSynchronize per transmit, float32/complex64 input; rank 0 "
                     "only",
        "served_requests": len(done), "served_seconds": span,
        "latency_ms": serving.latency_summary(done),
        "requests_per_s": len(done) / span,
        "clocks": clock_info,
        "gpu_launches": int(sum(classes[r.cls].workload.n_tx for r in done)),
        "mode": "value: each request's acquisition already on the device",
    }
    if not args.no_e2e:
        _, done_h, span_h = serve(True, SERVING_RATE_HZ, max(1, args.steps) * SERVING_REQUESTS_PER_STEP, 4,
                                  SERVING_REFERENCE_SECONDS)
        # per transmit, mach's binding copies that transmit's channel data and arrivals plus the
        # element and scan coordinates
        h2d = sum(prep[r.cls]["acq_host"][0].nbytes + prep[r.cls]["arr_h"].nbytes
                  + (prep[r.cls]["rx_h"].nbytes + prep[r.cls]["scan_h"].nbytes) * classes[r.cls].workload.n_tx
                  for r in done_h)
        d2h = sum(prep[r.cls]["out_h"].numel() * prep[r.cls]["out_h"].element_size() for r in done_h)
        per_step = len(done_h) / SERVING_REQUESTS_PER_STEP
        line["e2e"] = {"value": sum(classes[r.cls].points for r in done_h) / span_h, "unit": "points/s",
                       "h2d_bytes_per_step": int(h2d / per_step), "d2h_bytes_per_step": int(d2h / per_step),
                       "requests_per_s": len(done_h) / span_h, "served_requests": len(done_h),
                       "latency_ms": serving.latency_summary(done_h),
                       "api": "mach's binding with host arrays per transmit (its CPU staging path), image read back"}
    return line


# ----------------------------------------------------------------------------- front end (RF -> IQ, ingest)


def frontend_input(name: str, device) -> torch.Tensor:
    """Seeded acquisition-order channel data: Gaussian RF (rf2iq) or IQ (ingest) samples."""
    g = torch.Generator(device=device).manual_seed(11)
    shape = FRONTEND_SHAPES[name]
    if name == "rf2iq":
        return torch.randn(shape, device=device, generator=g)
    return torch.complex(torch.randn(shape, device=device, generator=g), torch.randn(shape, device=device, generator=g))


def frontend_reference_step(name: str, x: np.ndarray) -> np.ndarray:
    """What mach runs on the host for this step: scipy.signal.hilbert on axis 0 then the einops
    rearrange (src/mach/io/uff.py:86-105), or the rearrange with the complex64 cast
    (examples/doppler.py:193-195)."""
    import einops

    pattern = "n_samples n_elements n_waves n_frames -> n_waves n_elements n_samples n_frames"
    if name == "rf2iq":
        import scipy.signal

        return np.asarray(einops.rearrange(scipy.signal.hilbert(x, axis=0), pattern))
    return np.ascontiguousarray(einops.rearrange(x, pattern), dtype=np.complex64)


def run_frontend(args, world, rank, local):
    """One step = the whole front-end job of the workload on the GPU (one kernel launch)."""
    from mach_b200 import _cuda_impl, ingest
    from oracle import analytic

    dev = torch.device("cuda", local)
    x = frontend_input(args.workload, dev)
    n_s, n_e, n_w, n_f = FRONTEND_SHAPES[args.workload]
    storage = args.storage or "c64"

    def run(src, out=None, sync=False):
        if args.workload == "rf2iq":
            return ingest.preprocess_signal(src, 0.0, storage=storage, out=out, sync=sync)
        return ingest.ingest(src, storage, out=out, sync=sync)

    out = run(x)
    torch.cuda.synchronize()
    samples = x.numel()
    alg = x.numel() * x.element_size() + out.numel() * out.element_size()

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        run(x, out)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = _cuda_impl.launch_count()
    stream = torch.cuda.current_stream(dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        starts[i].record(stream)
        run(x, out)
        ends[i].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches = _cuda_impl.launch_count() - launches0
    clock_info = clocks.stop()
    per_step = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = max_over_ranks(starts[0].elapsed_time(ends[-1]), world)
    kernel_s = statistics.mean(per_step) / 1e3
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / kernel_s / 1e9
    line = {
        "metric": FRONTEND_METRIC, "value": world * samples * args.steps / (total_ms / 1e3), "unit": "samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.workload == "rf2iq" else "c64",
        "data": "synthetic (seeded Gaussian channel samples; no public dataset offline)",
        "config": {"workload": f"{args.workload}: {WORKLOAD_DESC[args.workload]}", "storage_out": storage,
                   "shape_in": [n_s, n_e, n_w, n_f], "samples_per_step": samples,
                   "l2": f"inputs larger than L2 ({alg / 1e6:.0f} MB per step > 126 MB), no flush",
                   "parallelism": f"replicas x{world} (one job per GPU, no exchange)"},
        "latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99))},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profiled_traffic(f"{args.workload}:{storage}").get("dram_bytes"),
                     "traffic_source": "ncu capture, not this run: "
                                       + profiled_traffic(f"{args.workload}:{storage}").get("source", ""),
                     "algorithmic_bytes_per_launch": alg,
                     "kernel_ms": kernel_s * 1e3, "peak_source": peak_kind},
        "clocks": clock_info,
    }
    if not args.no_e2e:  # pinned host input -> GPU -> pinned host output, through the public API
        x_h = x.cpu().pin_memory()
        out_h = torch.empty(out.shape, dtype=out.dtype).pin_memory()

        def e2e_step():
            run(x_h, out)
            out_h.copy_(out, non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()

        e2e_step()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        dt = max_over_ranks(time.perf_counter() - t0, world)
        line["e2e"] = {"value": world * samples * args.steps / dt, "unit": "samples/s",
                       "h2d_bytes_per_step": int(x_h.numel() * x_h.element_size()),
                       "d2h_bytes_per_step": int(out_h.numel() * out_h.element_size()),
                       "ms_per_step": dt / args.steps * 1e3, "api": "mach_b200.ingest with pinned host tensors"}
    if rank == 0 and world == 1:
        # accuracy against the FP64 oracle and the CPU baseline (mach's host step), on a sample of waves
        x_np = x.cpu().numpy()
        got = out.cpu().numpy()
        if got.ndim == 5:
            got = got[..., 0] + 1j * got[..., 1]

        def host(n_take):
            t0 = time.perf_counter()
            r = frontend_reference_step(args.workload, x_np[:, :, :n_take])
            return r, time.perf_counter() - t0

        n_take = 1
        ref, dt = host(n_take)
        while dt < 0.25 * args.cpu_seconds and n_take < n_w:
            n_take = min(n_w, max(n_take + 1, int(n_take * 0.5 * args.cpu_seconds / max(dt, 1e-3))))
            ref, dt = host(n_take)
        reps = 1
        if dt < 0.25 * args.cpu_seconds:
            reps = int(min(100, np.ceil(0.5 * args.cpu_seconds / max(dt, 1e-4))))
            t0 = time.perf_counter()
            for _ in range(reps):
                host(n_take)
            dt = time.perf_counter() - t0
        if not args.no_cpu_baseline:
            what = "scipy.signal.hilbert + einops rearrange" if args.workload == "rf2iq" else \
                "einops rearrange + complex64 cast"
            line["cpu_baseline"] = {
                "value": n_s * n_e * n_take * n_f * reps / dt, "unit": "samples/s", "cores": 1, "kind": "reference",
                "sample": f"{n_take} of {n_w} waves{f', {reps} passes' if reps > 1 else ''}: mach's host step "
                          f"({what}), {dt:.1f} s"}
        want = analytic.preprocess_signal(x_np[:, :, :n_take]) if args.workload == "rf2iq" else ref
        line["accuracy"] = {"rel_l2_vs_fp64_oracle": float(np.linalg.norm(got[:n_take] - want) / np.linalg.norm(want)),
                            "waves_checked": n_take}
    return line


def run_frontend_reference(args, world, rank, local):
    """mach's host implementation of the front-end step (scipy / einops / NumPy), whole job per step."""
    x = frontend_input(args.workload, torch.device("cuda", local)).cpu().numpy()
    n_s, n_e, n_w, n_f = FRONTEND_SHAPES[args.workload]
    for _ in range(min(args.warmup, 1)):
        frontend_reference_step(args.workload, x)
    lat = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s = time.perf_counter()
        frontend_reference_step(args.workload, x)
        lat.append((time.perf_counter() - s) * 1e3)
    dt = time.perf_counter() - t0
    value = x.size * args.steps / dt
    return {"metric": FRONTEND_METRIC, "value": value, "unit": "samples/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.workload == "rf2iq" else "c64",
            "data": "synthetic (seeded Gaussian channel samples; no public dataset offline)",
            "config": {"workload": f"{args.workload}: {WORKLOAD_DESC[args.workload]}", "shape_in": [n_s, n_e, n_w, n_f],
                       "parallelism": "rank 0 only, host cores"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": 1, "kind": "reference",
                             "sample": "the whole job per step"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------------------- reference arm


def run_reference(args, world, rank, local):
    from oracle import machref

    if not machref.available():
        return {"impl": "reference", "unavailable": "mach's kernel was not built into oracle/_ref (no reference checkout)"}
    line = measure_reference(args, args.workload, args.storage, world, headline=True)
    names = []
    for name, _ in parse_also(args):
        if name not in names:
            names.append(name)
    if names:
        line["workloads"] = [measure_reference(args, name, None, world, headline=False) for name in names]
    return with_serving(line, run_serving_reference, args, world, rank, local)


def measure_reference(args, name, storage, world, headline):
    """mach's kernel on one workload: float32 / complex64 input (int16 widened exactly, times
    its scale), one launch + cudaDeviceSynchronize per transmit, into a zeroed output."""
    from oracle import machref

    frames, side = (args.frames, args.side) if headline else (None, None)
    w = make_workload(name, frames, side)
    storage = storage or w.storage
    ch = w.channel
    if ch.dtype == torch.int16:
        ch = ch.to(torch.float32) * w.channel_scale
    ch = ch.contiguous()
    is_c = ch.is_complex()
    rx = torch.as_tensor(w.rx_coords_m, device="cuda")
    scan = torch.as_tensor(w.scan_coords_m, device="cuda")
    arr = torch.as_tensor(w.tx_wave_arrivals_s, device="cuda")
    out = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if is_c else torch.float32, device="cuda")
    keys = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
            "interp_type")
    p = {k: w.params[k] for k in keys}
    ch_ptrs = [ch[t].data_ptr() for t in range(w.n_tx)]
    arr_ptrs = [arr[t].data_ptr() for t in range(w.n_tx)]

    def step():
        out.zero_()
        machref.beamform_device(ch_ptrs, rx.data_ptr(), scan.data_ptr(), arr_ptrs, out.data_ptr(), is_complex=is_c,
                                n_rx=w.n_rx, n_samples=w.n_samples, n_vox=w.n_vox, n_frames=w.n_frames, **p)

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lat = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s = time.perf_counter()
        step()
        torch.cuda.synchronize()
        lat.append((time.perf_counter() - s) * 1e3)
    dt = time.perf_counter() - t0
    clock_info = clocks.stop()
    line = {
        "metric": METRIC, "value": w.points * args.steps / dt, "unit": "points/s", "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded simulation of the configuration; no public dataset offline)",
        "config": workload_config(name, w, storage, world),
        "reference": "mach 0.1.3 src/mach/kernel.cu compiled for sm_100a from its unmodified source; one launch + "
                     "cudaDeviceSynchronize per transmit into a zeroed complex64/float32 out (mach.experimental loop); "
                     "rank 0 only",
        "reference_input": "complex64" if is_c else ("float32 (int16 samples x scale, exact)"
                                                     if w.storage == "i16" else "float32"),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "clocks": clock_info,
        "gpu_launches": w.n_tx * args.steps,
    }
    if not args.no_e2e:
        ch_h = ch.cpu().pin_memory()
        rx_h, scan_h = w.rx_coords_m, w.scan_coords_m
        arr_h = np.ascontiguousarray(w.tx_wave_arrivals_s)
        ch_np = ch_h.numpy()
        out_h = torch.zeros_like(out, device="cpu").pin_memory()

        def e2e_step():
            out.zero_()
            machref.beamform_host(ch_np, rx_h, scan_h, arr_h, None, out_on_device_ptr=out.data_ptr(), **p)
            out_h.copy_(out)

        e2e_step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        per_tx = ch_np[0].nbytes + arr_h[0].nbytes + rx_h.nbytes + scan_h.nbytes
        line["e2e"] = {"value": w.points * args.steps / dt, "unit": "points/s",
                       "h2d_bytes_per_step": int(per_tx * w.n_tx),
                       "d2h_bytes_per_step": int(out_h.numel() * 8 if is_c else out_h.numel() * 4),
                       "ms_per_step": dt / args.steps * 1e3,
                       "api": "mach's binding with host arrays per transmit (its CPU staging path), device out"}
        del ch_h, out_h, ch_np
    del ch, out, rx, scan, arr
    w.channel = None
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return line


def main():
    global DELAY_CHOICE
    args = parse_args()
    DELAY_CHOICE = args.delay
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            if rank != 0:
                return
            runner = {"serving": run_serving_reference, "rf2iq": run_frontend_reference,
                      "ingest": run_frontend_reference}.get(args.workload, run_reference)
        else:
            runner = {"serving": run_serving, "rf2iq": run_frontend, "ingest": run_frontend}.get(args.workload, run_ours)
        line = runner(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1 and torch.distributed.is_initialized():
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
