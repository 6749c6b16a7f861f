"""Shared helpers for the parity tests: run the CUDA path, the oracle and the reference kernel."""

from __future__ import annotations

import numpy as np

from mach_b200 import workloads as W
from oracle import das_fp64, oracle_c

PARAM_KEYS = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
              "interp_type")


def small(name: str, **over):
    """Reduced-size versions of the benchmark configurations (same physics, oracle-friendly sizes)."""
    base = {
        "plain2d": dict(n_x=48, n_z=64, n_elements=64, n_samples=1200),
        "compound": dict(n_x=40, n_z=48, n_tx=6, n_elements=64, n_samples=1800, n_speckle=1500),
        "doppler": dict(n_x=24, n_z=32, n_tx=3, n_frames=40, n_elements=64, n_samples=1024, n_scatterers=400),
        "volume3d": dict(n_side=12, n_elem_side=12, n_frames=4, n_samples=1400, n_scatterers=40),
    }[name]
    base.update(over)
    return W.CONFIGS[name](device="cpu", **base)


def channel_numpy(ch):
    """numpy view of a (torch) channel tensor in its storage layout (trailing (I, Q) for pairs)."""
    import torch

    if isinstance(ch, torch.Tensor):
        if ch.dtype == torch.bfloat16:
            return ch.view(torch.int16).cpu().numpy().view(np.uint16)
        if ch.dtype == torch.float16:
            return ch.cpu().numpy()
        return ch.cpu().numpy()
    return np.asarray(ch)


def oracle(w: W.Workload, channel=None, storage: str | None = None, voxel_subset=None) -> np.ndarray:
    """FP64 C oracle on the exact samples the GPU sees."""
    ch = channel_numpy(w.channel if channel is None else channel)
    storage = storage or w.storage
    return oracle_c.beamform_c(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, storage=storage,
                               channel_scale=w.channel_scale, voxel_subset=voxel_subset,
                               **{k: w.params[k] for k in PARAM_KEYS})


def gpu_compound(w: W.Workload, channel=None, device="cuda", interp_type=None, **kw) -> np.ndarray:
    """mach_b200.experimental.beamform on device-resident torch tensors."""
    import torch

    from mach_b200 import experimental

    ch = (w.channel if channel is None else channel).to(device)
    p = {k: w.params[k] for k in PARAM_KEYS}
    if interp_type is not None:
        p["interp_type"] = interp_type
    out = experimental.beamform(
        ch, torch.as_tensor(w.rx_coords_m, device=device), torch.as_tensor(w.scan_coords_m, device=device),
        torch.as_tensor(w.tx_wave_arrivals_s, device=device), channel_scale=w.channel_scale, **p, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def reference_compound(w: W.Workload, device="cuda") -> np.ndarray:
    """mach's own CUDA kernel (oracle/_ref), one launch per transmit, float32 / complex64 input."""
    import torch

    from oracle import machref

    ch = w.channel
    if ch.dtype == torch.int16:
        ch = ch.to(torch.float32) * w.channel_scale
    ch = ch.to(device).contiguous()
    rx = torch.as_tensor(w.rx_coords_m, device=device).contiguous()
    scan = torch.as_tensor(w.scan_coords_m, device=device).contiguous()
    arr = torch.as_tensor(w.tx_wave_arrivals_s, device=device).contiguous()
    is_c = ch.is_complex()
    out = torch.zeros((w.n_vox, w.n_frames), dtype=torch.complex64 if is_c else torch.float32, device=device)
    machref.beamform_device(
        [ch[t].data_ptr() for t in range(w.n_tx)], rx.data_ptr(), scan.data_ptr(),
        [arr[t].data_ptr() for t in range(w.n_tx)], out.data_ptr(), is_complex=is_c, n_rx=w.n_rx,
        n_samples=w.n_samples, n_vox=w.n_vox, n_frames=w.n_frames, **{k: w.params[k] for k in PARAM_KEYS},
    )
    torch.cuda.synchronize()
    return out.cpu().numpy()


nrms_db = das_fp64.nrms_db
rel_l2 = das_fp64.rel_l2
