"""Seeded synthetic beamforming workloads (the benchmark and test configurations).

No public dataset is available offline, so each configuration is simulated:
point scatterers echo a Gaussian-windowed two-cycle pulse at the exact FP64
round-trip delay (transmit arrival + receive path), plus white noise.  RF data
keeps the carrier; IQ data is the analytic baseband echo
``0.5 A env(t - tau) exp(-i 2 pi f0 tau)`` (what demodulation by ``exp(-i 2 pi f0 t)``
and a low-pass filter give), so mach's ``exp(+i 2 pi f0 tau)`` rotation refocuses it.

Configurations (``numpy.random.default_rng(seed)``, seed = configuration index):

* ``plain2d``   -- 128-el linear array, 0.3 mm pitch, f0 5.208 MHz, fs 20.832 MHz, float32 RF
  [1, 128, 2048, 1], 20 scatterers, 256x256 grid x in [-19, 19] mm, z in [5, 45] mm,
  linear interpolation, Hann apodisation (alpha 1) at f# 1.5.
* ``compound``  -- same array, 75 plane waves over [-16, 16] deg, 3328 IQ samples, 20,000
  speckle scatterers N(0,1) + 10 bright points, 512x512 grid over 40 x 50 mm, quadratic
  interpolation, f# 1.75, alpha 0.5 (mach's default), f_mod 5.208 MHz.
* ``doppler``   -- 128 el, f0 5 MHz, fs 20 MHz, 5 plane waves over [-4, 4] deg, 200 frames,
  1024 IQ samples, a 15 mm speckle disk at 20 mm depth rotating 2 rad/s at 1 kHz frame rate,
  256x256 grid, linear interpolation, f# 1.0, alpha 0 (mach's own Doppler benchmark settings).
* ``volume3d``  -- 32x32 matrix array (0.3 mm pitch), f0 3 MHz, fs 12 MHz, 9 diverging waves
  from virtual sources on a 3x3 grid 10 mm behind the array, int16 RF [9, 1024, 2048, F],
  128^3 grid over 20 x 20 x 40 mm, linear interpolation, f# 1.0, alpha 0.5.

Every generator takes size knobs so tests can run reduced versions of the same physics.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from mach_b200 import geometry, wavefront

LINEAR, QUADRATIC, NEAREST = 1, 2, 0


@dataclass
class Workload:
    name: str
    channel: Any  # [n_tx, n_rx, n_samples, n_frames] complex64 / float32 (torch or numpy), or int16
    rx_coords_m: np.ndarray  # [n_rx, 3] float32
    scan_coords_m: np.ndarray  # [n_vox, 3] float32
    tx_wave_arrivals_s: np.ndarray  # [n_tx, n_vox] float32
    params: dict = field(default_factory=dict)
    storage: str = "f32"
    channel_scale: float = 1.0
    grid_shape: tuple = ()

    @property
    def n_tx(self) -> int:
        return int(self.channel.shape[0])

    @property
    def n_rx(self) -> int:
        return int(self.channel.shape[1])

    @property
    def n_samples(self) -> int:
        return int(self.channel.shape[2])

    @property
    def n_frames(self) -> int:
        return int(self.channel.shape[3])

    @property
    def n_vox(self) -> int:
        return int(self.scan_coords_m.shape[0])

    @property
    def points(self) -> int:
        """voxel x channel x transmit x frame."""
        return self.n_vox * self.n_rx * self.n_tx * self.n_frames

    @property
    def is_complex(self) -> bool:
        return self.storage in ("c64", "cf16", "cbf16", "ci16")


def linear_array(n_elements: int, pitch_m: float) -> np.ndarray:
    """Element positions of a linear array along x, centred at 0 (like src/mach/io/must.py:71-88)."""
    x = np.arange(n_elements, dtype=np.float64) * pitch_m
    x -= x.mean()
    return np.stack([x, np.zeros_like(x), np.zeros_like(x)], axis=-1)


def matrix_array(n_side: int, pitch_m: float) -> np.ndarray:
    """n_side x n_side matrix array in the z = 0 plane, row-major over (x, y), centred."""
    c = np.arange(n_side, dtype=np.float64) * pitch_m
    c -= c.mean()
    xx, yy = np.meshgrid(c, c, indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), np.zeros(n_side * n_side)], axis=-1)


def scan_grid(*axes: np.ndarray) -> np.ndarray:
    """Flattened meshgrid, last axis fastest (src/mach/io/must.py:91-104)."""
    return np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, len(axes))


def _torch_device(device: str | None):
    import torch

    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    return torch, torch.device(device)


def _synthesize(
    rx: np.ndarray,
    scatterers_per_frame,  # callable(frame) -> (positions [n, 3] float64, amplitudes [n] float64)
    tx_delay,  # callable(positions [n, 3]) -> [n_tx, n] float64 transmit arrival (s)
    *,
    n_tx: int,
    n_samples: int,
    n_frames: int,
    fs: float,
    f0: float,
    c: float,
    iq: bool,
    noise_std: float,
    rng: np.random.Generator,
    device: str | None,
):
    """Echo synthesis on torch (GPU when available).  Returns [n_tx, n_rx, n_samples, n_frames]."""
    torch, dev = _torch_device(device)
    n_rx = rx.shape[0]
    sigma = 0.5 / f0  # Gaussian window: +-1 cycle at 1/e^2, a two-cycle pulse
    half = int(math.ceil(3.0 * sigma * fs))
    taps = torch.arange(-half, half + 1, device=dev, dtype=torch.float64)
    rx_t = torch.as_tensor(rx, device=dev, dtype=torch.float64)
    cdtype = torch.complex128 if iq else torch.float64
    out = torch.zeros((n_tx, n_rx, n_frames, n_samples), dtype=torch.complex64 if iq else torch.float32, device=dev)
    for f in range(n_frames):
        pos, amp = scatterers_per_frame(f)
        pos_t = torch.as_tensor(pos, device=dev, dtype=torch.float64)
        amp_t = torch.as_tensor(amp, device=dev, dtype=torch.float64)
        t_tx = torch.as_tensor(tx_delay(pos), device=dev, dtype=torch.float64)  # [n_tx, n]
        t_rx = torch.cdist(rx_t, pos_t) / c  # [n_rx, n]
        for t in range(n_tx):
            tau = t_tx[t][None, :] + t_rx  # [n_rx, n]
            centre = torch.floor(tau * fs)
            idx = centre[..., None] + taps  # [n_rx, n, K]
            dt = idx / fs - tau[..., None]
            env = torch.exp(-0.5 * (dt / sigma) ** 2)
            if iq:
                val = (0.5 * amp_t[None, :, None] * env).to(cdtype) * torch.exp(
                    -1j * 2.0 * math.pi * f0 * tau
                )[..., None]
            else:
                val = amp_t[None, :, None] * env * torch.cos(2.0 * math.pi * f0 * dt)
            inb = (idx >= 0) & (idx < n_samples)
            flat = (torch.arange(n_rx, device=dev)[:, None, None] * n_samples + idx.long()).masked_select(inb)
            sig = torch.zeros(n_rx * n_samples, dtype=cdtype, device=dev)
            sig.index_add_(0, flat, val.masked_select(inb))
            out[t, :, f, :] = sig.view(n_rx, n_samples).to(out.dtype)
    if noise_std > 0:
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(rng.integers(2**62)))
        if iq:
            noise = torch.randn(out.shape, generator=gen, device=dev, dtype=torch.float32) + 1j * torch.randn(
                out.shape, generator=gen, device=dev, dtype=torch.float32
            )
            out += (noise_std / math.sqrt(2.0)) * noise.to(torch.complex64)
        else:
            out += noise_std * torch.randn(out.shape, generator=gen, device=dev, dtype=torch.float32)
    return out.permute(0, 1, 3, 2).contiguous()  # -> [n_tx, n_rx, n_samples, n_frames]


def _plane_arrivals(scan: np.ndarray, angles_rad: np.ndarray, c: float) -> np.ndarray:
    dirs = geometry.ultrasound_angles_to_cartesian(angles_rad, np.zeros_like(angles_rad))
    return np.stack([wavefront.plane(np.zeros(3), scan, d) / c for d in dirs])  # float64


def plain2d(*, n_x: int = 256, n_z: int = 256, n_elements: int = 128, n_samples: int = 2048,
            seed: int = 0, device: str | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    f0, fs, c = 5.208e6, 20.832e6, 1540.0
    rx = linear_array(n_elements, 0.3e-3)
    xs = np.linspace(-19e-3, 19e-3, n_x)
    zs = np.linspace(5e-3, 45e-3, n_z)
    scan = scan_grid(xs, np.zeros(1), zs)
    pos = np.stack([rng.uniform(-19e-3, 19e-3, 20), np.zeros(20), rng.uniform(5e-3, 45e-3, 20)], axis=-1)
    amp = np.ones(20)
    angles = np.zeros(1)
    ch = _synthesize(rx, lambda f: (pos, amp), lambda p: _plane_arrivals(p, angles, c), n_tx=1,
                     n_samples=n_samples, n_frames=1, fs=fs, f0=f0, c=c, iq=False, noise_std=0.01, rng=rng,
                     device=device)
    arrivals = _plane_arrivals(scan, angles, c)
    return Workload(
        "plain2d", ch, rx.astype(np.float32), scan.astype(np.float32), arrivals.astype(np.float32),
        dict(f_number=1.5, rx_start_s=0.0, sampling_freq_hz=fs, sound_speed_m_s=c, modulation_freq_hz=0.0,
             tukey_alpha=1.0, interp_type=LINEAR), "f32", 1.0, (n_x, n_z),
    )


def compound(*, n_x: int = 512, n_z: int = 512, n_tx: int = 75, n_elements: int = 128, n_samples: int = 3328,
             n_speckle: int = 20000, seed: int = 1, device: str | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    f0, fs, c = 5.208e6, 20.832e6, 1540.0
    rx = linear_array(n_elements, 0.3e-3)
    xs = np.linspace(-20e-3, 20e-3, n_x)
    zs = np.linspace(5e-3, 55e-3, n_z)
    scan = scan_grid(xs, np.zeros(1), zs)
    spk = np.stack([rng.uniform(-20e-3, 20e-3, n_speckle), np.zeros(n_speckle), rng.uniform(5e-3, 55e-3, n_speckle)], -1)
    bright = np.stack([rng.uniform(-15e-3, 15e-3, 10), np.zeros(10), rng.uniform(10e-3, 50e-3, 10)], -1)
    pos = np.concatenate([spk, bright])
    amp = np.concatenate([rng.standard_normal(n_speckle), np.full(10, 30.0)])
    angles = np.deg2rad(np.linspace(-16.0, 16.0, n_tx))
    ch = _synthesize(rx, lambda f: (pos, amp), lambda p: _plane_arrivals(p, angles, c), n_tx=n_tx,
                     n_samples=n_samples, n_frames=1, fs=fs, f0=f0, c=c, iq=True, noise_std=0.01, rng=rng,
                     device=device)
    arrivals = _plane_arrivals(scan, angles, c)
    return Workload(
        "compound", ch, rx.astype(np.float32), scan.astype(np.float32), arrivals.astype(np.float32),
        dict(f_number=1.75, rx_start_s=0.0, sampling_freq_hz=fs, sound_speed_m_s=c, modulation_freq_hz=f0,
             tukey_alpha=0.5, interp_type=QUADRATIC), "c64", 1.0, (n_x, n_z),
    )


def doppler(*, n_x: int = 256, n_z: int = 256, n_tx: int = 5, n_frames: int = 200, n_elements: int = 128,
            n_samples: int = 1024, n_scatterers: int = 3000, seed: int = 2, device: str | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    f0, fs, c = 5.0e6, 20.0e6, 1540.0
    rx = linear_array(n_elements, 0.3e-3)
    xs = np.linspace(-16e-3, 16e-3, n_x)
    zs = np.linspace(4e-3, 36e-3, n_z)
    scan = scan_grid(xs, np.zeros(1), zs)
    radius, cz = 15e-3, 20e-3
    r = radius * np.sqrt(rng.uniform(0, 1, n_scatterers))
    th = rng.uniform(0, 2 * np.pi, n_scatterers)
    amp = rng.standard_normal(n_scatterers)
    omega_per_frame = 2.0 / 1000.0  # 2 rad/s at 1 kHz

    def at_frame(f: int):
        a = th + omega_per_frame * f
        return np.stack([r * np.cos(a), np.zeros_like(r), cz + r * np.sin(a)], -1), amp

    angles = np.deg2rad(np.linspace(-4.0, 4.0, n_tx))
    ch = _synthesize(rx, at_frame, lambda p: _plane_arrivals(p, angles, c), n_tx=n_tx, n_samples=n_samples,
                     n_frames=n_frames, fs=fs, f0=f0, c=c, iq=True, noise_std=0.01, rng=rng, device=device)
    arrivals = _plane_arrivals(scan, angles, c)
    return Workload(
        "doppler", ch, rx.astype(np.float32), scan.astype(np.float32), arrivals.astype(np.float32),
        dict(f_number=1.0, rx_start_s=0.0, sampling_freq_hz=fs, sound_speed_m_s=c, modulation_freq_hz=f0,
             tukey_alpha=0.0, interp_type=LINEAR), "c64", 1.0, (n_x, n_z),
    )


def volume3d(*, n_side: int = 128, n_frames: int = 1, n_elem_side: int = 32, n_samples: int = 2048,
             n_scatterers: int = 200, seed: int = 3, device: str | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    f0, fs, c = 3.0e6, 12.0e6, 1540.0
    rx = matrix_array(n_elem_side, 0.3e-3)
    xs = np.linspace(-10e-3, 10e-3, n_side)
    zs = np.linspace(5e-3, 45e-3, n_side)
    scan = scan_grid(xs, xs, zs)
    pos = np.stack([rng.uniform(-10e-3, 10e-3, n_scatterers), rng.uniform(-10e-3, 10e-3, n_scatterers),
                    rng.uniform(5e-3, 45e-3, n_scatterers)], -1)
    amp = rng.standard_normal(n_scatterers)
    sources = [np.array([sx, sy, -10e-3]) for sx in (-3e-3, 0.0, 3e-3) for sy in (-3e-3, 0.0, 3e-3)]

    def tx_delay(p):
        return np.stack([wavefront.spherical(np.zeros(3), p, s) / c for s in sources])

    ch = _synthesize(rx, lambda f: (pos, amp), tx_delay, n_tx=len(sources), n_samples=n_samples,
                     n_frames=n_frames, fs=fs, f0=f0, c=c, iq=False, noise_std=0.05, rng=rng, device=device)
    # ADC-style int16 samples: full scale at 4x the peak echo.
    peak = float(ch.abs().max())
    scale = 4.0 * peak / 32767.0
    import torch

    ch = (ch / scale).round().clamp(-32768, 32767).to(torch.int16)
    arrivals = tx_delay(scan)
    return Workload(
        "volume3d", ch, rx.astype(np.float32), scan.astype(np.float32), arrivals.astype(np.float32),
        dict(f_number=1.0, rx_start_s=0.0, sampling_freq_hz=fs, sound_speed_m_s=c, modulation_freq_hz=0.0,
             tukey_alpha=0.5, interp_type=LINEAR), "i16", scale, (n_side, n_side, n_side),
    )


def to_storage(w: Workload, storage: str):
    """Channel data of ``w`` converted to a reduced-precision storage format (torch tensor)."""
    import torch

    ch = w.channel
    if storage == w.storage:
        return ch
    if storage in ("cf16", "cbf16"):
        dt = torch.float16 if storage == "cf16" else torch.bfloat16
        return torch.view_as_real(ch.to(torch.complex64)).to(dt).contiguous()
    if storage in ("f16", "bf16"):
        return ch.to(torch.float16 if storage == "f16" else torch.bfloat16).contiguous()
    raise ValueError(f"no conversion from {w.storage} to {storage}")


def as_storage(w: Workload, storage: str):
    """``(channel, channel_scale)`` of ``w`` in ``storage``; int16 storage is scaled to use
    the range +-20000 (real RF keeps its own ADC scale when it already is int16)."""
    import torch

    if storage == w.storage:
        return w.channel, w.channel_scale
    if storage in ("ci16", "i16"):
        x = w.channel
        if x.dtype == torch.int16:
            x = x.to(torch.float32) * w.channel_scale
        x = torch.view_as_real(x.to(torch.complex64)) if storage == "ci16" else x.to(torch.float32)
        scale = float(x.abs().max()) / 20000.0 or 1.0
        return (x / scale).round().clamp(-32768, 32767).to(torch.int16).contiguous(), scale
    ch = w.channel
    if ch.dtype == torch.int16:
        ch = ch.to(torch.float32) * w.channel_scale
        w = Workload(w.name, ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, w.params, "f32", 1.0)
    return to_storage(w, storage), 1.0


CONFIGS = {"plain2d": plain2d, "compound": compound, "doppler": doppler, "volume3d": volume3d}
