"""Generate the golden fixtures: mach's own CUDA kernel run on small seeded inputs.

mach ships no value-level golden vectors and has no CPU implementation, so the fixtures
are produced by the reference kernel itself -- ``src/mach/kernel.cu`` compiled from its
unmodified source into ``oracle/_ref/libmachref.so`` (see ``oracle/build.py``) -- driven
exactly like ``mach.experimental.beamform`` (one launch per transmit into one output).

Needs a CUDA GPU.  Usage: ``python tests/golden/make_golden.py [out_dir]``
(default: this directory).  Each case is one ``<name>.npz`` holding the inputs, the
parameters and ``ref_out``.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))


def _linear(n, pitch):
    x = (np.arange(n) - (n - 1) / 2) * pitch
    return np.stack([x, np.zeros(n), np.zeros(n)], -1)


def _grid(xs, ys, zs):
    return np.stack(np.meshgrid(xs, ys, zs, indexing="ij"), -1).reshape(-1, 3)


def _plane(scan, angle, c):
    d = np.array([np.sin(angle), 0.0, np.cos(angle)])
    return scan @ d / c


def cases():
    c = 1540.0
    rng = np.random.default_rng(1234)
    out = {}

    # 1. RF, linear, Hann (alpha 1) at f# 1.5, one transmit, one frame
    rx = _linear(32, 0.3e-3)
    scan = _grid(np.linspace(-4e-3, 4e-3, 16), [0.0], np.linspace(8e-3, 20e-3, 20))
    out["rf_linear_hann"] = dict(
        channel=rng.standard_normal((1, 32, 600, 1)).astype(np.float32), rx=rx, scan=scan,
        arrivals=_plane(scan, 0.0, c)[None], f_number=1.5, rx_start_s=0.0, sampling_freq_hz=20.832e6,
        sound_speed_m_s=c, modulation_freq_hz=0.0, tukey_alpha=1.0, interp_type=1)

    # 2. IQ, quadratic, 3 steered plane waves compounded, alpha 0.5, f# 1.75
    rx = _linear(16, 0.3e-3)
    scan = _grid(np.linspace(-3e-3, 3e-3, 12), [0.0], np.linspace(6e-3, 14e-3, 16))
    ch = (rng.standard_normal((3, 16, 600, 1)) + 1j * rng.standard_normal((3, 16, 600, 1))).astype(np.complex64)
    out["iq_quadratic_compound"] = dict(
        channel=ch, rx=rx, scan=scan, arrivals=np.stack([_plane(scan, a, c) for a in np.deg2rad([-10, 0, 10])]),
        f_number=1.75, rx_start_s=0.0, sampling_freq_hz=20.832e6, sound_speed_m_s=c, modulation_freq_hz=5.208e6,
        tukey_alpha=0.5, interp_type=2)

    # 3. IQ, linear, 10 frames, 2 transmits, no apodization, non-zero rx_start
    rx = _linear(8, 0.3e-3)
    scan = _grid(np.linspace(-1e-3, 1e-3, 6), [0.0], np.linspace(4e-3, 8e-3, 10))
    ch = (rng.standard_normal((2, 8, 256, 10)) + 1j * rng.standard_normal((2, 8, 256, 10))).astype(np.complex64)
    out["iq_linear_frames"] = dict(
        channel=ch, rx=rx, scan=scan, arrivals=np.stack([_plane(scan, a, c) for a in np.deg2rad([-3, 3])]),
        f_number=1.0, rx_start_s=1.5e-6, sampling_freq_hz=20e6, sound_speed_m_s=c, modulation_freq_hz=5e6,
        tukey_alpha=0.0, interp_type=1)

    # 4. RF, nearest neighbour, 3 frames, alpha 0.5
    rx = _linear(16, 0.3e-3)
    scan = _grid(np.linspace(-2e-3, 2e-3, 8), [0.0], np.linspace(5e-3, 12e-3, 12))
    out["rf_nearest_frames"] = dict(
        channel=rng.standard_normal((1, 16, 500, 3)).astype(np.float32), rx=rx, scan=scan,
        arrivals=_plane(scan, 0.0, c)[None], f_number=1.0, rx_start_s=0.0, sampling_freq_hz=20e6,
        sound_speed_m_s=c, modulation_freq_hz=0.0, tukey_alpha=0.5, interp_type=0)

    # 5. 3-D: 8x8 matrix array, 2 diverging waves, 2 frames, linear, alpha 0.5
    side = (np.arange(8) - 3.5) * 0.3e-3
    xx, yy = np.meshgrid(side, side, indexing="ij")
    rx = np.stack([xx.ravel(), yy.ravel(), np.zeros(64)], -1)
    scan = _grid(np.linspace(-1e-3, 1e-3, 5), np.linspace(-1e-3, 1e-3, 5), np.linspace(3e-3, 6e-3, 8))
    arrivals = []
    for sx in (-1e-3, 1e-3):
        src = np.array([sx, 0.0, -5e-3])
        arrivals.append((np.linalg.norm(src) * -1.0 + np.linalg.norm(scan - src, axis=-1)) / c)
    out["rf3d_diverging"] = dict(
        channel=rng.standard_normal((2, 64, 256, 2)).astype(np.float32), rx=rx, scan=scan,
        arrivals=np.stack(arrivals), f_number=1.0, rx_start_s=0.0, sampling_freq_hz=12e6, sound_speed_m_s=c,
        modulation_freq_hz=0.0, tukey_alpha=0.5, interp_type=1)
    for case in out.values():
        case["rx"] = np.ascontiguousarray(case["rx"], dtype=np.float32)
        case["scan"] = np.ascontiguousarray(case["scan"], dtype=np.float32)
        case["arrivals"] = np.ascontiguousarray(case["arrivals"], dtype=np.float32)
    return out


PARAMS = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
          "interp_type")


def run_reference(case) -> np.ndarray:
    import torch

    from oracle import machref

    ch = torch.as_tensor(case["channel"]).cuda().contiguous()
    rx = torch.as_tensor(case["rx"]).cuda()
    scan = torch.as_tensor(case["scan"]).cuda()
    arr = torch.as_tensor(case["arrivals"]).cuda()
    n_tx, n_rx, n_s, n_f = ch.shape
    out = torch.zeros((scan.shape[0], n_f), dtype=ch.dtype, device="cuda")
    machref.beamform_device([ch[t].data_ptr() for t in range(n_tx)], rx.data_ptr(), scan.data_ptr(),
                            [arr[t].data_ptr() for t in range(n_tx)], out.data_ptr(), is_complex=ch.is_complex(),
                            n_rx=n_rx, n_samples=n_s, n_vox=scan.shape[0], n_frames=n_f,
                            **{k: case[k] for k in PARAMS})
    torch.cuda.synchronize()
    return out.cpu().numpy()


def main(out_dir: Path) -> None:
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, case in cases().items():
        ref = run_reference(case)
        np.savez(out_dir / f"{name}.npz", ref_out=ref, **case)
        print(name, ref.shape, float(np.abs(ref).max()))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
