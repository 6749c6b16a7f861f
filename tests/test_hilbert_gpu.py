"""mach_b200_hilbert (RF -> IQ by the analytic signal) against the FP64 oracle, which is pinned
to scipy.signal.hilbert.  FP32 transforms: tolerance 1e-5 relative L2 for complex64 output."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import analytic
from tests import _helpers as H

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).parent / "golden" / "analytic" / "hilbert_cases.npz"
TOL = 1e-5


def _rf(shape, seed=0):
    return np.random.default_rng(seed).normal(size=shape).astype(np.float32)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 8, 13, 100, 416, 1024, 1031, 1400, 1800, 3328])
@pytest.mark.parametrize("n_frames", [1, 3])
def test_channel_layout_matches_oracle(cuda, n, n_frames):
    import torch

    from mach_b200 import ingest

    x = _rf((2, 5, n, n_frames), seed=n)
    got = ingest.hilbert(torch.as_tensor(x, device="cuda")).cpu().numpy()
    want = analytic.analytic_signal(x, axis=2)
    assert got.dtype == np.complex64 and got.shape == x.shape
    np.testing.assert_array_equal(got.real, x)  # the real part is the input itself
    assert H.rel_l2(got, want) <= TOL


def test_golden_scipy_cases(cuda):
    import torch

    from mach_b200 import ingest

    g = np.load(GOLDEN)
    for key in g.files:
        if not key.startswith("x_"):
            continue
        n = int(key[2:])
        x = g[key][:, :, np.newaxis]  # (n, 3, 1): samples, elements, waves
        got = ingest.hilbert(torch.as_tensor(x, device="cuda"), layout="acquisition").cpu().numpy()
        assert got.shape == (1, 3, n, 1)
        want = g[f"z_{n}"].T[np.newaxis, :, :, np.newaxis]
        assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max()), n


@pytest.mark.parametrize("n_frames", [1, 2, 16])
@pytest.mark.parametrize("src", ["f32", "i16", "f16", "bf16"])
def test_acquisition_layout_fuses_rearrange(cuda, n_frames, src):
    import torch

    from mach_b200 import ingest

    x = _rf((1024, 24, 3, n_frames), seed=n_frames)
    if src == "i16":
        t = torch.as_tensor(np.round(x * 1000).astype(np.int16))
        ref = t.numpy().astype(np.float64) * 1e-3
        scale = 1e-3
    else:
        t = torch.as_tensor(x).to({"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[src])
        ref = t.float().numpy().astype(np.float64)
        scale = 1.0
    got = ingest.preprocess_signal(t.cuda(), 0.0, storage="c64", scale=scale).cpu().numpy()
    want = analytic.preprocess_signal(ref)
    assert got.shape == (3, 24, 1024, n_frames)
    assert H.rel_l2(got, want) <= TOL


@pytest.mark.parametrize("dst", ["cf16", "cbf16", "ci16"])
def test_reduced_complex_storage(cuda, dst):
    import torch

    from mach_b200 import ingest

    x = _rf((2, 8, 1800, 4), seed=3)
    scale = 1000.0 if dst == "ci16" else 1.0
    got = ingest.hilbert(torch.as_tensor(x, device="cuda"), dst, scale=scale)
    assert got.shape == (2, 8, 1800, 4, 2)
    pair = got.float().cpu().numpy() / scale
    z = pair[..., 0] + 1j * pair[..., 1]
    want = analytic.analytic_signal(x, axis=2)
    bound = {"cf16": -60.0, "cbf16": -45.0, "ci16": -55.0}[dst]
    assert H.nrms_db(z, want) <= bound


def test_int16_destination_saturates(cuda):
    import torch

    from mach_b200 import ingest

    x = np.zeros((1, 1, 64, 1), dtype=np.float32)
    x[0, 0, 10, 0] = 1.0
    got = ingest.hilbert(torch.as_tensor(x, device="cuda"), "ci16", scale=1e6).cpu().numpy()
    assert got[0, 0, 10, 0, 0] == 32767
    assert got.min() == -32768 and got.max() == 32767


def test_host_input_and_errors(cuda):
    import torch

    from mach_b200 import ingest

    x = _rf((1, 4, 600, 2), seed=5)
    got = ingest.hilbert(torch.as_tensor(x)).cpu().numpy()  # CPU tensor: staged
    assert H.rel_l2(got, analytic.analytic_signal(x, axis=2)) <= TOL
    with pytest.raises(TypeError):
        ingest.hilbert(torch.zeros((1, 1, 8, 1), dtype=torch.complex64, device="cuda"))
    with pytest.raises(RuntimeError, match="too long"):
        ingest.hilbert(torch.zeros((1, 1, 20000, 1), device="cuda"))


def test_beamform_after_hilbert_matches_oracle(cuda):
    """RF volume -> IQ on the GPU -> beamformed with modulation 0, against the FP64 beamforming
    oracle on the oracle's IQ."""
    import torch

    from mach_b200 import experimental, ingest
    from oracle import oracle_c

    w = H.small("volume3d", n_side=8, n_elem_side=8, n_frames=2)
    rf = (w.channel.to(torch.float32) * w.channel_scale).numpy()  # [n_tx, n_rx, n_s, n_f]
    iq = ingest.hilbert(torch.as_tensor(rf, device="cuda"))
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    p["modulation_freq_hz"] = 0.0
    dev = "cuda"
    got = experimental.beamform(iq, torch.as_tensor(w.rx_coords_m, device=dev),
                                torch.as_tensor(w.scan_coords_m, device=dev),
                                torch.as_tensor(w.tx_wave_arrivals_s, device=dev), **p).cpu().numpy()
    iq_ref = analytic.analytic_signal(rf, axis=2).astype(np.complex64)
    want = oracle_c.beamform_c(iq_ref, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, storage="c64", **p)
    assert np.abs(want).max() > 0
    assert H.nrms_db(got, want) <= -80.0
