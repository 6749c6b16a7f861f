"""GPU parity: the sm_100a kernels against the FP64 oracle and against mach's own kernel.

Bars (from the project's correctness contract):
* FP32 storage (float32 RF / complex64 IQ): relative L2 error <= 1e-5 against mach's
  reference CUDA kernel run on the same inputs (oracle/_ref, built from mach's source);
* every result reports its normalised RMS error against the FP64 oracle; FP32 storage
  must be <= -60 dB there too, and reduced-precision storage <= -60 dB measured against
  the oracle run on the unquantised data (bfloat16 is reported, see test_storage_nrms).
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu

REL_L2_VS_REFERENCE = 1e-5
NRMS_DB_FP32 = -60.0
NRMS_DB_REDUCED = -60.0


def _machref_available() -> bool:
    from oracle import machref

    return machref.available()


needs_ref = pytest.mark.skipif(not _machref_available(), reason="reference kernel library not built")


@pytest.mark.parametrize("name", ["plain2d", "compound", "doppler"])
def test_fp32_vs_oracle(cuda, name):
    w = H.small(name)
    got = H.gpu_compound(w)
    want = H.oracle(w)
    db = H.nrms_db(got, want)
    print(f"{name}: nRMS vs FP64 oracle {db:.1f} dB")
    assert db <= NRMS_DB_FP32


@needs_ref
@pytest.mark.parametrize("name", ["plain2d", "compound", "doppler", "volume3d"])
def test_vs_reference_kernel(cuda, name):
    w = H.small(name)
    ref = H.reference_compound(w)
    if w.storage == "i16":
        import torch

        # mach only takes float32: compare on the widened samples (scale already applied)
        w.channel = w.channel.to(torch.float32) * w.channel_scale
        w.channel_scale = 1.0
        w.storage = "f32"
        got = H.gpu_compound(w)
    else:
        got = H.gpu_compound(w)
    err = H.rel_l2(got, ref)
    print(f"{name}: rel L2 vs reference kernel {err:.3e}")
    assert err <= REL_L2_VS_REFERENCE


@needs_ref
@pytest.mark.parametrize("interp", [0, 1, 2])
@pytest.mark.parametrize("alpha", [0.0, 0.5, 1.0])
@pytest.mark.parametrize("f_number", [1.0, 3.0])
def test_parameter_grid_vs_reference(cuda, interp, alpha, f_number):
    w = H.small("compound", n_x=16, n_z=24, n_tx=3)
    w.params.update(interp_type=interp, tukey_alpha=alpha, f_number=f_number)
    ref = H.reference_compound(w)
    got = H.gpu_compound(w)
    assert H.rel_l2(got, ref) <= REL_L2_VS_REFERENCE


@needs_ref
@pytest.mark.parametrize("n_frames", [1, 2, 3, 8, 9, 16, 17, 33, 70])
def test_frame_counts_vs_reference(cuda, n_frames):
    w = H.small("doppler", n_x=12, n_z=16, n_tx=2, n_frames=n_frames)
    ref = H.reference_compound(w)
    got = H.gpu_compound(w)
    assert H.rel_l2(got, ref) <= REL_L2_VS_REFERENCE


@needs_ref
def test_sample_index_bit_exact(cuda):
    """Ramp data makes the output equal the kernel's FP32 sample index: it must match mach bit for bit."""
    import torch

    rng = np.random.default_rng(7)
    n_s = 4096
    ramp = torch.arange(n_s, dtype=torch.float32).reshape(1, 1, n_s, 1)
    w = H.small("plain2d")
    n_vox = 4096
    scan = np.stack([rng.uniform(-8e-3, 8e-3, n_vox), rng.uniform(-3e-3, 3e-3, n_vox),
                     rng.uniform(20e-3, 60e-3, n_vox)], -1).astype(np.float32)
    w.scan_coords_m = scan
    w.rx_coords_m = np.array([[0.7e-3, -0.2e-3, 0.05e-3]], dtype=np.float32)
    w.tx_wave_arrivals_s = (rng.uniform(10e-3, 60e-3, (1, n_vox)) / 1540.0).astype(np.float32)
    w.channel = ramp
    w.params.update(f_number=0.01, tukey_alpha=0.0, interp_type=1, rx_start_s=1.3e-6, sampling_freq_hz=31.25e6)
    ref = H.reference_compound(w)
    got = H.gpu_compound(w)
    valid = ref[:, 0] != 0
    assert valid.sum() > n_vox // 2
    assert np.array_equal(got[valid, 0], ref[valid, 0])


@pytest.mark.parametrize("storage", ["cf16", "cbf16"])
def test_storage_nrms(cuda, storage):
    """Reduced-precision IQ storage against the oracle on the unquantised complex64 data."""
    from mach_b200 import workloads as W

    w = H.small("compound")
    want = H.oracle(w)
    got = H.gpu_compound(w, channel=W.to_storage(w, storage))
    db = H.nrms_db(got, want)
    exact = H.nrms_db(got, H.oracle(w, channel=W.to_storage(w, storage), storage=storage))
    print(f"{storage}: nRMS {db:.1f} dB end to end, {exact:.1f} dB vs oracle on the stored samples")
    # The arithmetic itself (FP32 delays, mach's fast sincos) stays below -60 dB on any storage;
    # float16 storage meets -60 dB end to end, bfloat16's 8-bit mantissa alone costs ~-53 dB.
    assert exact <= NRMS_DB_REDUCED
    if storage == "cf16":
        assert db <= NRMS_DB_REDUCED
    else:
        assert db <= -50.0


def test_int16_storage_vs_oracle(cuda):
    w = H.small("volume3d")
    got = H.gpu_compound(w)
    want = H.oracle(w)
    db = H.nrms_db(got, want)
    print(f"volume3d int16: nRMS {db:.1f} dB")
    assert db <= NRMS_DB_REDUCED


def test_accumulates_into_device_out(cuda):
    import torch

    from mach_b200 import experimental

    w = H.small("compound", n_x=8, n_z=8, n_tx=2)
    first = H.gpu_compound(w)
    out = torch.as_tensor(first, device="cuda").clone()
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    experimental.beamform(w.channel.to("cuda"), torch.as_tensor(w.rx_coords_m, device="cuda"),
                          torch.as_tensor(w.scan_coords_m, device="cuda"),
                          torch.as_tensor(w.tx_wave_arrivals_s, device="cuda"), out=out, **p)
    assert H.rel_l2(out.cpu().numpy(), 2 * first) <= 1e-6


def test_host_inputs_match_device_inputs(cuda):
    """Host (pageable and pinned) buffers go through the staging path and give the same sums."""
    import torch

    from mach_b200 import experimental

    w = H.small("compound", n_tx=19)
    dev = H.gpu_compound(w)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    for pin in (False, True):
        ch = w.channel.pin_memory() if pin else w.channel
        out = torch.full((w.n_vox, 1), 5.0 + 1j, dtype=torch.complex64)
        with pytest.warns(UserWarning, match="latency"):
            experimental.beamform(ch, w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s, out=out, **p)
        # A CPU `out` is overwritten, not accumulated into (mach semantics).
        assert H.rel_l2(out.numpy(), dev) <= 1e-6


def test_single_transmit_api_matches_compound(cuda):
    import torch

    import mach_b200 as mach

    w = H.small("plain2d")
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    ch = w.channel[0].to("cuda")
    out = mach.beamform(ch, torch.as_tensor(w.rx_coords_m, device="cuda"),
                        torch.as_tensor(w.scan_coords_m, device="cuda"),
                        torch.as_tensor(w.tx_wave_arrivals_s[0], device="cuda"), **p)
    assert out.is_cuda and out.shape == (w.n_vox, 1)
    assert H.rel_l2(out.cpu().numpy(), H.gpu_compound(w)) <= 1e-6


def test_numpy_inputs_single_transmit(cuda):
    import mach_b200 as mach

    w = H.small("plain2d")
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    with pytest.warns(UserWarning, match="latency"):
        out = mach.beamform(w.channel[0].numpy(), w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s[0], **p)
    assert isinstance(out, np.ndarray)
    assert H.nrms_db(out, H.oracle(w)) <= NRMS_DB_FP32


def test_edge_cases(cuda):
    import torch

    from mach_b200 import experimental

    w = H.small("compound", n_x=4, n_z=8, n_tx=2)
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    rx = torch.as_tensor(w.rx_coords_m, device="cuda")
    ch = w.channel.to("cuda")
    # empty scan grid
    out = experimental.beamform(ch, rx, torch.zeros((0, 3), device="cuda"),
                                torch.zeros((2, 0), device="cuda"), **p)
    assert out.shape == (0, 1)
    # voxels at and above the array plane, far outside the recording
    scan = torch.tensor([[0.0, 0.0, 0.0], [1e-3, 0.0, -5e-3], [0.0, 0.0, 1.0]], device="cuda")
    arr = torch.zeros((2, 3), device="cuda")
    out = experimental.beamform(ch, rx, scan, arr, **{**p, "tukey_alpha": 0.0})
    w2 = H.small("compound", n_x=4, n_z=8, n_tx=2)
    w2.scan_coords_m = scan.cpu().numpy()
    w2.tx_wave_arrivals_s = arr.cpu().numpy()
    w2.params["tukey_alpha"] = 0.0
    want = H.oracle(w2)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-4, atol=1e-3)
    # tukey_alpha outside [0, 1] raises with mach's message
    with pytest.raises(RuntimeError, match="tukey_alpha must be in range"):
        experimental.beamform(ch, rx, scan, arr, **{**p, "tukey_alpha": 1.5})
