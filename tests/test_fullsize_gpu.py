"""Parity on the full-size configurations the benchmark runs (not the shrunken test jobs):
the 75-transmit compounding job, the 200-frame Doppler ensemble and the 128^3 3-D volume with
1 and 16 frames, each on its production shapes and kernels (tile maps, frame chunks, window
sizes, transmit loops).

* FP32-exact storage (complex64, int16 x scale) with mach's FP32 delay arithmetic: relative
  L2 error <= 1e-5 against mach's own kernel (oracle/_ref, built from mach's source) on the
  whole job, and <= -60 dB normalised RMS against the FP64 oracle on a seeded voxel subset;
* FP16 storage (split delays, the API default for it): <= -60 dB against the FP64 oracle run
  on the unrounded source data, on a seeded voxel subset.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu

REL_L2_VS_REFERENCE = 1e-5
NRMS_DB = -60.0


def _needs_ref():
    from oracle import machref

    if not machref.available():
        pytest.skip("reference kernel library not built")


def _workload(name: str, n_frames: int | None = None):
    from mach_b200 import workloads as W

    if name == "volume3d":
        return W.volume3d(n_frames=n_frames or 1, device="cuda")
    return W.CONFIGS[name](device="cuda")


def _subset(n_vox: int, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n_vox, size=min(n, n_vox), replace=False))


def _ours(w, channel, storage, scale, delay):
    """The job through mach_b200.experimental.beamform, device-resident inputs."""
    import torch

    from mach_b200 import experimental

    dev = "cuda"
    out = experimental.beamform(
        channel.to(dev), torch.as_tensor(w.rx_coords_m, device=dev), torch.as_tensor(w.scan_coords_m, device=dev),
        torch.as_tensor(w.tx_wave_arrivals_s, device=dev), channel_scale=scale, delay=delay,
        **{k: w.params[k] for k in H.PARAM_KEYS})
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle_subset(w, channel, storage, scale, sel):
    from oracle import oracle_c

    return oracle_c.beamform_c(H.channel_numpy(channel), w.rx_coords_m, w.scan_coords_m, w.tx_wave_arrivals_s,
                               storage=storage, channel_scale=scale, voxel_subset=sel,
                               **{k: w.params[k] for k in H.PARAM_KEYS})


@pytest.mark.parametrize("name,n_frames", [("compound", None), ("doppler", None), ("volume3d", 1),
                                           ("volume3d", 16)])
def test_full_size_exact_storage_vs_reference_kernel_and_oracle(cuda, name, n_frames):
    _needs_ref()
    w = _workload(name, n_frames)
    got = _ours(w, w.channel, w.storage, w.channel_scale, "reference")
    ref = H.reference_compound(w)
    err = H.rel_l2(got, ref)
    sel = _subset(w.n_vox, 2048 if name == "volume3d" else 4096, seed=17)
    db = H.nrms_db(got[sel], _oracle_subset(w, w.channel, w.storage, w.channel_scale, sel))
    print(f"{name} {w.storage} {w.n_frames} frames: rel L2 vs mach {err:.2e}, {db:.1f} dB vs FP64 oracle")
    assert np.abs(ref).max() > 0
    assert err <= REL_L2_VS_REFERENCE
    assert db <= NRMS_DB


@pytest.mark.parametrize("name,n_frames,storage", [("compound", None, "cf16"), ("doppler", None, "cf16"),
                                                   ("volume3d", 16, "f16")])
def test_full_size_fp16_storage_vs_oracle(cuda, name, n_frames, storage):
    from mach_b200 import workloads as W

    w = _workload(name, n_frames)
    ch, scale = W.as_storage(w, storage)
    got = _ours(w, ch, storage, scale, "split")
    sel = _subset(w.n_vox, 2048 if name == "volume3d" else 4096, seed=23)
    on_source = H.nrms_db(got[sel], _oracle_subset(w, w.channel, w.storage, w.channel_scale, sel))
    on_stored = H.nrms_db(got[sel], _oracle_subset(w, ch, storage, scale, sel))
    print(f"{name} {storage}: {on_source:.1f} dB vs the oracle on the source data, {on_stored:.1f} dB on the "
          f"stored samples")
    assert on_source <= NRMS_DB
    assert on_stored <= NRMS_DB
