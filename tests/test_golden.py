"""Golden fixtures produced by mach's own CUDA kernel (tests/golden/make_golden.py).

CPU: pins the FP64 oracle to the reference's outputs (the oracle's semantics -- aperture,
Tukey window, interpolation taps and bounds, IQ rotation sign, compounding -- must agree;
the remaining difference is FP32 rounding inside the reference).
GPU: the sm_100a kernels must reproduce the reference outputs within relative L2 1e-5.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import das_fp64, oracle_c

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))
PARAMS = ("f_number", "rx_start_s", "sampling_freq_hz", "sound_speed_m_s", "modulation_freq_hz", "tukey_alpha",
          "interp_type")
ORACLE_PIN_DB = -60.0

pytestmark = pytest.mark.skipif(not CASES, reason="no golden fixtures generated yet")


def _load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        case = {k: z[k] for k in z.files}
    for k in PARAMS:
        case[k] = case[k].item()
    return case


@pytest.mark.parametrize("name", CASES or ["none"])
def test_oracle_matches_reference_golden(name):
    case = _load(name)
    storage = "c64" if np.iscomplexobj(case["channel"]) else "f32"
    y = oracle_c.beamform_c(case["channel"], case["rx"], case["scan"], case["arrivals"], storage=storage,
                            **{k: case[k] for k in PARAMS})
    db = das_fp64.nrms_db(y, case["ref_out"])
    assert np.abs(case["ref_out"]).max() > 0
    assert db <= ORACLE_PIN_DB, f"{name}: oracle vs reference {db:.1f} dB"
    y_np = das_fp64.beamform_fp64(case["channel"], case["rx"], case["scan"], case["arrivals"],
                                  **{k: case[k] for k in PARAMS})
    assert das_fp64.rel_l2(y_np, y) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES or ["none"])
def test_kernel_matches_reference_golden(name):
    import torch

    from mach_b200 import experimental

    case = _load(name)
    out = experimental.beamform(
        torch.as_tensor(case["channel"]).cuda(), torch.as_tensor(case["rx"]).cuda(),
        torch.as_tensor(case["scan"]).cuda(), torch.as_tensor(case["arrivals"]).cuda(),
        **{k: case[k] for k in PARAMS})
    err = das_fp64.rel_l2(out.cpu().numpy(), case["ref_out"])
    assert err <= 1e-5, f"{name}: rel L2 {err:.2e} vs mach's kernel"
