"""Channel-data ingest kernel: the rearranged and converted array equals NumPy's
rearrange + cast (src/mach/io/uff.py:70-105) for every storage pair and odd sizes."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REAL = ["f32", "f16", "bf16", "i16"]
CPLX = ["c64", "cf16", "cbf16", "ci16"]


def _source(storage, shape, rng):
    import torch

    x = rng.standard_normal(shape + ((2,) if storage != "f32" and storage in CPLX else ())).astype(np.float32) * 300
    if storage == "f32":
        return torch.as_tensor(x)
    if storage == "c64":
        z = rng.standard_normal(shape).astype(np.float32) * 300 + 1j * rng.standard_normal(shape).astype(np.float32)
        return torch.as_tensor(z.astype(np.complex64))
    t = torch.as_tensor(x)
    if storage in ("f16", "cf16"):
        return t.half()
    if storage in ("bf16", "cbf16"):
        return t.bfloat16()
    return t.round().clamp(-32768, 32767).short()


def _expected(src, dst_storage, scale):
    """float32 value x scale, then the destination's rounding, in acquisition -> beamformer order."""
    import torch

    v = torch.view_as_real(src) if src.is_complex() else src
    v = v.float() * scale
    if v.dim() == 5 or (src.is_complex() and v.dim() == 5):
        v = v.permute(2, 1, 0, 3, 4)
    else:
        v = v.permute(2, 1, 0, 3)
    v = v.contiguous()
    if dst_storage in ("f32", "c64"):
        return torch.view_as_complex(v) if dst_storage == "c64" else v
    if dst_storage in ("f16", "cf16"):
        return v.half()
    if dst_storage in ("bf16", "cbf16"):
        return v.bfloat16()
    return v.round().clamp(-32768, 32767).short()


@pytest.mark.parametrize("src_storage,dst_storage",
                         [(a, b) for a in REAL for b in REAL] + [(a, b) for a in CPLX for b in CPLX])
@pytest.mark.parametrize("frames", [1, 2, 5, 16])
def test_ingest_matches_rearrange_and_cast(cuda, src_storage, dst_storage, frames):
    import torch

    from mach_b200.ingest import ingest

    rng = np.random.default_rng(frames)
    src = _source(src_storage, (37, 5, 3, frames), rng)
    scale = 0.5 if dst_storage.endswith("i16") and not src_storage.endswith("i16") else 1.0
    got = ingest(src.cuda(), dst_storage, scale=scale, complex_pairs=src_storage in CPLX and src_storage != "c64")
    torch.cuda.synchronize()
    want = _expected(src, dst_storage, scale)
    assert got.shape == want.shape and got.dtype == want.dtype
    assert torch.equal(got.cpu(), want)


def test_ingest_from_host_and_three_dims(cuda):
    import torch

    from mach_b200.ingest import ingest

    src = torch.randn(70, 9, 4)
    got = ingest(src, "f16")  # CPU tensor, no frame axis
    torch.cuda.synchronize()
    assert tuple(got.shape) == (4, 9, 70, 1)
    assert torch.equal(got.cpu()[..., 0], src.permute(2, 1, 0).half())


def test_ingest_rejects_mixed_complexity(cuda):
    import torch

    from mach_b200.ingest import ingest

    with pytest.raises(ValueError, match="both be real"):
        ingest(torch.randn(4, 3, 2, 1, device="cuda"), "cf16")
