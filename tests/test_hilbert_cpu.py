"""The analytic-signal oracle against scipy (what mach calls, src/mach/io/uff.py:88) and the
committed golden cases; argument errors of mach_b200_hilbert that need no GPU."""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

from oracle import analytic

GOLDEN = Path(__file__).parent / "golden" / "analytic" / "hilbert_cases.npz"
LIB = Path(__file__).resolve().parents[1] / "mach_b200" / "libmach_b200.so"


def test_oracle_matches_golden_scipy_cases():
    g = np.load(GOLDEN)
    lengths = sorted(int(k[2:]) for k in g.files if k.startswith("x_"))
    assert lengths[0] == 1 and 416 in lengths
    for n in lengths:
        np.testing.assert_allclose(analytic.analytic_signal(g[f"x_{n}"], axis=0), g[f"z_{n}"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 5, 6, 97, 128, 1400])
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_oracle_matches_scipy_on_any_axis(n, axis):
    scipy_signal = pytest.importorskip("scipy.signal")
    shape = [3, 4, 2]
    shape[axis] = n
    x = np.random.default_rng(n + axis).normal(size=shape)
    np.testing.assert_allclose(analytic.analytic_signal(x, axis=axis), scipy_signal.hilbert(x, axis=axis), rtol=0,
                               atol=1e-12)


def test_oracle_preprocess_matches_reference_steps():
    scipy_signal = pytest.importorskip("scipy.signal")
    x = np.random.default_rng(7).normal(size=(50, 6, 3, 2))  # (samples, elements, waves, frames)
    want = np.transpose(scipy_signal.hilbert(x, axis=0), (2, 1, 0, 3))
    np.testing.assert_allclose(analytic.preprocess_signal(x), want, rtol=0, atol=1e-12)
    x3 = x[..., 0]
    assert analytic.preprocess_signal(x3).shape == (3, 6, 50, 1)


def _lib():
    lib = ctypes.CDLL(str(LIB))
    lib.mach_b200_last_error.restype = ctypes.c_char_p
    f = lib.mach_b200_hilbert
    U32 = ctypes.c_uint32
    f.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, U32, U32, U32, U32,
                  ctypes.c_float, ctypes.c_void_p, U32]
    f.restype = ctypes.c_int
    return lib


def test_hilbert_rejects_bad_arguments_without_gpu():
    lib = _lib()
    assert lib.mach_b200_hilbert(1, 1, 0, 1, 1, 8, 1, 1, 1, 1.0, None, 0) == 1  # complex source
    assert b"real channel data" in lib.mach_b200_last_error()
    assert lib.mach_b200_hilbert(0, 1, 0, 0, 1, 8, 1, 1, 1, 1.0, None, 0) == 1  # real destination
    assert lib.mach_b200_hilbert(0, 1, 2, 1, 1, 8, 1, 1, 1, 1.0, None, 0) == 1
    assert b"src_layout" in lib.mach_b200_last_error()
    assert lib.mach_b200_hilbert(9, 1, 0, 1, 1, 8, 1, 1, 1, 1.0, None, 0) == 1
    assert b"storage" in lib.mach_b200_last_error()
    assert lib.mach_b200_hilbert(0, 1, 0, 1, 1, 0, 1, 1, 1, 1.0, None, 0) == 0  # nothing to do
    assert lib.mach_b200_hilbert(0, None, 0, 1, 1, 8, 1, 1, 1, 1.0, None, 0) == 1
