"""FP64 NumPy oracle for the analytic signal (RF -> IQ at modulation frequency 0).

TEST INFRASTRUCTURE ONLY. Nothing in the ``mach_b200`` product path imports, links or
executes this file; only ``tests/`` use it, as the checker of ``mach_b200_hilbert``.

mach turns real RF into IQ on the host with ``scipy.signal.hilbert(signal, axis=0)``
(src/mach/io/uff.py:86-88; scipy >= 1.13.1, pyproject.toml:43; 1.18.1 is installed here) and
then rearranges ``(n_samples, n_elements, n_waves, n_frames)`` to
``(n_waves, n_elements, n_samples, n_frames)`` (src/mach/io/uff.py:90-102).  scipy's published
algorithm (Marple, IEEE TSP 47(9), 1999): ``X = FFT(x)``; ``h[0] = 1``; ``h[k] = 2`` for
``0 < k < n/2``; ``h[n/2] = 1`` for even ``n``; ``h = 0`` on negative frequencies;
``z = IFFT(h X)``.  Pinned against scipy itself and against ``tests/golden/analytic/hilbert_cases.npz``
(made by ``tests/golden/analytic/make_hilbert_golden.py``).
"""

from __future__ import annotations

import numpy as np


def analytic_signal(x: np.ndarray, axis: int = 0) -> np.ndarray:
    """``scipy.signal.hilbert(x, axis=axis)`` restated in FP64."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[axis]
    h = np.zeros(n)
    if n > 0:
        h[0] = 1.0
        if n % 2 == 0:
            h[n // 2] = 1.0
            h[1:n // 2] = 2.0
        else:
            h[1:(n + 1) // 2] = 2.0
    shape = [1] * x.ndim
    shape[axis] = n
    return np.fft.ifft(np.fft.fft(x, axis=axis) * h.reshape(shape), axis=axis)


def preprocess_signal(signal: np.ndarray) -> np.ndarray:
    """src/mach/io/uff.py:70-105 for modulation frequency 0: the analytic signal along the
    samples of ``(n_samples, n_elements, n_waves[, n_frames])``, then
    ``(n_waves, n_elements, n_samples, n_frames)``."""
    z = analytic_signal(signal, axis=0)
    if z.ndim == 3:
        z = z[..., np.newaxis]
    return np.ascontiguousarray(z.transpose(2, 1, 0, 3))
