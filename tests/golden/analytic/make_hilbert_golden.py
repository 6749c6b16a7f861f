"""Generate tests/golden/analytic/hilbert_cases.npz: scipy.signal.hilbert on seeded real columns.

scipy.signal.hilbert is what mach calls for RF -> IQ (src/mach/io/uff.py:88).  Run from the
repository root:  python tests/golden/analytic/make_hilbert_golden.py
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import scipy
import scipy.signal

LENGTHS = (1, 2, 3, 7, 8, 12, 13, 30, 64, 100, 416)


def main() -> None:
    rng = np.random.default_rng(20250)
    out = {"scipy_version": np.array(scipy.__version__)}
    for n in LENGTHS:
        x = rng.normal(size=(n, 3)).astype(np.float32)  # 3 columns, samples on axis 0
        out[f"x_{n}"] = x
        out[f"z_{n}"] = scipy.signal.hilbert(x.astype(np.float64), axis=0)
    np.savez_compressed(Path(__file__).with_name("hilbert_cases.npz"), **out)


if __name__ == "__main__":
    main()
