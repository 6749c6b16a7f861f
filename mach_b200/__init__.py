"""B200-native delay-and-sum ultrasound beamforming, a drop-in for ``mach``.

Same public surface as mach (src/mach/__init__.py:17-31): ``beamform``, ``kernel``,
``experimental``, ``wavefront``, ``geometry``, ``Array``.  ``import mach_b200 as mach``
is enough for code written against mach's API.  The beamformer runs in hand-written
sm_100a CUDA kernels in ``libmach_b200.so`` (C ABI: ``include/mach_b200.h``).

The submodules are imported on first use, so that host-only helpers (``geometry``,
``wavefront``, ``workloads``) can be used without opening the CUDA library.  The first
use of anything that beamforms loads the library and raises ``ImportError`` if it is
missing; there is no fallback.
"""

from __future__ import annotations

import importlib

__version__ = "0.2.0"

# public name -> (submodule, attribute or None for the submodule itself)
_LAZY = {
    "Array": ("_array_api", "Array"),
    "InterpolationType": ("_cuda_impl", "InterpolationType"),
    "beamform": ("kernel", "beamform"),
    "experimental": ("experimental", None),
    "geometry": ("geometry", None),
    "kernel": ("kernel", None),
    "wavefront": ("wavefront", None),
}

__all__ = [
    "Array",
    "InterpolationType",
    "__version__",
    "beamform",
    "experimental",
    "geometry",
    "kernel",
    "wavefront",
]


def __getattr__(name: str):
    try:
        module, attr = _LAZY[name]
    except KeyError:
        raise AttributeError(f"module 'mach_b200' has no attribute {name!r}") from None
    mod = importlib.import_module(f"mach_b200.{module}")
    value = mod if attr is None else getattr(mod, attr)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_LAZY))
