"""B200-native delay-and-sum ultrasound beamforming, a drop-in for ``mach``.

Same public surface as mach (src/mach/__init__.py:17-31): ``beamform``, ``kernel``,
``experimental``, ``wavefront``, ``geometry``, ``Array``.  ``import mach_b200 as mach``
is enough for code written against mach's API.  The beamformer runs in hand-written
sm_100a CUDA kernels in ``libmach_b200.so`` (C ABI: ``include/mach_b200.h``).
"""

from mach_b200 import experimental, geometry, kernel, wavefront
from mach_b200._array_api import Array
from mach_b200._cuda_impl import InterpolationType
from mach_b200.kernel import beamform

__version__ = "0.1.0"

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
