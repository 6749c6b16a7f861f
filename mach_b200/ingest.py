"""Channel-data ingest on the GPU: acquisition order to the beamformer's layout.

UFF files and PyMUST hand channel data as ``[n_samples, n_elements, n_waves(, n_frames)]``;
the beamformer wants ``[n_waves, n_elements, n_samples, n_frames]`` in its storage type.
mach rearranges with einops on the host and casts with NumPy (src/mach/io/uff.py:70-105,
examples/doppler.py:193-195).  :func:`ingest` does both in one pass of one kernel
(``mach_b200_ingest``), reading and writing each sample once.
"""

from __future__ import annotations

from typing import Any

from mach_b200 import _cuda_impl

_lib = _cuda_impl._lib

_DTYPES = {  # storage code -> (torch dtype, trailing (I, Q) axis)
    "f32": ("float32", False), "c64": ("complex64", False), "f16": ("float16", False), "cf16": ("float16", True),
    "bf16": ("bfloat16", False), "cbf16": ("bfloat16", True), "i16": ("int16", False), "ci16": ("int16", True),
}


def storage_of_tensor(t, complex_pairs: bool | None = None) -> str:
    """Storage code of a torch tensor in acquisition order.  16-bit data is complex (a trailing
    (I, Q) axis of 2) when ``complex_pairs`` says so, or by default when it has 5 dimensions."""
    name = str(t.dtype).replace("torch.", "")
    if name == "complex64":
        return "c64"
    if name == "float32":
        return "f32"
    codes = {"float16": "f16", "bfloat16": "bf16", "int16": "i16"}
    if name not in codes:
        raise TypeError(f"unsupported channel dtype {t.dtype}")
    pairs = complex_pairs if complex_pairs is not None else t.dim() == 5
    if pairs and t.shape[-1] != 2:
        raise ValueError("16-bit complex data needs a trailing (I, Q) axis of length 2")
    return ("c" + codes[name]) if pairs else codes[name]


def ingest(signal: Any, storage: str | None = None, *, scale: float = 1.0, complex_pairs: bool | None = None,
           out: Any = None, sync: bool = True) -> Any:
    """Rearrange and convert channel data on the GPU.

    Args:
        signal: torch tensor ``[n_samples, n_elements, n_waves]`` or ``[..., n_frames]``
            (float32, complex64, float16, bfloat16, int16), with a trailing ``(I, Q)`` axis of 2
            for 16-bit complex data (say ``complex_pairs=True`` when the shape alone is
            ambiguous).  A CPU tensor is copied to the current GPU.
        storage: destination storage code (``"f32"``, ``"c64"``, ``"f16"``, ``"cf16"``, ``"bf16"``,
            ``"cbf16"``, ``"i16"``, ``"ci16"``); default: the source's.
        scale: every value is multiplied by it before rounding to the destination type
            (int16 destinations saturate).
        out: optional destination tensor ``[n_waves, n_elements, n_samples, n_frames(, 2)]``.

    Returns:
        The channel data in the beamformer's layout, on the GPU.
    """
    import torch

    src = storage_of_tensor(signal, complex_pairs)
    pairs_in = src in ("cf16", "cbf16", "ci16")
    core = signal.shape[:-1] if pairs_in else signal.shape
    if len(core) == 3:
        core = (*core, 1)
    if len(core) != 4:
        raise ValueError("signal must be [n_samples, n_elements, n_waves] or [n_samples, n_elements, n_waves, n_frames]")
    n_s, n_e, n_w, n_f = (int(d) for d in core)
    dst = storage or src
    if dst not in _DTYPES:
        raise ValueError(f"unknown storage {dst!r}")
    if (src in ("c64", "cf16", "cbf16", "ci16")) != (dst in ("c64", "cf16", "cbf16", "ci16")):
        raise ValueError("source and destination must both be real or both be complex")
    dt_name, pairs_out = _DTYPES[dst]
    shape = (n_w, n_e, n_s, n_f) + ((2,) if pairs_out else ())
    if out is None:
        out = torch.empty(shape, dtype=getattr(torch, dt_name), device="cuda")
    elif tuple(out.shape) != shape or not out.is_cuda or not out.is_contiguous():
        raise ValueError(f"out must be a contiguous CUDA tensor of shape {list(shape)}")
    sig = signal.contiguous()
    stream = torch.cuda.current_stream().cuda_stream
    flags = 0 if (sync or not sig.is_cuda) else _cuda_impl.FLAG_ASYNC
    rc = _lib.mach_b200_ingest(_cuda_impl.STORAGE_CODES[src], sig.data_ptr(), _cuda_impl.STORAGE_CODES[dst],
                               out.data_ptr(), n_s, n_e, n_w, n_f, float(scale), stream, flags)
    _cuda_impl._raise_for(rc)
    return out


_COMPLEX_OF = {"f32": "c64", "f16": "cf16", "bf16": "cbf16", "i16": "ci16"}


def hilbert(signal: Any, storage: str | None = None, *, layout: str = "channel", scale: float = 1.0,
            out: Any = None, sync: bool = True) -> Any:
    """RF -> IQ by the analytic signal ``x + i H{x}`` along the samples, on the GPU.

    The result is ``scipy.signal.hilbert(x, axis=samples)``, mach's RF -> IQ step for
    modulation frequency 0 (src/mach/io/uff.py:86-88); beamform it with
    ``modulation_freq_hz=0``.  One kernel (``mach_b200_hilbert``) reads each sample once, runs
    the transforms in shared memory (FP32, exact twiddles) and writes the IQ once.

    Args:
        signal: real torch tensor (float32, float16, bfloat16, int16): ``[n_waves, n_elements,
            n_samples, n_frames]`` for ``layout="channel"``, or the acquisition order
            ``[n_samples, n_elements, n_waves(, n_frames)]`` for ``layout="acquisition"``, which
            also does the rearrange of src/mach/io/uff.py:90-102.  A CPU tensor is copied to
            the current GPU.
        storage: complex destination storage (``"c64"``, ``"cf16"``, ``"cbf16"``, ``"ci16"``);
            default: the complex form of the source's.
        scale: both parts are multiplied by it before rounding (int16 saturates).
        out: optional destination ``[n_waves, n_elements, n_samples, n_frames]`` (complex64) or
            ``[..., 2]`` (16-bit pairs).

    Returns:
        The IQ channel data in the beamformer's layout, on the GPU.
    """
    import torch

    src = storage_of_tensor(signal, complex_pairs=False)
    if src not in _COMPLEX_OF:
        raise TypeError("the analytic signal needs real channel data (float32, float16, bfloat16 or int16)")
    dst = storage or _COMPLEX_OF[src]
    if dst not in ("c64", "cf16", "cbf16", "ci16"):
        raise ValueError(f"storage must be a complex storage code, got {dst!r}")
    if layout not in ("channel", "acquisition"):
        raise ValueError(f"layout must be 'channel' or 'acquisition', got {layout!r}")
    dims = tuple(int(d) for d in signal.shape)
    if layout == "acquisition" and len(dims) == 3:
        dims = (*dims, 1)
    if len(dims) != 4:
        raise ValueError("signal must have 4 dimensions (3 or 4 in the acquisition layout)")
    if layout == "channel":
        n_w, n_e, n_s, n_f = dims
    else:
        n_s, n_e, n_w, n_f = dims
    dt_name, pairs_out = _DTYPES[dst]
    shape = (n_w, n_e, n_s, n_f) + ((2,) if pairs_out else ())
    if out is None:
        out = torch.empty(shape, dtype=getattr(torch, dt_name), device="cuda")
    elif tuple(out.shape) != shape or not out.is_cuda or not out.is_contiguous() or out.dtype != getattr(torch, dt_name):
        raise ValueError(f"out must be a contiguous CUDA {dt_name} tensor of shape {list(shape)}")
    sig = signal.contiguous()
    stream = torch.cuda.current_stream().cuda_stream
    flags = 0 if (sync or not sig.is_cuda) else _cuda_impl.FLAG_ASYNC
    code = _cuda_impl.LAYOUT_CHANNEL if layout == "channel" else _cuda_impl.LAYOUT_ACQUISITION
    rc = _lib.mach_b200_hilbert(_cuda_impl.STORAGE_CODES[src], sig.data_ptr(), code, _cuda_impl.STORAGE_CODES[dst],
                                out.data_ptr(), n_s, n_e, n_w, n_f, float(scale), stream, flags)
    _cuda_impl._raise_for(rc)
    return out


def preprocess_signal(signal_data: Any, modulation_frequency: float, *, storage: str | None = None,
                      scale: float = 1.0, out: Any = None, sync: bool = True) -> Any:
    """src/mach/io/uff.py:70-105 on the GPU: acquisition-order channel data
    ``[n_samples, n_elements, n_waves(, n_frames)]`` to the beamformer's
    ``[n_waves, n_elements, n_samples, n_frames]``.

    With ``modulation_frequency == 0`` real RF becomes IQ through the analytic signal
    (:func:`hilbert`, one kernel for transform and rearrange).  Otherwise the data is taken as
    already demodulated and only rearranged and converted (:func:`ingest`); mach's own
    function reaches an undefined name on that branch (src/mach/io/uff.py:87-91).
    """
    if modulation_frequency == 0:
        return hilbert(signal_data, storage, layout="acquisition", scale=scale, out=out, sync=sync)
    return ingest(signal_data, storage, scale=scale, out=out, sync=sync)
