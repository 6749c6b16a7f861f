"""mach_b200_beamform_ensemble_noalloc: the ensemble kernel without any GPU allocation.

Some hosts cannot let a library allocate GPU memory: a process whose own allocator has
reserved all of HBM, or a real-time acquisition loop where a memory pool that grows inside a
call could stall it.  This entry point keeps the kernel's scratch (its work-item counters) in
a static device array of the library.  The tests call it through the C ABI, twice in a row on
the same output, and compare each image with mach_b200_beamform_ex (which allocates its
counters per call) on the same job and with the FP64 oracle.  Around the two calls they check
that no memory was taken: the high-water marks of the process's default CUDA memory pool and
of the library's own pool do not move, neither pool reserves more, and torch's allocator holds
the same bytes.

The file name makes pytest collect it last.
"""

from __future__ import annotations

import ctypes

import pytest

from tests import _helpers as H

pytestmark = pytest.mark.gpu


def _bind():
    from mach_b200 import _cuda_impl

    lib = _cuda_impl._lib
    fn = lib.mach_b200_beamform_ensemble_noalloc
    fn.argtypes = list(lib.mach_b200_beamform_ex.argtypes)
    fn.restype = ctypes.c_int
    return lib, fn


class _MemoryWatch:
    """High-water marks and reservations of the default pool (CUDA runtime) and of the
    library's pool (mach_b200_pool_stats), plus torch's allocated bytes."""

    def __init__(self, lib):
        import torch
        from cuda.bindings import runtime as rt

        self.lib, self.rt, self.torch = lib, rt, torch
        self.dev = torch.cuda.current_device()
        err, self.pool = rt.cudaDeviceGetDefaultMemPool(self.dev)
        assert err == rt.cudaError_t.cudaSuccess, err

    def _default(self, reset):
        rt = self.rt
        if reset:
            from cuda.bindings import driver

            res = rt.cudaMemPoolSetAttribute(self.pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                             driver.cuuint64_t(0))
            err = res[0] if isinstance(res, tuple) else res
            assert err == rt.cudaError_t.cudaSuccess, err
        err, high = rt.cudaMemPoolGetAttribute(self.pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)
        assert err == rt.cudaError_t.cudaSuccess, err
        err, reserved = rt.cudaMemPoolGetAttribute(self.pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
        assert err == rt.cudaError_t.cudaSuccess, err
        return int(high), int(reserved)

    def _library(self, reset):
        high, reserved = ctypes.c_uint64(0), ctypes.c_uint64(0)
        rc = self.lib.mach_b200_pool_stats(self.dev, int(reset), ctypes.byref(high), ctypes.byref(reserved))
        assert rc == 0, self.lib.mach_b200_last_error()
        return high.value, reserved.value

    def start(self):
        self.torch.cuda.synchronize()
        self.before = (self._default(True), self._library(True), self.torch.cuda.memory_allocated(),
                       self.torch.cuda.memory_reserved())

    def check(self):
        self.torch.cuda.synchronize()
        (d_high, d_res), (l_high, l_res), t_alloc, t_res = self.before
        assert self._default(False) == (d_high, d_res), "the default memory pool grew"
        assert self._library(False) == (l_high, l_res), "the library's memory pool was used"
        assert self.torch.cuda.memory_allocated() == t_alloc
        assert self.torch.cuda.memory_reserved() == t_res


def _job(storage: str, interp: int = 1):
    import torch

    from mach_b200 import workloads as W

    w = H.small("doppler", n_x=16, n_z=32, n_tx=3, n_frames=64)
    ch, scale = W.as_storage(w, storage)
    dev = "cuda"
    t = {
        "channel": ch.contiguous().to(dev),
        "rx": torch.as_tensor(w.rx_coords_m, device=dev).contiguous(),
        "scan": torch.as_tensor(w.scan_coords_m, device=dev).contiguous(),
        "arr": torch.as_tensor(w.tx_wave_arrivals_s, device=dev).contiguous(),
    }
    p = {k: w.params[k] for k in H.PARAM_KEYS}
    p["interp_type"] = interp
    return w, t, p, scale


def _call(fn, storage, w, t, p, scale, out, options):
    import torch

    from mach_b200 import _cuda_impl

    n_tx, n_rx, n_s, n_f = (int(d) for d in t["channel"].shape[:4])
    return fn(_cuda_impl.STORAGE_CODES[storage], t["channel"].data_ptr(), t["rx"].data_ptr(), t["scan"].data_ptr(),
              t["arr"].data_ptr(), out.data_ptr(), n_tx, n_rx, n_s, w.n_vox, n_f, p["f_number"], p["rx_start_s"],
              p["sampling_freq_hz"], p["sound_speed_m_s"], p["modulation_freq_hz"], p["tukey_alpha"],
              p["interp_type"], scale, torch.cuda.current_stream().cuda_stream, ctypes.byref(options))


@pytest.mark.parametrize("storage", ["c64", "cf16", "i16"])
@pytest.mark.parametrize("interp", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(cuda, storage, interp):
    import torch

    from mach_b200 import _cuda_impl, _grid

    lib, fn = _bind()
    lib.mach_b200_pool_stats.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64),
                                         ctypes.POINTER(ctypes.c_uint64)]
    lib.mach_b200_pool_stats.restype = ctypes.c_int
    if storage == "i16":  # real RF: a frame pair per lane
        w = H.small("volume3d", n_side=8, n_elem_side=8, n_frames=64)
        ch, scale = w.channel, w.channel_scale
        dev = "cuda"
        t = {"channel": ch.contiguous().to(dev), "rx": torch.as_tensor(w.rx_coords_m, device=dev),
             "scan": torch.as_tensor(w.scan_coords_m, device=dev),
             "arr": torch.as_tensor(w.tx_wave_arrivals_s, device=dev)}
        p = {k: w.params[k] for k in H.PARAM_KEYS}
        p["interp_type"] = interp
        dtype = torch.float32
    else:
        w, t, p, scale = _job(storage, interp)
        dtype = torch.complex64
    opts = _cuda_impl.make_options(_cuda_impl.FLAG_OVERWRITE, grid_shape=_grid.detect(t["scan"]), kernel="ensemble")
    shape = (w.n_vox, int(t["channel"].shape[3]))
    want = torch.zeros(shape, dtype=dtype, device="cuda")
    assert _call(lib.mach_b200_beamform_ex, storage, w, t, p, scale, want, opts) == 0, lib.mach_b200_last_error()
    got = torch.full(shape, 7.0, dtype=dtype, device="cuda")
    w.params["interp_type"] = interp
    w.channel_scale = scale
    oracle = H.oracle(w, channel=t["channel"].cpu(), storage=storage)
    watch = _MemoryWatch(lib)
    for _ in range(2):  # the second call must find its counters zeroed again
        launches = lib.mach_b200_launch_count()
        watch.start()
        assert _call(fn, storage, w, t, p, scale, got, opts) == 0, lib.mach_b200_last_error()
        watch.check()
        assert lib.mach_b200_launch_count() == launches + 1
        a, b = got.cpu().numpy(), want.cpu().numpy()
        assert abs(b).max() > 0
        assert H.rel_l2(a, b) <= 2e-6
        db = H.nrms_db(a, oracle)
        assert db <= -60.0, f"{storage}: {db:.1f} dB against the FP64 oracle"


def test_noalloc_rejects_what_it_cannot_run(cuda):
    import torch

    from mach_b200 import _cuda_impl, _grid

    lib, fn = _bind()
    w, t, p, scale = _job("c64", 2)  # quadratic taps: not an ensemble-kernel job
    opts = _cuda_impl.make_options(_cuda_impl.FLAG_OVERWRITE, grid_shape=_grid.detect(t["scan"]))
    out = torch.zeros((w.n_vox, 64), dtype=torch.complex64, device="cuda")
    assert _call(fn, "c64", w, t, p, scale, out, opts) == 1
    assert b"ensemble kernel" in lib.mach_b200_last_error()
    p["interp_type"] = 1
    host_out = torch.zeros((w.n_vox, 64), dtype=torch.complex64)
    assert _call(fn, "c64", w, t, p, scale, host_out, opts) == 1
    assert b"device memory" in lib.mach_b200_last_error()
    opts.tx_model = 1  # a wave model needs a device buffer for its arrivals
    out = torch.zeros((w.n_vox, 64), dtype=torch.complex64, device="cuda")
    assert _call(fn, "c64", w, t, p, scale, out, opts) == 1
    assert b"tx_model 0" in lib.mach_b200_last_error()
