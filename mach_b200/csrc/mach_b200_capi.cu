// C ABI of mach_b200 (declared in include/mach_b200.h): argument checks, host-buffer
// staging, launch planning and the kernel dispatch.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "das_gather.cuh"
#include "mach_b200.h"

#ifndef MACH_B200_NVCC_VERSION
#define MACH_B200_NVCC_VERSION "0.0.0"
#endif
#define MACH_B200_VERSION "0.1.0"

namespace mach_b200 {
// Instantiated once per storage type in das_gather_<storage>.cu.
extern template cudaError_t launch_das_gather<kF32>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kC64>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kF16>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kCF16>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kBF16>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kCBF16>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kI16>(const DasArgs&, int, int, dim3, cudaStream_t);
extern template cudaError_t launch_das_gather<kCI16>(const DasArgs&, int, int, dim3, cudaStream_t);
}  // namespace mach_b200

namespace {

using namespace mach_b200;

thread_local std::string g_error;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define MACH_B200_CUDA_TRY(expr)                                                                  \
    do {                                                                                          \
        cudaError_t err_ = (expr);                                                                \
        if (err_ != cudaSuccess) {                                                                \
            return fail(MACH_B200_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(err_));   \
        }                                                                                         \
    } while (0)

size_t storage_bytes(int storage) {
    switch (storage) {
        case kF32: return 4;
        case kC64: return 8;
        case kF16: case kBF16: case kI16: return 2;
        default: return 4;  // cf16, cbf16, ci16
    }
}

enum Residency { kOnDevice, kHostPinned, kHostPageable };

// Where does `p` live?  Device pointers must belong to `device`.
int residency(const void* p, int device, Residency* r, const char* name) {
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *r = kHostPageable;
        return MACH_B200_OK;
    }
    switch (attr.type) {
        case cudaMemoryTypeDevice:
        case cudaMemoryTypeManaged:
            if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
                return fail(MACH_B200_ERR_DEVICE,
                            "%s is on CUDA device %d but the current device is %d", name, attr.device,
                            device);
            }
            *r = kOnDevice;
            return MACH_B200_OK;
        case cudaMemoryTypeHost:
            *r = kHostPinned;
            return MACH_B200_OK;
        default:
            *r = kHostPageable;
            return MACH_B200_OK;
    }
}

struct LaunchPlan {
    int shape;
    int passes;
    dim3 grid;
};

LaunchPlan plan_launch(uint64_t n_vox, uint32_t n_frames) {
    LaunchPlan p{};
    if (n_frames <= 1) {
        p.shape = kShapeOneFrame;
        p.passes = 1;
    } else if (n_frames <= 8) {
        p.shape = kShapeFewFrames;
        p.passes = static_cast<int>(n_frames);
    } else if (n_frames <= 16) {
        p.shape = kShapeHalfWarp;
        p.passes = 1;
    } else {
        p.shape = kShapeWarp;
        p.passes = static_cast<int>(std::min<uint32_t>(8, (n_frames + 31) / 32));
    }
    const ShapeInfo si = shape_info(p.shape);
    const uint64_t vox_per_cta = static_cast<uint64_t>(kThreadsPerBlock / 32) * (32 / si.lpv);
    p.grid.x = static_cast<unsigned>((n_vox + vox_per_cta - 1) / vox_per_cta);
    const uint32_t frames_per_cta = static_cast<uint32_t>(si.lpv * p.passes);
    p.grid.y = (n_frames + frames_per_cta - 1) / frames_per_cta;
    p.grid.z = 1;
    return p;
}

cudaError_t dispatch(int storage, const DasArgs& a, int interp, const LaunchPlan& plan, cudaStream_t st) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    switch (storage) {
        case kF32: return launch_das_gather<kF32>(a, interp, plan.shape, plan.grid, st);
        case kC64: return launch_das_gather<kC64>(a, interp, plan.shape, plan.grid, st);
        case kF16: return launch_das_gather<kF16>(a, interp, plan.shape, plan.grid, st);
        case kCF16: return launch_das_gather<kCF16>(a, interp, plan.shape, plan.grid, st);
        case kBF16: return launch_das_gather<kBF16>(a, interp, plan.shape, plan.grid, st);
        case kCBF16: return launch_das_gather<kCBF16>(a, interp, plan.shape, plan.grid, st);
        case kI16: return launch_das_gather<kI16>(a, interp, plan.shape, plan.grid, st);
        default: return launch_das_gather<kCI16>(a, interp, plan.shape, plan.grid, st);
    }
}

// Stream-ordered device buffer released at scope exit (on the stream it was allocated on).
struct DeviceBuffer {
    void* ptr = nullptr;
    cudaStream_t stream = nullptr;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    cudaError_t alloc(size_t bytes, cudaStream_t st) {
        stream = st;
        return cudaMallocAsync(&ptr, bytes ? bytes : 1, st);
    }
    ~DeviceBuffer() {
        if (ptr) cudaFreeAsync(ptr, stream);
    }
};

struct EventPair {
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~EventPair() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    cudaError_t create() {
        for (auto& e : ev) {
            const cudaError_t err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (err != cudaSuccess) return err;
        }
        return cudaSuccess;
    }
};

struct StreamHolder {
    cudaStream_t s = nullptr;
    ~StreamHolder() {
        if (s) cudaStreamDestroy(s);
    }
};

int compound_impl(int32_t storage, const void* channel_data, const float* rx_coords_m,
                  const float* scan_coords_m, const float* tx_wave_arrivals_s, void* out, uint32_t n_tx,
                  uint32_t n_rx, uint32_t n_samples, uint64_t n_scan, uint32_t n_frames, float f_number,
                  float rx_start_s, float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                  float tukey_alpha, int32_t interp_type, float channel_scale, cudaStream_t stream,
                  uint32_t flags) {
    g_error.clear();
    if (storage < kF32 || storage > kCI16) return fail(MACH_B200_ERR_VALUE, "unknown storage code %d", storage);
    if (interp_type < kNearest || interp_type > kQuadratic) {
        return fail(MACH_B200_ERR_VALUE, "interp_type must be 0 (NearestNeighbor), 1 (Linear) or 2 (Quadratic), got %d",
                    interp_type);
    }
    // Same range check and message as mach (src/mach/kernel.cu:745-748).
    if (!(tukey_alpha >= 0.0f && tukey_alpha <= 1.0f)) {
        return fail(MACH_B200_ERR_VALUE, "Error: tukey_alpha must be in range [0, 1], but got %f", tukey_alpha);
    }
    if (n_scan == 0 || n_frames == 0) return MACH_B200_OK;  // empty output: nothing to write
    if (!out || !scan_coords_m) return fail(MACH_B200_ERR_VALUE, "out and scan_coords_m must not be NULL");
    const bool need_channel = n_tx > 0 && n_rx > 0 && n_samples > 0;
    if (need_channel && (!channel_data || !rx_coords_m || !tx_wave_arrivals_s)) {
        return fail(MACH_B200_ERR_VALUE, "channel_data, rx_coords_m and tx_wave_arrivals_s must not be NULL");
    }
    if (n_frames > 65535u * 256u) return fail(MACH_B200_ERR_VALUE, "n_frames %u is too large", n_frames);
    // Sample indices are exact FP32 integers only up to 2^24 (the interpolation bounds rely on it).
    if (n_samples > (1u << 24)) return fail(MACH_B200_ERR_VALUE, "n_samples %u exceeds 2^24", n_samples);
    if (n_rx > 0x7fffffffu || n_tx > 0x7fffffffu) return fail(MACH_B200_ERR_VALUE, "n_rx / n_tx too large");
    if (n_scan > 0x7fffffffull * 4ull) {
        return fail(MACH_B200_ERR_VALUE, "n_scan %llu is too large", static_cast<unsigned long long>(n_scan));
    }

    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    Residency r_ch = kOnDevice, r_rx = kOnDevice, r_scan = kOnDevice, r_arr = kOnDevice, r_out = kOnDevice;
    int rc;
    if (need_channel) {
        if ((rc = residency(channel_data, device, &r_ch, "channel_data"))) return rc;
        if ((rc = residency(rx_coords_m, device, &r_rx, "rx_coords_m"))) return rc;
        if ((rc = residency(tx_wave_arrivals_s, device, &r_arr, "tx_wave_arrivals_s"))) return rc;
    }
    if ((rc = residency(scan_coords_m, device, &r_scan, "scan_coords_m"))) return rc;
    if ((rc = residency(out, device, &r_out, "out"))) return rc;

    const bool cplx = (storage & 1) != 0;
    const size_t esz = storage_bytes(storage);
    const size_t out_bytes = static_cast<size_t>(n_scan) * n_frames * (cplx ? 8 : 4);

    DasArgs a{};
    a.rx = rx_coords_m;
    a.scan = scan_coords_m;
    a.n_vox = static_cast<int64_t>(n_scan);
    a.n_rx = static_cast<int32_t>(need_channel ? n_rx : 0);
    a.n_samples = static_cast<int32_t>(n_samples);
    a.n_frames = static_cast<int32_t>(n_frames);
    a.row_stride = static_cast<int64_t>(n_samples) * n_frames;
    a.inv_c = 1.0f / sound_speed_m_s;  // kernel.cu:750, FP32 on the host
    a.fs = sampling_freq_hz;
    a.t0 = rx_start_s;
    a.two_f_number = 2.0f * f_number;
    a.alpha = tukey_alpha;
    a.one_minus_alpha = 1.0f - tukey_alpha;
    a.mod_rad = (2.0f * kPi) * modulation_freq_hz;  // kernel.cu:571
    a.scale = channel_scale;
    a.hi_nearest = static_cast<float>(n_samples) - 0.5f;
    a.hi_linear = static_cast<float>(n_samples - 1u);
    a.hi_quadratic = static_cast<float>(n_samples) - 2.0f;
    a.apod = tukey_alpha > 0.0f;
    a.rotate = cplx && modulation_freq_hz != 0.0f;
    const bool overwrite = (flags & MACH_B200_FLAG_OVERWRITE) != 0u || r_out != kOnDevice;
    const LaunchPlan plan = plan_launch(n_scan, n_frames);
    a.frame_passes = plan.passes;

    const bool all_device = r_ch == kOnDevice && r_rx == kOnDevice && r_scan == kOnDevice && r_arr == kOnDevice &&
                            r_out == kOnDevice;
    if (all_device) {
        a.channel = channel_data;
        a.arrivals = tx_wave_arrivals_s;
        a.out = out;
        a.n_tx = static_cast<int32_t>(need_channel ? n_tx : 0);
        a.accumulate = overwrite ? 0 : 1;
        MACH_B200_CUDA_TRY(dispatch(storage, a, interp_type, plan, stream));
        if (!(flags & MACH_B200_FLAG_ASYNC)) MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
        return MACH_B200_OK;
    }

    // ---- staging path: some buffers live in host memory ----
    DeviceBuffer d_rx, d_scan, d_out, d_ch[2], d_arr[2];
    if (need_channel && r_rx != kOnDevice) {
        MACH_B200_CUDA_TRY(d_rx.alloc(static_cast<size_t>(n_rx) * 12, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_rx.ptr, rx_coords_m, static_cast<size_t>(n_rx) * 12,
                                           cudaMemcpyHostToDevice, stream));
        a.rx = static_cast<const float*>(d_rx.ptr);
    }
    if (r_scan != kOnDevice) {
        MACH_B200_CUDA_TRY(d_scan.alloc(static_cast<size_t>(n_scan) * 12, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_scan.ptr, scan_coords_m, static_cast<size_t>(n_scan) * 12,
                                           cudaMemcpyHostToDevice, stream));
        a.scan = static_cast<const float*>(d_scan.ptr);
    }
    void* dev_out = out;
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(d_out.alloc(out_bytes, stream));
        dev_out = d_out.ptr;
    }
    a.out = dev_out;

    const size_t tx_bytes = static_cast<size_t>(n_rx) * n_samples * n_frames * esz;
    const size_t arr_bytes = static_cast<size_t>(n_scan) * 4;
    if (!need_channel) {
        // No samples to gather: the result is zero.
        MACH_B200_CUDA_TRY(cudaMemsetAsync(dev_out, 0, out_bytes, stream));
    } else if (r_ch == kOnDevice && r_arr == kOnDevice) {
        a.channel = channel_data;
        a.arrivals = tx_wave_arrivals_s;
        a.n_tx = static_cast<int32_t>(n_tx);
        a.accumulate = overwrite ? 0 : 1;
        MACH_B200_CUDA_TRY(dispatch(storage, a, interp_type, plan, stream));
    } else {
        // Transmit chunks copied on a side stream while the previous chunk is gathered.
        const uint32_t chunk = std::max<uint32_t>(1u, std::min<uint32_t>(n_tx, (n_tx + 7u) / 8u));
        StreamHolder copy;
        EventPair copied, consumed;
        MACH_B200_CUDA_TRY(cudaStreamCreateWithFlags(&copy.s, cudaStreamNonBlocking));
        MACH_B200_CUDA_TRY(copied.create());
        MACH_B200_CUDA_TRY(consumed.create());
        // The copy stream must not start before buffers allocated on `stream` exist.
        cudaEvent_t ready;
        MACH_B200_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        for (int b = 0; b < 2; ++b) {
            if (r_ch != kOnDevice) MACH_B200_CUDA_TRY(d_ch[b].alloc(tx_bytes * chunk, stream));
            if (r_arr != kOnDevice) MACH_B200_CUDA_TRY(d_arr[b].alloc(arr_bytes * chunk, stream));
        }
        cudaEventRecord(ready, stream);
        cudaStreamWaitEvent(copy.s, ready, 0);
        cudaEventDestroy(ready);
        const char* h_ch = static_cast<const char*>(channel_data);
        const char* h_arr = reinterpret_cast<const char*>(tx_wave_arrivals_s);
        uint32_t k = 0;
        for (uint32_t t0 = 0; t0 < n_tx; t0 += chunk, ++k) {
            const uint32_t nt = std::min(chunk, n_tx - t0);
            const int b = static_cast<int>(k & 1u);
            if (k >= 2) MACH_B200_CUDA_TRY(cudaStreamWaitEvent(copy.s, consumed.ev[b], 0));
            if (r_ch != kOnDevice) {
                MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_ch[b].ptr, h_ch + tx_bytes * t0, tx_bytes * nt,
                                                   cudaMemcpyHostToDevice, copy.s));
                a.channel = d_ch[b].ptr;
            } else {
                a.channel = h_ch + tx_bytes * t0;
            }
            if (r_arr != kOnDevice) {
                MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_arr[b].ptr, h_arr + arr_bytes * t0, arr_bytes * nt,
                                                   cudaMemcpyHostToDevice, copy.s));
                a.arrivals = static_cast<const float*>(d_arr[b].ptr);
            } else {
                a.arrivals = reinterpret_cast<const float*>(h_arr + arr_bytes * t0);
            }
            MACH_B200_CUDA_TRY(cudaEventRecord(copied.ev[b], copy.s));
            MACH_B200_CUDA_TRY(cudaStreamWaitEvent(stream, copied.ev[b], 0));
            a.n_tx = static_cast<int32_t>(nt);
            a.accumulate = (k > 0 || !overwrite) ? 1 : 0;
            MACH_B200_CUDA_TRY(dispatch(storage, a, interp_type, plan, stream));
            MACH_B200_CUDA_TRY(cudaEventRecord(consumed.ev[b], stream));
        }
        // Later frees on `stream` must wait for the copy stream's last use of the buffers.
        MACH_B200_CUDA_TRY(cudaStreamWaitEvent(stream, copied.ev[(k - 1) & 1u], 0));
    }
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(out, dev_out, out_bytes, cudaMemcpyDeviceToHost, stream));
    }
    // Host buffers are in use until the stream drains: always synchronous here.
    MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    return MACH_B200_OK;
}

}  // namespace

extern "C" {

int mach_b200_beamform_f32(const float* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                           const float* tx_wave_arrivals_s, float* out, uint32_t n_rx, uint32_t n_samples,
                           uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                           float tukey_alpha, int32_t interp_type) {
    return compound_impl(kF32, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, 1u, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, 1.0f, nullptr, 0u);
}

int mach_b200_beamform_c64(const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                           const float* tx_wave_arrivals_s, void* out, uint32_t n_rx, uint32_t n_samples,
                           uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                           float tukey_alpha, int32_t interp_type) {
    return compound_impl(kC64, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, 1u, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, 1.0f, nullptr, 0u);
}

int mach_b200_beamform_compound(int32_t storage, const void* channel_data, const float* rx_coords_m,
                                const float* scan_coords_m, const float* tx_wave_arrivals_s, void* out,
                                uint32_t n_tx, uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                                float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha,
                                int32_t interp_type, float channel_scale, void* cuda_stream, uint32_t flags) {
    return compound_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, channel_scale,
                         static_cast<cudaStream_t>(cuda_stream), flags);
}

const char* mach_b200_last_error(void) { return g_error.c_str(); }

const char* mach_b200_nvcc_version(void) { return MACH_B200_NVCC_VERSION; }

const char* mach_b200_version(void) { return MACH_B200_VERSION; }

uint64_t mach_b200_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
