// Transmit arrivals from a wave model: arr[t][v] for plane or spherical waves, formed on the
// device so that the [n_tx][n_scan] array never crosses the host link.
//
// For transmit t with table row q = params[8 t .. 8 t + 8) (origin xyz, unit direction or
// focus xyz, time offset, unused), the arrival at scan point p is the distance of
// src/mach/wavefront.py:8-116 divided by the sound speed, plus the offset:
//   plane      d = (p - o) . direction
//   spherical  d = |o - f| sign(f_z - o_z) - |f - p| sign(f_z - p_z)
// computed in FP64 from the FP32 scan point and rounded to FP32, which is what a host
// evaluation in float64 followed by mach's float32 cast (src/mach/kernel.py:231-233) gives.
// One thread per (point, transmit); writes are coalesced along the points.
#include <cstdint>

#include "das_launch.cuh"

namespace mach_b200 {
namespace {

__global__ void __launch_bounds__(256) tx_arrivals_kernel(int model, const double* __restrict__ params,
                                                          const float* __restrict__ scan, int64_t n_scan, int n_tx,
                                                          double c, float* __restrict__ out) {
    for (int t = blockIdx.y; t < n_tx; t += gridDim.y) {
        const double* q = params + 8 * static_cast<int64_t>(t);
        const double ox = __ldg(q + 0), oy = __ldg(q + 1), oz = __ldg(q + 2);
        const double gx = __ldg(q + 3), gy = __ldg(q + 4), gz = __ldg(q + 5);
        const double offset = __ldg(q + 6);
        const double of = sqrt((ox - gx) * (ox - gx) + (oy - gy) * (oy - gy) + (oz - gz) * (oz - gz));
        const double so = gz > oz ? 1.0 : (gz < oz ? -1.0 : 0.0);
        for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n_scan;
             v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            const double px = __ldg(scan + 3 * v + 0), py = __ldg(scan + 3 * v + 1), pz = __ldg(scan + 3 * v + 2);
            double d;
            if (model == 1) {
                d = (px - ox) * gx + (py - oy) * gy + (pz - oz) * gz;
            } else {
                const double fp = sqrt((gx - px) * (gx - px) + (gy - py) * (gy - py) + (gz - pz) * (gz - pz));
                const double sp = gz > pz ? 1.0 : (gz < pz ? -1.0 : 0.0);
                d = of * so - fp * sp;
            }
            out[static_cast<int64_t>(t) * n_scan + v] = static_cast<float>(d / c + offset);
        }
    }
}

}  // namespace

cudaError_t launch_tx_arrivals(int model, const double* params, const float* scan, int64_t n_scan, int n_tx,
                               double sound_speed, float* out, cudaStream_t st) {
    if (n_scan <= 0 || n_tx <= 0) return cudaSuccess;
    const int64_t bx = std::min<int64_t>((n_scan + 255) / 256, 4096);
    const dim3 grid(static_cast<unsigned>(bx), static_cast<unsigned>(std::min(n_tx, 65535)), 1);
    tx_arrivals_kernel<<<grid, 256, 0, st>>>(model, params, scan, n_scan, n_tx, sound_speed, out);
    return cudaGetLastError();
}

}  // namespace mach_b200
