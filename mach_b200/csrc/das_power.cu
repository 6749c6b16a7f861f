// Power-Doppler epilogue for jobs the fused path does not take: out[v] (+)= sum over frames
// of |x[v][f]|^2, one warp per scan point (lanes stride over the frames, coalesced).
#include "das_launch.cuh"

namespace mach_b200 {

__global__ void __launch_bounds__(256) das_power_kernel(const void* in, float* out, int64_t n_vox, int n_frames,
                                                        int cplx, int accumulate) {
    const int64_t v = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (v >= n_vox) return;  // whole warps leave together
    float s = 0.f;
    if (cplx) {
        const float2* row = static_cast<const float2*>(in) + v * n_frames;
        for (int f = lane; f < n_frames; f += 32) {
            const float2 x = row[f];
            s = __fmaf_rn(x.x, x.x, __fmaf_rn(x.y, x.y, s));
        }
    } else {
        const float* row = static_cast<const float*>(in) + v * n_frames;
        for (int f = lane; f < n_frames; f += 32) s = __fmaf_rn(row[f], row[f], s);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[v] = accumulate ? __fadd_rn(out[v], s) : s;
}

cudaError_t launch_power_epilogue(const void* in, float* out, int64_t n_vox, int n_frames, bool cplx, bool accumulate,
                                  cudaStream_t stream) {
    if (n_vox <= 0) return cudaSuccess;
    const int64_t blocks = (n_vox * 32 + 255) / 256;
    das_power_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(in, out, n_vox, n_frames, cplx ? 1 : 0,
                                                                          accumulate ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace mach_b200
