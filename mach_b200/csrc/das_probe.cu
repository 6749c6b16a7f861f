// L2 read-bandwidth probe: the denominator of the L2 roofline that the gather kernels are
// measured against (their sample rows come from L2, not from HBM, once the first CTA of a
// region has touched them).  Every thread streams 16-byte words of a device buffer with
// ld.global.cg (cached in L2, not in L1), four loads in flight per thread, for `passes`
// passes; the XOR of the words goes to a device word so that no load is dead code.  With a
// buffer smaller than L2 and the first pass untimed, every later pass is served by L2.
#include <cuda_runtime.h>

#include <cstdint>

#include "mach_b200.h"

namespace {

__device__ unsigned g_probe_sink;

__device__ __forceinline__ uint4 load_cg(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

__global__ void __launch_bounds__(512) l2_read_kernel(const uint4* __restrict__ buf, int64_t n_words, int passes) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned x = 0;
    for (int p = 0; p < passes; ++p) {
        int64_t i = first;
        for (; i + 3 * stride < n_words; i += 4 * stride) {
            const uint4 a = load_cg(buf + i);
            const uint4 b = load_cg(buf + i + stride);
            const uint4 c = load_cg(buf + i + 2 * stride);
            const uint4 d = load_cg(buf + i + 3 * stride);
            x ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        for (; i < n_words; i += stride) {
            const uint4 a = load_cg(buf + i);
            x ^= a.x ^ a.y ^ a.z ^ a.w;
        }
    }
    if (x == 0x9e3779b9u) g_probe_sink = x;  // data-dependent store: the loads stay live
}

}  // namespace

extern "C" int mach_b200_probe_l2_read(const void* buffer, uint64_t bytes, uint32_t passes, void* cuda_stream) {
    if (buffer == nullptr || bytes < 16 || bytes % 16 != 0 || reinterpret_cast<uintptr_t>(buffer) % 16 != 0 ||
        passes == 0) {
        return MACH_B200_ERR_VALUE;
    }
    int device = 0, sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return MACH_B200_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return MACH_B200_ERR_CUDA;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, buffer) != cudaSuccess || attr.type != cudaMemoryTypeDevice ||
        attr.device != device) {
        cudaGetLastError();
        return MACH_B200_ERR_VALUE;
    }
    l2_read_kernel<<<sms * 4, 512, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
        static_cast<const uint4*>(buffer), static_cast<int64_t>(bytes / 16), static_cast<int>(passes));
    return cudaGetLastError() == cudaSuccess ? MACH_B200_OK : MACH_B200_ERR_CUDA;
}
