// Channel-data ingest: acquisition order (n_samples, n_elements, n_waves, n_frames) to the
// beamformer's (n_waves, n_elements, n_samples, n_frames), converted to a storage type in the
// same pass (src/mach/io/uff.py:70-105 rearranges with einops and casts on the host).
//
// A "row" is the n_frames (x2 for complex) contiguous scalars of one (sample, element, wave);
// the permutation moves whole rows.  Short rows (<= 16 bytes of output) go through a 32 x 32
// shared-memory tile per element, so that both the reads (consecutive waves) and the writes
// (consecutive samples) are coalesced; longer rows are already contiguous runs and are copied
// by one warp each.  Pure data movement: the bound is HBM bandwidth (read + write once).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "das_device.cuh"

namespace mach_b200 {
namespace {

template <typename T>
struct Scalar;
template <>
struct Scalar<float> {
    __device__ static float get(float x) { return x; }
    __device__ static float put(float v) { return v; }
};
template <>
struct Scalar<__half> {
    __device__ static float get(__half x) { return __half2float(x); }
    __device__ static __half put(float v) { return __float2half_rn(v); }
};
template <>
struct Scalar<__nv_bfloat16> {
    __device__ static float get(__nv_bfloat16 x) { return __bfloat162float(x); }
    __device__ static __nv_bfloat16 put(float v) { return __float2bfloat16_rn(v); }
};
template <>
struct Scalar<short> {
    __device__ static float get(short x) { return static_cast<float>(x); }
    __device__ static short put(float v) {
        const float r = rintf(fminf(fmaxf(v, -32768.0f), 32767.0f));
        return static_cast<short>(r);
    }
};

template <typename In, typename Out>
__device__ __forceinline__ Out convert(In x, float scale) {
    return Scalar<Out>::put(__fmul_rn(Scalar<In>::get(x), scale));
}

constexpr int kTile = 32;

// Short rows: tile of 32 samples x 32 waves of one element, R scalars per row.
template <typename In, typename Out, int R>
__global__ void __launch_bounds__(kTile * 8) ingest_tile_kernel(const In* __restrict__ src, Out* __restrict__ dst,
                                                                int n_s, int n_e, int n_w, float scale) {
    __shared__ Out tile[kTile][kTile + 1][R];
    const int w0 = blockIdx.x * kTile, s0 = blockIdx.y * kTile, e = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int sl = ty; sl < kTile; sl += 8) {
        const int s = s0 + sl, w = w0 + tx;
        if (s < n_s && w < n_w) {
            const In* row = src + ((static_cast<int64_t>(s) * n_e + e) * n_w + w) * R;
#pragma unroll
            for (int r = 0; r < R; ++r) tile[sl][tx][r] = convert<In, Out>(row[r], scale);
        }
    }
    __syncthreads();
    for (int wl = ty; wl < kTile; wl += 8) {
        const int w = w0 + wl, s = s0 + tx;
        if (s < n_s && w < n_w) {
            Out* row = dst + ((static_cast<int64_t>(w) * n_e + e) * n_s + s) * R;
#pragma unroll
            for (int r = 0; r < R; ++r) row[r] = tile[tx][wl][r];
        }
    }
}

// Long rows: one warp per row, lanes over the row's scalars.
template <typename In, typename Out>
__global__ void __launch_bounds__(256) ingest_row_kernel(const In* __restrict__ src, Out* __restrict__ dst, int n_s,
                                                         int n_e, int n_w, int64_t row_len, float scale) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t n_rows = static_cast<int64_t>(n_s) * n_e * n_w;
    if (row >= n_rows) return;
    const int w = static_cast<int>(row % n_w);
    const int64_t se = row / n_w;
    const int e = static_cast<int>(se % n_e);
    const int s = static_cast<int>(se / n_e);
    const In* in = src + row * row_len;
    Out* out = dst + ((static_cast<int64_t>(w) * n_e + e) * n_s + s) * row_len;
    for (int64_t i = lane; i < row_len; i += 32) out[i] = convert<In, Out>(in[i], scale);
}

template <typename In, typename Out>
cudaError_t ingest_typed(const void* src, void* dst, int n_s, int n_e, int n_w, int64_t row_len, float scale,
                         cudaStream_t st) {
    const In* s = static_cast<const In*>(src);
    Out* d = static_cast<Out*>(dst);
    const dim3 block(kTile, 8, 1);
    const dim3 grid((n_w + kTile - 1) / kTile, (n_s + kTile - 1) / kTile, n_e);
    if (row_len * static_cast<int64_t>(sizeof(Out)) <= 16 && grid.y <= 65535u && grid.z <= 65535u) {
        switch (row_len) {
            case 1: ingest_tile_kernel<In, Out, 1><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            case 2: ingest_tile_kernel<In, Out, 2><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            case 3: ingest_tile_kernel<In, Out, 3><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            case 4: ingest_tile_kernel<In, Out, 4><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            case 6: ingest_tile_kernel<In, Out, 6><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            case 8: ingest_tile_kernel<In, Out, 8><<<grid, block, 0, st>>>(s, d, n_s, n_e, n_w, scale); break;
            default: goto rows;
        }
        return cudaGetLastError();
    }
rows:
    {
        const int64_t n_rows = static_cast<int64_t>(n_s) * n_e * n_w;
        const int64_t blocks = (n_rows * 32 + 255) / 256;
        ingest_row_kernel<In, Out><<<static_cast<unsigned>(blocks), 256, 0, st>>>(s, d, n_s, n_e, n_w, row_len, scale);
    }
    return cudaGetLastError();
}

template <typename In>
cudaError_t ingest_to(int dst_code, const void* src, void* dst, int n_s, int n_e, int n_w, int64_t row_len,
                      float scale, cudaStream_t st) {
    switch (dst_code) {
        case kF32:
        case kC64: return ingest_typed<In, float>(src, dst, n_s, n_e, n_w, row_len, scale, st);
        case kF16:
        case kCF16: return ingest_typed<In, __half>(src, dst, n_s, n_e, n_w, row_len, scale, st);
        case kBF16:
        case kCBF16: return ingest_typed<In, __nv_bfloat16>(src, dst, n_s, n_e, n_w, row_len, scale, st);
        default: return ingest_typed<In, short>(src, dst, n_s, n_e, n_w, row_len, scale, st);
    }
}

}  // namespace

// Complex codes move (I, Q) pairs as two scalars of the row; the caller has checked that
// source and destination are both real or both complex.
cudaError_t launch_ingest(int src_code, const void* src, int dst_code, void* dst, int n_s, int n_e, int n_w,
                          int n_frames, float scale, cudaStream_t st) {
    const int64_t row_len = static_cast<int64_t>(n_frames) * ((src_code & 1) ? 2 : 1);
    switch (src_code) {
        case kF32:
        case kC64: return ingest_to<float>(dst_code, src, dst, n_s, n_e, n_w, row_len, scale, st);
        case kF16:
        case kCF16: return ingest_to<__half>(dst_code, src, dst, n_s, n_e, n_w, row_len, scale, st);
        case kBF16:
        case kCBF16: return ingest_to<__nv_bfloat16>(dst_code, src, dst, n_s, n_e, n_w, row_len, scale, st);
        default: return ingest_to<short>(dst_code, src, dst, n_s, n_e, n_w, row_len, scale, st);
    }
}

}  // namespace mach_b200
