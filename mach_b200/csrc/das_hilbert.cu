// Analytic signal of real channel data along the sample axis (RF -> IQ with modulation
// frequency 0), optionally fused with the acquisition-order rearrange.
//
// mach's UFF front end calls scipy.signal.hilbert(signal, axis=0) on the host and then
// rearranges (src/mach/io/uff.py:70-105).  scipy forms the analytic signal with FFTs: the
// spectrum X of each column is multiplied by h (1 at DC, 2 on positive frequencies, 1 at
// Nyquist for even lengths, 0 on negative frequencies) and transformed back (Marple, "Computing
// the discrete-time analytic signal via FFT", IEEE TSP 47(9), 1999).  Written as
// z = x + i y with y = IFFT(-i sgn(k) X), the imaginary part is a real-linear map of x, so two
// real columns x1, x2 packed as x1 + i x2 share one forward and one inverse FFT:
// IFFT(-i sgn X(x1 + i x2)) = y1 + i y2.
//
// One CTA takes a group of columns (an even number), keeps their FFTs in shared memory and
// runs a mixed-radix Stockham FFT (self-sorting, out of place between two buffers): radix 8,
// 4 and 2 butterflies in registers, any other prime factor as a direct sum per output.  The
// twiddles W_n^m (m < n) are one FP64-accurate table per CTA, so every stage reads exact
// roots of unity.  Loads and stores walk the group either sample-fastest (contiguous columns)
// or column-fastest (contiguous rows of frames, or the acquisition order's element / wave
// rows), whichever is contiguous in memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "das_device.cuh"
#include "das_launch.cuh"

namespace mach_b200 {
namespace {

constexpr int kHilThreads = 256;

template <typename T>
struct RealIn;
template <>
struct RealIn<float> {
    __device__ static float get(const float* p) { return __ldg(p); }
};
template <>
struct RealIn<__half> {
    __device__ static float get(const __half* p) { return __half2float(__ldg(p)); }
};
template <>
struct RealIn<__nv_bfloat16> {
    __device__ static float get(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
};
template <>
struct RealIn<short> {
    __device__ static float get(const short* p) { return static_cast<float>(__ldg(p)); }
};

template <typename T>
struct ComplexOut;
template <>
struct ComplexOut<float> {
    __device__ static void put(float* p, float re, float im) { *reinterpret_cast<float2*>(p) = make_float2(re, im); }
};
template <>
struct ComplexOut<__half> {
    __device__ static void put(__half* p, float re, float im) {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(re, im);
    }
};
template <>
struct ComplexOut<__nv_bfloat16> {
    __device__ static void put(__nv_bfloat16* p, float re, float im) {
        *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(re, im);
    }
};
template <>
struct ComplexOut<short> {
    __device__ static short sat(float v) { return static_cast<short>(rintf(fminf(fmaxf(v, -32768.0f), 32767.0f))); }
    __device__ static void put(short* p, float re, float im) {
        short2 s;
        s.x = sat(re);
        s.y = sat(im);
        *reinterpret_cast<short2*>(p) = s;
    }
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a * b, or a * conj(b) for the inverse transform
template <bool INV>
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    if (INV) return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -(a.x * b.y)));
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}
// times -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 v) {
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
    const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = mul_mi<INV>(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2 (&v)[R]) {
    if constexpr (R == 2) {
        const float2 a = v[0];
        v[0] = cadd(a, v[1]);
        v[1] = csub(a, v[1]);
    } else if constexpr (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else {  // R == 8: two radix-4 transforms of the even and odd inputs, then radix 2
        float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<INV>(e0, e1, e2, e3);
        dft4<INV>(o0, o1, o2, o3);
        const float h = 0.70710678118654752f;  // 1 / sqrt(2)
        // o1 *= W8^1, o2 *= W8^2 = -i, o3 *= W8^3 (conjugates for the inverse)
        o1 = INV ? make_float2((o1.x - o1.y) * h, (o1.x + o1.y) * h) : make_float2((o1.x + o1.y) * h, (o1.y - o1.x) * h);
        o2 = mul_mi<INV>(o2);
        o3 = INV ? make_float2(-(o3.x + o3.y) * h, (o3.x - o3.y) * h) : make_float2((o3.y - o3.x) * h, -(o3.x + o3.y) * h);
        v[0] = cadd(e0, o0);
        v[4] = csub(e0, o0);
        v[1] = cadd(e1, o1);
        v[5] = csub(e1, o1);
        v[2] = cadd(e2, o2);
        v[6] = csub(e2, o2);
        v[3] = cadd(e3, o3);
        v[7] = csub(e3, o3);
    }
}

// The multiplier -i sgn(k) / n between the transforms, applied as the inverse transform's
// first stage reads spectrum bin k.
__device__ __forceinline__ float2 hilbert_bin(float2 v, int k, int n, float inv_n) {
    const int twice = 2 * k;
    if (k == 0 || twice == n) return make_float2(0.f, 0.f);
    return twice < n ? make_float2(v.y * inv_n, -v.x * inv_n) : make_float2(-v.y * inv_n, v.x * inv_n);
}

// One Stockham stage with a register butterfly: L = n / R butterflies per column pair.
template <int R, bool INV>
__device__ __forceinline__ void stage_small(const float2* __restrict__ tw, const float2* in, float2* out, int n,
                                            int ns, int pairs, bool spectrum_mul, float inv_n) {
    const int L = n / R;
    const int tw_step = n / (ns * R);
    for (int item = threadIdx.x; item < pairs * L; item += blockDim.x) {
        const int p = item / L, j = item - p * L;
        const int k = j % ns;
        const float2* src = in + p * n;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = src[j + r * L];
            if (spectrum_mul) x = hilbert_bin(x, j + r * L, n, inv_n);
            v[r] = r == 0 ? x : cmul<INV>(x, tw[r * k * tw_step]);
        }
        dft_small<R, INV>(v);
        float2* dst = out + p * n + (j / ns) * ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[r * ns] = v[r];
    }
}

// One Stockham stage of any radix R, each output a direct sum of its R inputs:
// out[(j / ns) ns R + k + q ns] = sum_r in[j + r L] W_n^(r (k n / (ns R) + q L)).
template <bool INV>
__device__ __forceinline__ void stage_generic(const float2* __restrict__ tw, const float2* in, float2* out, int n,
                                              int ns, int R, int pairs, bool spectrum_mul, float inv_n) {
    const int L = n / R;
    const int tw_step = n / (ns * R);
    for (int item = threadIdx.x; item < pairs * n; item += blockDim.x) {
        const int p = item / n, rest = item - p * n;
        const int q = rest / L, j = rest - q * L;
        const int k = j % ns;
        const float2* src = in + p * n;
        const int step = k * tw_step + q * L;  // < n
        int e = 0;
        float2 acc = make_float2(0.f, 0.f);
        for (int r = 0; r < R; ++r) {
            float2 x = src[j + r * L];
            if (spectrum_mul) x = hilbert_bin(x, j + r * L, n, inv_n);
            const float2 t = cmul<INV>(x, tw[e]);
            acc = cadd(acc, t);
            e += step;
            if (e >= n) e -= n;
        }
        out[p * n + (j / ns) * ns * R + k + q * ns] = acc;
    }
}

// Full transform of `pairs` columns of length n; the result ends in `a` (buffers swap per stage).
template <bool INV>
__device__ void fft_columns(const HilbertArgs& g, const float2* tw, float2*& a, float2*& b, int pairs, bool spectrum_mul) {
    int ns = 1;
    for (int s = 0; s < g.n_stages; ++s) {
        const int R = g.radix[s];
        const bool mul = spectrum_mul && s == 0;
        if (R == 8) {
            stage_small<8, INV>(tw, a, b, g.n, ns, pairs, mul, g.inv_n);
        } else if (R == 4) {
            stage_small<4, INV>(tw, a, b, g.n, ns, pairs, mul, g.inv_n);
        } else if (R == 2) {
            stage_small<2, INV>(tw, a, b, g.n, ns, pairs, mul, g.inv_n);
        } else {
            stage_generic<INV>(tw, a, b, g.n, ns, R, pairs, mul, g.inv_n);
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        ns *= R;
    }
}

__device__ __forceinline__ int64_t column_offset(int64_t c, const HilbertArgs& g, const int64_t (&stride)[3]) {
    const int64_t c0 = c % g.n0, t = c / g.n0;
    const int64_t c1 = t % g.n1, c2 = t / g.n1;
    return c0 * stride[0] + c1 * stride[1] + c2 * stride[2];
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kHilThreads) hilbert_kernel(const HilbertArgs g) {
    extern __shared__ float2 hil_smem[];
    const int n = g.n;
    const int C = g.cols_per_cta, P = C / 2;
    float2* tw = hil_smem;
    float2* buf0 = hil_smem + n;
    float2* buf1 = buf0 + static_cast<int64_t>(P) * n;
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * m / n, &sn, &cs);
        tw[m] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
    }
    const In* src = static_cast<const In*>(g.src);
    Out* dst = static_cast<Out*>(g.dst);
    const int64_t n_groups = (g.n_cols + C - 1) / C;
    const int total = C * n;
    for (int64_t grp = blockIdx.x; grp < n_groups; grp += gridDim.x) {
        const int64_t c_begin = grp * C;
        for (int i = threadIdx.x; i < total; i += blockDim.x) {
            int k, s;
            if (g.load_cols_fast) {
                k = i % C;
                s = i / C;
            } else {
                s = i % n;
                k = i / n;
            }
            const int64_t c = c_begin + k;
            float x = 0.f;
            if (c < g.n_cols) x = RealIn<In>::get(src + column_offset(c, g, g.src_stride) + s * g.src_sample);
            reinterpret_cast<float*>(buf0 + (k >> 1) * n + s)[k & 1] = x;
        }
        __syncthreads();
        float2* a = buf0;
        float2* b = buf1;
        fft_columns<false>(g, tw, a, b, P, false);
        if (g.n_stages == 0) {  // n == 1: the imaginary part is zero
            for (int p = threadIdx.x; p < P; p += blockDim.x) a[p * n] = make_float2(0.f, 0.f);
            __syncthreads();
        } else {
            fft_columns<true>(g, tw, a, b, P, true);
        }
        for (int i = threadIdx.x; i < total; i += blockDim.x) {
            int k, s;
            if (g.store_cols_fast) {
                k = i % C;
                s = i / C;
            } else {
                s = i % n;
                k = i / n;
            }
            const int64_t c = c_begin + k;
            if (c >= g.n_cols) continue;
            const float x = RealIn<In>::get(src + column_offset(c, g, g.src_stride) + s * g.src_sample);
            const float y = reinterpret_cast<const float*>(a + (k >> 1) * n + s)[k & 1];
            ComplexOut<Out>::put(dst + 2 * (column_offset(c, g, g.dst_stride) + s * g.dst_sample), x * g.scale,
                                 y * g.scale);
        }
        __syncthreads();
    }
}

template <typename In, typename Out>
cudaError_t hilbert_typed(const HilbertArgs& g, int blocks, size_t smem, cudaStream_t st) {
    auto k = hilbert_kernel<In, Out>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    k<<<blocks, kHilThreads, smem, st>>>(g);
    return cudaGetLastError();
}

template <typename In>
cudaError_t hilbert_to(int dst_code, const HilbertArgs& g, int blocks, size_t smem, cudaStream_t st) {
    switch (dst_code) {
        case kC64: return hilbert_typed<In, float>(g, blocks, smem, st);
        case kCF16: return hilbert_typed<In, __half>(g, blocks, smem, st);
        case kCBF16: return hilbert_typed<In, __nv_bfloat16>(g, blocks, smem, st);
        default: return hilbert_typed<In, short>(g, blocks, smem, st);
    }
}

}  // namespace

int hilbert_plan(int n, int* radix, int max_stages) {
    int count = 0, m = n;
    for (int r : {8, 4, 2}) {
        while (m % r == 0) {
            if (count == max_stages) return -1;
            radix[count++] = r;
            m /= r;
        }
    }
    for (int p = 3; m > 1; p += 2) {
        while (m % p == 0) {
            if (count == max_stages) return -1;
            radix[count++] = p;
            m /= p;
        }
        if (static_cast<int64_t>(p) * p > m && m > 1) {  // what is left is prime
            if (count == max_stages) return -1;
            radix[count++] = m;
            m = 1;
        }
    }
    return count;
}

cudaError_t launch_hilbert(int src_code, int dst_code, const HilbertArgs& g, int blocks, size_t smem,
                           cudaStream_t st) {
    switch (src_code) {
        case kF32: return hilbert_to<float>(dst_code, g, blocks, smem, st);
        case kF16: return hilbert_to<__half>(dst_code, g, blocks, smem, st);
        case kBF16: return hilbert_to<__nv_bfloat16>(dst_code, g, blocks, smem, st);
        default: return hilbert_to<short>(dst_code, g, blocks, smem, st);
    }
}

}  // namespace mach_b200
