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
// One CTA takes a group of 2, 4, 8 or 16 columns, keeps their FFTs in shared memory and runs a
// mixed-radix Stockham FFT (self-sorting, out of place between two buffers): radix 16, 8, 4, 2,
// 3, 5, 7, 11 and 13 butterflies in registers, a larger prime factor as a direct sum per
// output.  Each stage reads its own twiddle table, laid out so that neighbouring butterflies
// read neighbouring entries; all tables together hold n - 1 roots, computed in FP64 once per
// CTA.  Column buffers carry one float2 of padding per 32, which keeps the strided writes of
// the first stages free of bank conflicts.  Loads and stores walk the group either
// sample-fastest (contiguous columns) or column-fastest (contiguous rows of frames, or the
// acquisition order's element / wave rows), whichever is contiguous in memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdint>

#include "das_device.cuh"
#include "das_launch.cuh"

namespace mach_b200 {
namespace {

constexpr int kHilThreads = 256;
constexpr int kHilMaxRegisterRadix = 16;  // larger radices use stage_generic
constexpr int kHilMaxCols = 16;

// Raw loads (no conversion, so a prefetched load stays in flight until its value is used) and
// the widening to float.
template <typename T>
struct RealIn {
    __device__ static T raw(const T* p) { return __ldg(p); }
    __device__ static float get(const T* p) { return widen(raw(p)); }
    __device__ static float widen(float x) { return x; }
    __device__ static float widen(__half x) { return __half2float(x); }
    __device__ static float widen(__nv_bfloat16 x) { return __bfloat162float(x); }
    __device__ static float widen(short x) { return static_cast<float>(x); }
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

// W16^m for m = 0..9 (cos(pi m / 8), sin(pi m / 8)); the forward root is cos - i sin.
__device__ __forceinline__ float2 w16(int m, bool inv) {
    constexpr float c[10] = {1.0f, 0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                             -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128676f, -1.0f,
                             -0.92387953251128676f};
    constexpr float s[10] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128676f, 1.0f,
                             0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                             -0.38268343236508977f};
    return make_float2(c[m], inv ? s[m] : -s[m]);
}

// Power-of-two radix in registers.
template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2 (&v)[R]) {
    if constexpr (R == 16) {  // 4 x 4: DFT4 over b of v[a + 4b], twiddle W16^(a c), DFT4 over a
#pragma unroll
        for (int a = 0; a < 4; ++a) dft4<INV>(v[a], v[a + 4], v[a + 8], v[a + 12]);
#pragma unroll
        for (int a = 1; a < 4; ++a) {
#pragma unroll
            for (int c = 1; c < 4; ++c) v[a + 4 * c] = cmul<false>(v[a + 4 * c], w16(a * c, INV));
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) dft4<INV>(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        float2 o[16];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
#pragma unroll
            for (int d = 0; d < 4; ++d) o[c + 4 * d] = v[4 * c + d];
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = o[k];
    } else if constexpr (R == 2) {
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
        o1 = cmul<false>(o1, w16(2, INV));  // W8^1
        o2 = mul_mi<INV>(o2);               // W8^2
        o3 = cmul<false>(o3, w16(6, INV));  // W8^3
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

// Physical float2 slot of element i of a column buffer: one float2 of padding after every 32,
// so that the strided writes of the first Stockham stages (stride R float2) and the
// contiguous reads of every stage both spread over all banks.
__device__ __forceinline__ int ph(int i) { return i + (i >> 5); }

// q = x / d, r = x % d for 0 <= x < 2^24 and 0 < d: a float reciprocal estimate that is off by
// at most one, then one integer correction.
__device__ __forceinline__ int fast_div(int x, int d, float rd, int& r) {
    int q = __float2int_rz(__int2float_rn(x) * rd);
    r = x - q * d;
    if (r < 0) {
        --q;
        r += d;
    } else if (r >= d) {
        ++q;
        r -= d;
    }
    return q;
}

// Odd radix R in registers, by the conjugate symmetry of the roots: with a_r = v_r + v_(R-r),
// b_r = v_r - v_(R-r) and W_R^m = c_m - i s_m (c, s = cos, sin of 2 pi m / R),
// out[q] = v_0 + sum_r a_r c_(rq) - i sum_r b_r s_(rq), out[R-q] the same with +i (r, q in
// 1..(R-1)/2; the signs of i swap for the inverse).  w[m] holds W_R^m (forward).  Output q goes
// straight to element d0 + q ns of dst.
template <int R, bool INV>
__device__ __forceinline__ void dft_odd_store(float2 (&v)[R], const float2 (&w)[R], float2* dst, int d0, int ns) {
    constexpr int H = (R - 1) / 2;
    float2 x0 = v[0];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
        const float2 a = cadd(v[r], v[R - r]), b = csub(v[r], v[R - r]);
        v[r] = a;
        v[R - r] = b;
        x0 = cadd(x0, a);
    }
#pragma unroll
    for (int q = 1; q <= H; ++q) {
        float2 A = v[0], B = make_float2(0.f, 0.f);
#pragma unroll
        for (int r = 1; r <= H; ++r) {
            const float2 root = w[(r * q) % R];  // (c, -s)
            A.x = fmaf(v[r].x, root.x, A.x);
            A.y = fmaf(v[r].y, root.x, A.y);
            B.x = fmaf(v[R - r].x, -root.y, B.x);
            B.y = fmaf(v[R - r].y, -root.y, B.y);
        }
        const float2 iB = make_float2(-B.y, B.x);  // i B
        dst[ph(d0 + q * ns)] = INV ? cadd(A, iB) : csub(A, iB);
        dst[ph(d0 + (R - q) * ns)] = INV ? csub(A, iB) : cadd(A, iB);
    }
    dst[ph(d0)] = x0;
}

// One Stockham stage with a register butterfly: L = n / R butterflies per column pair; the
// column pairs are `stride` float2 apart.  `stw` holds this stage's twiddles
// W_(ns R)^(r k) at [k (R - 1) + r - 1] (consecutive butterflies read neighbouring entries),
// `roots` the R roots W_R^m of an odd radix.
template <int R, bool INV>
__device__ __forceinline__ void stage_small(const float2* __restrict__ stw, const float2* __restrict__ roots,
                                            const float2* in, float2* out, int n, int stride, int ns, int pairs,
                                            bool spectrum_mul, float inv_n) {
    const int L = n / R;
    const float rL = 1.0f / static_cast<float>(L), rns = 1.0f / static_cast<float>(ns);
    float2 w[R];
    if constexpr (R != 2 && R != 4 && R != 8 && R != 16) {
#pragma unroll
        for (int m = 0; m < R; ++m) w[m] = roots[m];
    }
    for (int item = threadIdx.x; item < pairs * L; item += blockDim.x) {
        int j, k;
        const int p = fast_div(item, L, rL, j);
        const int jb = fast_div(j, ns, rns, k);
        const float2* src = in + p * stride;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = src[ph(j + r * L)];
            if (spectrum_mul) x = hilbert_bin(x, j + r * L, n, inv_n);
            v[r] = r == 0 ? x : cmul<INV>(x, stw[k * (R - 1) + r - 1]);
        }
        float2* dst = out + p * stride;
        const int d0 = jb * ns * R + k;
        if constexpr (R == 2 || R == 4 || R == 8 || R == 16) {
            dft_small<R, INV>(v);
#pragma unroll
            for (int r = 0; r < R; ++r) dst[ph(d0 + r * ns)] = v[r];
        } else {
            dft_odd_store<R, INV>(v, w, dst, d0, ns);
        }
    }
}

// One Stockham stage of any radix R, each output a direct sum of its R inputs:
// out[(j / ns) ns R + k + q ns] = sum_r in[j + r L] W_n^(r (k n / (ns R) + q L)).  For prime
// factors above 13 only: the roots are evaluated in FP64 as they are needed.
template <bool INV>
__device__ __forceinline__ void stage_generic(const float2* in, float2* out, int n, int stride, int ns, int R,
                                              int pairs, bool spectrum_mul, float inv_n) {
    const int L = n / R;
    const int tw_step = n / (ns * R);
    const float rn = 1.0f / static_cast<float>(n), rL = 1.0f / static_cast<float>(L),
                rns = 1.0f / static_cast<float>(ns);
    for (int item = threadIdx.x; item < pairs * n; item += blockDim.x) {
        int rest, j, k;
        const int p = fast_div(item, n, rn, rest);
        const int q = fast_div(rest, L, rL, j);
        const int jb = fast_div(j, ns, rns, k);
        const float2* src = in + p * stride;
        const int step = k * tw_step + q * L;  // < n
        int e = 0;
        float2 acc = make_float2(0.f, 0.f);
        for (int r = 0; r < R; ++r) {
            float2 x = src[ph(j + r * L)];
            if (spectrum_mul) x = hilbert_bin(x, j + r * L, n, inv_n);
            double sn, cs;
            sincospi(-2.0 * e / n, &sn, &cs);
            acc = cadd(acc, cmul<INV>(x, make_float2(static_cast<float>(cs), static_cast<float>(sn))));
            e += step;
            if (e >= n) e -= n;
        }
        out[p * stride + ph(jb * ns * R + k + q * ns)] = acc;
    }
}

// Full transform of `pairs` columns of length n; the result ends in `a` (buffers swap per stage).
// ODD: the plan has odd radices (their register butterflies cost registers that power-of-two
// plans do not need).
template <bool INV, bool ODD>
__device__ void fft_columns(const HilbertArgs& g, const float2* stw_all, const float2* roots_all, float2*& a, float2*& b,
                            int pairs, bool spectrum_mul) {
    int ns = 1, roots_at = 0;
    const int n = g.n, st = g.pair_stride;
    for (int s = 0; s < g.n_stages; ++s) {
        const int R = g.radix[s];
        const bool mul = spectrum_mul && s == 0;
        const float2* tw = stw_all + (ns - 1);
        const float2* roots = roots_all + roots_at;
        if (R <= kHilMaxRegisterRadix && (R & 1)) roots_at += R;
        if (R == 16) {
            stage_small<16, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n);
        } else if (R == 8) {
            stage_small<8, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n);
        } else if (R == 4) {
            stage_small<4, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n);
        } else if (R == 2) {
            stage_small<2, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n);
        } else if constexpr (ODD) {
            switch (R) {
                case 3: stage_small<3, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n); break;
                case 5: stage_small<5, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n); break;
                case 7: stage_small<7, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n); break;
                case 11: stage_small<11, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n); break;
                case 13: stage_small<13, INV>(tw, roots, a, b, n, st, ns, pairs, mul, g.inv_n); break;
                default: stage_generic<INV>(a, b, n, st, ns, R, pairs, mul, g.inv_n); break;
            }
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

constexpr int kHilPrefetch = 32;  // samples per thread of the next group held in registers

// Sample (k, s) of element idx of a group walk: column-fastest or sample-fastest.
__device__ __forceinline__ void group_element(int idx, bool cols_fast, int lc, int n, float rn, int& k, int& s) {
    if (cols_fast) {
        k = idx & ((1 << lc) - 1);
        s = idx >> lc;
    } else {
        k = fast_div(idx, n, rn, s);
    }
}

// Persistent loop over column groups.  While a group is transformed, the next group's samples
// (up to kHilPrefetch per thread) are already on their way from HBM into registers; the
// group's own samples wait in shared memory (xs) for the output phase, which writes
// z = x + i y.  Jobs too long for xs re-read x from global memory (L2) instead.
template <typename In, typename Out, bool ODD>
__global__ void __launch_bounds__(kHilThreads, 2) hilbert_kernel(const HilbertArgs g) {
    extern __shared__ float2 hil_smem[];
    __shared__ int64_t src_off[2][kHilMaxCols], dst_off[2][kHilMaxCols];
    const int n = g.n;
    const int lc = g.cols_log2, C = 1 << lc, P = C >> 1;
    const int st = g.pair_stride;
    const int total = C * n;
    const float rn = 1.0f / static_cast<float>(n);
    float2* stw = hil_smem;        // [n]: stage s at ns_s - 1, entry (k, r) at k (R - 1) + r - 1
    float2* roots = hil_smem + n;  // [kHilRoots]: W_R^m of each odd register radix
    float2* buf0 = roots + kHilRoots;
    float2* buf1 = buf0 + P * st;
    float* xs = reinterpret_cast<float*>(buf1 + P * st);  // [C n] when g.x_in_smem
    {
        int ns = 1, roots_at = 0;
        for (int s = 0; s < g.n_stages; ++s) {
            const int R = g.radix[s], count = ns * (R - 1);
            for (int i = threadIdx.x; i < count; i += blockDim.x) {
                const int k = i / (R - 1), r = i - k * (R - 1) + 1;
                double sn, cs;
                sincospi(-2.0 * (r * k) / (ns * R), &sn, &cs);
                stw[ns - 1 + i] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
            }
            if (R <= kHilMaxRegisterRadix && (R & 1)) {
                for (int m = threadIdx.x; m < R; m += blockDim.x) {
                    double sn, cs;
                    sincospi(-2.0 * m / R, &sn, &cs);
                    roots[roots_at + m] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
                }
                roots_at += R;
            }
            ns *= R;
        }
    }
    const In* src = static_cast<const In*>(g.src);
    Out* dst = static_cast<Out*>(g.dst);
    const int64_t n_groups = (g.n_cols + C - 1) >> lc;
    const bool lfast = g.load_cols_fast != 0, sfast = g.store_cols_fast != 0;
    auto set_offsets = [&](int64_t grp, int slot) {
        if (threadIdx.x < C) {
            const int64_t c = (grp << lc) + threadIdx.x;
            src_off[slot][threadIdx.x] = c < g.n_cols ? column_offset(c, g, g.src_stride) : -1;
            dst_off[slot][threadIdx.x] = c < g.n_cols ? column_offset(c, g, g.dst_stride) : -1;
        }
    };
    In pre[kHilPrefetch];  // raw: widened only when written to shared memory
    auto prefetch = [&](int slot) {
#pragma unroll
        for (int i = 0; i < kHilPrefetch; ++i) {
            const int idx = threadIdx.x + i * kHilThreads;
            pre[i] = In{};
            if (idx < total) {
                int k, s;
                group_element(idx, lfast, lc, n, rn, k, s);
                const int64_t off = src_off[slot][k];
                if (off >= 0) pre[i] = RealIn<In>::raw(src + off + s * g.src_sample);
            }
        }
    };
    int64_t grp = blockIdx.x;
    if (grp < n_groups) set_offsets(grp, 0);
    __syncthreads();
    if (grp < n_groups) prefetch(0);
    for (int it = 0; grp < n_groups; grp += gridDim.x, ++it) {
        const int cur = it & 1;
        const int64_t next = grp + gridDim.x;
        if (next < n_groups) set_offsets(next, cur ^ 1);
        // registers (and, past kHilPrefetch per thread, direct loads) -> column buffers and xs
#pragma unroll
        for (int i = 0; i < kHilPrefetch; ++i) {
            const int idx = threadIdx.x + i * kHilThreads;
            if (idx < total) {
                int k, s;
                group_element(idx, lfast, lc, n, rn, k, s);
                const float x = RealIn<In>::widen(pre[i]);
                reinterpret_cast<float*>(buf0 + (k >> 1) * st)[2 * ph(s) + (k & 1)] = x;
                if (g.x_in_smem) xs[lfast ? s * C + k : k * n + s] = x;
            }
        }
        for (int idx = threadIdx.x + kHilPrefetch * kHilThreads; idx < total; idx += kHilThreads) {
            int k, s;
            group_element(idx, lfast, lc, n, rn, k, s);
            const int64_t off = src_off[cur][k];
            const float x = off >= 0 ? RealIn<In>::get(src + off + s * g.src_sample) : 0.f;
            reinterpret_cast<float*>(buf0 + (k >> 1) * st)[2 * ph(s) + (k & 1)] = x;
            if (g.x_in_smem) xs[lfast ? s * C + k : k * n + s] = x;
        }
        __syncthreads();
        if (next < n_groups) prefetch(cur ^ 1);  // in flight during the transforms
        float2* a = buf0;
        float2* b = buf1;
        fft_columns<false, ODD>(g, stw, roots, a, b, P, false);
        if (g.n_stages == 0) {  // n == 1: the imaginary part is zero
            for (int p = threadIdx.x; p < P; p += blockDim.x) a[p * st] = make_float2(0.f, 0.f);
            __syncthreads();
        } else {
            fft_columns<true, ODD>(g, stw, roots, a, b, P, true);
        }
        for (int idx = threadIdx.x; idx < total; idx += kHilThreads) {
            int k, s;
            group_element(idx, sfast, lc, n, rn, k, s);
            const int64_t doff = dst_off[cur][k];
            if (doff < 0) continue;
            const float x = g.x_in_smem ? xs[lfast ? s * C + k : k * n + s] : RealIn<In>::get(src + src_off[cur][k] + s * g.src_sample);
            const float y = reinterpret_cast<const float*>(a + (k >> 1) * st)[2 * ph(s) + (k & 1)];
            ComplexOut<Out>::put(dst + 2 * (doff + s * g.dst_sample), x * g.scale, y * g.scale);
        }
        __syncthreads();
    }
}

template <typename In, typename Out>
cudaError_t hilbert_typed(const HilbertArgs& g, size_t smem, cudaStream_t st) {
    bool odd = false;
    for (int s = 0; s < g.n_stages; ++s) odd = odd || (g.radix[s] & (g.radix[s] - 1)) != 0;
    auto k = odd ? hilbert_kernel<In, Out, true> : hilbert_kernel<In, Out, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&device)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kHilThreads, smem)) != cudaSuccess) return e;
    const int64_t groups = (g.n_cols + (int64_t{1} << g.cols_log2) - 1) >> g.cols_log2;
    const int64_t resident = static_cast<int64_t>(std::max(1, per_sm)) * sms;
    const int blocks = static_cast<int>(groups < resident ? groups : resident);
    k<<<blocks, kHilThreads, smem, st>>>(g);
    return cudaGetLastError();
}

template <typename In>
cudaError_t hilbert_to(int dst_code, const HilbertArgs& g, size_t smem, cudaStream_t st) {
    switch (dst_code) {
        case kC64: return hilbert_typed<In, float>(g, smem, st);
        case kCF16: return hilbert_typed<In, __half>(g, smem, st);
        case kCBF16: return hilbert_typed<In, __nv_bfloat16>(g, smem, st);
        default: return hilbert_typed<In, short>(g, smem, st);
    }
}

}  // namespace

int hilbert_plan(int n, int* radix, int max_stages) {
    int count = 0, m = n;
    for (int r : {16, 8, 4, 2}) {
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

cudaError_t launch_hilbert(int src_code, int dst_code, const HilbertArgs& g, size_t smem, cudaStream_t st) {
    switch (src_code) {
        case kF32: return hilbert_to<float>(dst_code, g, smem, st);
        case kF16: return hilbert_to<__half>(dst_code, g, smem, st);
        case kBF16: return hilbert_to<__nv_bfloat16>(dst_code, g, smem, st);
        default: return hilbert_to<short>(dst_code, g, smem, st);
    }
}

}  // namespace mach_b200
