// Device-side building blocks of the mach_b200 delay-and-sum gather kernels.
//
// Arithmetic that decides WHICH samples are read and at WHAT fractional position
// (aperture test, delay, sample index, interpolation taps, phase) is written with
// explicit IEEE intrinsics in the operation order of mach's kernel, so the FP32
// results agree with the reference bit for bit (src/mach/kernel.cu:444-483,
// 583, 634-661; interpolation 106-252).  That order is part of the contract: a
// one-ulp change in the delay moves the IQ phase by ~1e-4 rad.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mach_b200 {

enum StorageCode : int {
    kF32 = 0,    // real float32 RF            (reference: float overload)
    kC64 = 1,    // complex64 IQ               (reference: complex<float> overload)
    kF16 = 2,    // real binary16
    kCF16 = 3,   // complex binary16 (I, Q)
    kBF16 = 4,   // real bfloat16
    kCBF16 = 5,  // complex bfloat16 (I, Q)
    kI16 = 6,    // real int16 (times a scale)
    kCI16 = 7,   // complex int16 (I, Q) (times a scale)
};

enum InterpCode : int { kNearest = 0, kLinear = 1, kQuadratic = 2 };

// pi as the reference spells it (src/mach/kernel.cu:67-68), a float literal.
constexpr float kPi = 3.14159265358979323846f;

// ---------------------------------------------------------------------------
// Storage traits: read one sample and widen it to FP32 (I in .x, Q in .y).
// ---------------------------------------------------------------------------
template <int S>
struct Storage;

template <>
struct Storage<kF32> {
    using T = float;
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const T* p) { return make_float2(__ldg(p), 0.f); }
};
template <>
struct Storage<kC64> {
    using T = float2;
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float2 load(const T* p) { return __ldg(p); }
};
template <>
struct Storage<kF16> {
    using T = __half;
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const T* p) {
        return make_float2(__half2float(__ldg(p)), 0.f);
    }
};
template <>
struct Storage<kCF16> {
    using T = __half2;
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float2 load(const T* p) { return __half22float2(__ldg(p)); }
};
template <>
struct Storage<kBF16> {
    using T = __nv_bfloat16;
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const T* p) {
        return make_float2(__bfloat162float(__ldg(p)), 0.f);
    }
};
template <>
struct Storage<kCBF16> {
    using T = __nv_bfloat162;
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float2 load(const T* p) {
        return __bfloat1622float2(__ldg(p));
    }
};
template <>
struct Storage<kI16> {
    using T = short;
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const T* p) {
        return make_float2(static_cast<float>(__ldg(p)), 0.f);
    }
};
template <>
struct Storage<kCI16> {
    using T = short2;
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float2 load(const T* p) {
        const short2 v = __ldg(p);
        return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    }
};

// ---------------------------------------------------------------------------
// Launch parameters (passed by value as a __grid_constant__).
// ---------------------------------------------------------------------------
struct DasArgs {
    const void* channel;    // [n_tx][n_rx][n_samples][n_frames] samples of the storage type
    const float* rx;        // [n_rx][3] element positions (m)
    const float* scan;      // [n_vox][3] voxel positions (m)
    const float* arrivals;  // [n_tx][n_vox] transmit arrival times (s)
    void* out;              // [n_vox][n_frames] float or float2
    int64_t n_vox;
    int32_t n_tx, n_rx, n_samples, n_frames;
    int64_t row_stride;     // n_samples * n_frames (samples per element row)
    float inv_c;            // 1.0f / c, rounded on the host as the reference does (kernel.cu:750)
    float fs;               // sampling frequency
    float t0;               // rx_start_s
    float two_f_number;     // 2.0f * f_number (exact doubling)
    float alpha;            // Tukey alpha
    float one_minus_alpha;  // 1.0f - alpha, as kernel.cu:341 evaluates it
    float mod_rad;          // (2.0f * pi) * f_mod rounded in FP32 (kernel.cu:571)
    float scale;            // storage dequantisation scale (1 for float storage)
    float hi_nearest;       // float(n_samples) - 0.5f   (kernel.cu:118)
    float hi_linear;        // float(n_samples - 1)      (kernel.cu:157)
    float hi_quadratic;     // float(n_samples) - 2.0f   (kernel.cu:208)
    int32_t apod;           // tukey_alpha > 0 (kernel.cu:749)
    int32_t rotate;         // complex storage and f_mod != 0 (kernel.cu:653)
    int32_t accumulate;     // out += result (reference semantics) instead of out = result
    int32_t frame_passes;   // frames handled per lane (multi-frame kernel)
    int32_t tx_chunk;       // transmits whose arrivals are staged in shared memory at once
    // Split-delay mode: sample positions and phases formed in FP64 per (voxel, element) and
    // per (voxel, transmit), each split into an integer sample base + FP32 fraction.
    int32_t split;
    int32_t power;          // ensemble kernel: out is float [n_vox], += sum over frames of |x|^2
    // Lane-voxel kernels on a known grid: map_fast = voxels along the contiguous axis,
    // map_outer = n_vox / map_fast, a warp takes 2^map_wlog of them along the contiguous axis;
    // map_fast = 0: tiles of 128 consecutive voxels.
    int32_t map_fast;
    int32_t map_wlog;
    int64_t map_outer;
    // tile_rev = 1: tiles in fast-axis-major order from the far end of the contiguous axis (the
    // deepest first for a depth-fastest scan, whose wide apertures make them the heaviest), so the
    // CTAs that start last take light tiles; 0: grid order (outer-major).
    int32_t tile_rev;
    int32_t frame_chunks;   // lane-voxel 8-frame chunks: CTA b takes tile b / frame_chunks, chunk b % frame_chunks
    int32_t e_begin;        // lane-voxel kernels: elements [e_begin, e_end) of this launch
    int32_t e_end;
    int32_t start_base;     // floor(-t0 * fs): samples before it belong to tau < 0
    float start_frac;       // -t0 * fs - start_base
    double fs_d;            // sampling frequency
    double t0_d;            // rx_start_s
    double fmod_d;          // modulation frequency
    double fs_over_c;       // fs / c
    double fmod_over_c;     // f_mod / c
};

// Integer base + FP32 fraction in [0, 1) of a non-negative-or-negative FP64 sample position.
struct SplitPos {
    int base;
    float frac;
};

__device__ __forceinline__ SplitPos split_position(double s) {
    const double b = floor(s);
    SplitPos p{static_cast<int>(b), static_cast<float>(s - b)};
    if (p.frac >= 1.0f) {  // s - b rounded up to 1.0f
        p.frac = 0.0f;
        p.base += 1;
    }
    return p;
}

// Fractional revolutions in [-0.5, 0.5] of an FP64 phase measured in cycles.
__device__ __forceinline__ float reduced_cycles(double cycles) {
    return static_cast<float>(cycles - rint(cycles));
}

// Half-Tukey weight of r = horizontal distance / aperture radius (kernel.cu:333-349).
__device__ __forceinline__ float tukey_weight(float r, float alpha, float one_minus_alpha) {
    if ((r < 0.0f) || (r > 1.0f)) return 0.0f;
    if (r <= one_minus_alpha) return 1.0f;
    const float mirror = __fsub_rn(1.0f, r);
    return __fmaf_rn(-0.5f, cosf(__fdiv_rn(__fmul_rn(kPi, mirror), alpha)), 0.5f);
}

// Receive path of one (voxel, element) pair: distance, apodisation weight and the
// aperture test (kernel.cu:444-483).  Independent of the transmit, so it is
// computed once and reused for every transmit and frame.
__device__ __forceinline__ void receive_path(const DasArgs& a, float ex, float ey, float ez, float vx,
                                             float vy, float vz, float radius, float radius_sq,
                                             float& dist, float& weight, bool& in_aperture) {
    const float dx = __fsub_rn(ex, vx);
    const float dy = __fsub_rn(ey, vy);
    const float dz = __fsub_rn(ez, vz);
    const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    in_aperture = !(h2 > radius_sq);
    dist = __fsqrt_rn(__fmaf_rn(dz, dz, h2));
    weight = 1.0f;
    if (a.apod) {
        weight = tukey_weight(__fdiv_rn(__fsqrt_rn(h2), radius), a.alpha, a.one_minus_alpha);
    }
}

// Transmit part: delay tau (kernel.cu:470) and the fractional sample index (kernel.cu:637).
// Returns false when the pair is skipped (kernel.cu:634) or the taps leave the row.
template <int INTERP>
__device__ __forceinline__ bool sample_position(const DasArgs& a, float dist, float tx_arrival,
                                                float& tau, float& s) {
    tau = __fmaf_rn(dist, a.inv_c, tx_arrival);
    if (tau < 0.0f) return false;
    s = __fmul_rn(__fsub_rn(tau, a.t0), a.fs);
    if constexpr (INTERP == kNearest) {
        if (!((s >= -0.5f) && (s <= a.hi_nearest))) return false;
        // round-half-even may reach n_samples when n_samples is even; that index is out of the row.
        return __float2uint_rn(s) < static_cast<unsigned>(a.n_samples);
    } else if constexpr (INTERP == kLinear) {
        return (s >= 0.0f) && (s <= a.hi_linear);
    } else {
        return (s >= 1.0f) && (s <= a.hi_quadratic);
    }
}

// Interpolate one frame at fractional sample s from `row` (samples strided by n_frames),
// following kernel.cu:106-252: nearest rounds half to even; linear is a + t (b - a);
// quadratic is the 3-tap Lagrange form around rint(s).
template <int S, int INTERP>
__device__ __forceinline__ float2 interpolate(const typename Storage<S>::T* row, float s,
                                              int64_t n_frames) {
    using ST = Storage<S>;
    if constexpr (INTERP == kNearest) {
        const unsigned idx = __float2uint_rn(s);
        return ST::load(row + static_cast<int64_t>(idx) * n_frames);
    } else if constexpr (INTERP == kLinear) {
        const unsigned i0 = __float2uint_rd(s);
        const unsigned i1 = __float2uint_ru(s);
        const float t = __fsub_rn(s, static_cast<float>(i0));
        const float2 lo = ST::load(row + static_cast<int64_t>(i0) * n_frames);
        const float2 hi = ST::load(row + static_cast<int64_t>(i1) * n_frames);
        float2 r;
        r.x = __fmaf_rn(t, __fsub_rn(hi.x, lo.x), lo.x);
        r.y = ST::kComplex ? __fmaf_rn(t, __fsub_rn(hi.y, lo.y), lo.y) : 0.f;
        return r;
    } else {
        const unsigned c = __float2uint_rn(s);
        const float x = __fsub_rn(s, static_cast<float>(c));
        const float hx = __fmul_rn(0.5f, x);
        const float wm = __fmul_rn(hx, __fsub_rn(x, 1.0f));
        const float w0 = __fmul_rn(__fsub_rn(1.0f, x), __fadd_rn(1.0f, x));
        const float wp = __fmul_rn(hx, __fadd_rn(x, 1.0f));
        const typename ST::T* p = row + static_cast<int64_t>(c) * n_frames;
        const float2 dm = ST::load(p - n_frames);
        const float2 d0 = ST::load(p);
        const float2 dp = ST::load(p + n_frames);
        float2 r;
        r.x = __fmaf_rn(wp, dp.x, __fmaf_rn(wm, dm.x, __fmul_rn(w0, d0.x)));
        r.y = ST::kComplex ? __fmaf_rn(wp, dp.y, __fmaf_rn(wm, dm.y, __fmul_rn(w0, d0.y))) : 0.f;
        return r;
    }
}

}  // namespace mach_b200
