// Voxel-per-lane gather kernel: one lane owns one voxel and all of its frames (1..8).
//
// Used for single-frame and few-frame jobs (plane-wave compounding, 2-D/3-D B-mode),
// where the work per (voxel, element, transmit) point is the delay arithmetic itself
// and the kernel is bound by instruction issue.  The structure keeps that work minimal:
//   * transmit arrival times of the CTA's 128 voxels are staged in shared memory once per
//     transmit chunk (one coalesced pass), so the inner loop reads them with one LDS;
//   * the receive path of a (voxel, element) pair -- distance, Tukey weight, aperture test --
//     is computed once and reused for every transmit of the chunk;
//   * elements are skipped per warp when no voxel of the warp can see them (bounding box
//     of the warp's 32 voxels against the f-number aperture, exact test per pair after);
//   * sample positions use FP32 add-with-rounding against 1.5 * 2^23 instead of float/int
//     conversions (those run on the quarter-rate XU pipe, already busy with sincos);
//   * for one frame the interpolation taps are adjacent, addressed by immediate offsets.
// Results stay in registers across elements and transmits; `out` is written once.
#pragma once

#include "das_device.cuh"

namespace mach_b200 {

constexpr int kLaneVoxelThreads = 128;
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23: x + magic has ulp 1 for 0 <= x < 2^22
constexpr int kRoundMagicBits = 0x4B400000;

// Sample position of one (voxel, element, transmit) point: integer tap index and
// interpolation weights, identical to mach's float/uint conversions (kernel.cu:125, 160-162,
// 214) for 0 <= s < 2^22.
struct TapPosition {
    int idx;   // nearest: the sample; linear: floor(s); quadratic: rint(s)
    float w0;  // linear: fraction t; quadratic: weight of idx - 1
    float w1;  // quadratic: weight of idx
    float w2;  // quadratic: weight of idx + 1
    int step;  // linear: 1 when t > 0 (ceil != floor), else 0
};

template <int INTERP>
__device__ __forceinline__ TapPosition tap_position(float s) {
    TapPosition p{};
    if constexpr (INTERP == kLinear) {
        const float r = __fadd_rd(s, kRoundMagic);
        p.idx = __float_as_int(r) - kRoundMagicBits;
        p.w0 = __fsub_rn(s, __fsub_rn(r, kRoundMagic));  // s - floor(s), exact
        p.step = p.w0 > 0.0f ? 1 : 0;
    } else {
        const float r = __fadd_rn(s, kRoundMagic);  // round half to even
        p.idx = __float_as_int(r) - kRoundMagicBits;
        if constexpr (INTERP == kQuadratic) {
            const float x = __fsub_rn(s, __fsub_rn(r, kRoundMagic));
            const float hx = __fmul_rn(0.5f, x);
            const float q = __fmul_rn(hx, x);
            p.w0 = __fsub_rn(q, hx);              // x (x - 1) / 2
            p.w1 = __fmaf_rn(-2.0f, q, 1.0f);     // (1 - x)(1 + x)
            p.w2 = __fadd_rn(q, hx);              // x (x + 1) / 2
        }
    }
    return p;
}

// Split-delay sample position: base + frac with frac in [0, 1).  Applies mach's bounds
// (kernel.cu:117, 156, 208) to s = base + frac exactly and rounds half to even.
template <int INTERP>
__device__ __forceinline__ bool split_tap_position(int base, float frac, int n_samples, TapPosition& tp) {
    if constexpr (INTERP == kLinear) {
        if (base < 0 || base > n_samples - 1 || (base == n_samples - 1 && frac != 0.0f)) return false;
        tp.idx = base;
        tp.w0 = frac;
        tp.step = frac > 0.0f ? 1 : 0;
        return true;
    } else {
        const int up = (frac > 0.5f || (frac == 0.5f && (base & 1))) ? 1 : 0;
        tp.idx = base + up;
        if constexpr (INTERP == kNearest) {
            return tp.idx >= 0 && tp.idx < n_samples;
        } else {
            if (base < 1 || base > n_samples - 2 || (base == n_samples - 2 && frac != 0.0f)) return false;
            const float x = __fsub_rn(frac, static_cast<float>(up));  // exact
            const float hx = __fmul_rn(0.5f, x);
            const float q = __fmul_rn(hx, x);
            tp.w0 = __fsub_rn(q, hx);
            tp.w1 = __fmaf_rn(-2.0f, q, 1.0f);
            tp.w2 = __fadd_rn(q, hx);
            return true;
        }
    }
}

// Phase of a split-delay point: cycles in [-1, 1] reduced to [-0.5, 0.5], then the fast
// sincos on an argument within [-pi, pi] (its accurate range).
__device__ __forceinline__ void split_phasor(float cycles, float& sn, float& cs) {
    const float whole = __fsub_rn(__fadd_rn(cycles, kRoundMagic), kRoundMagic);
    __sincosf(__fmul_rn(__fsub_rn(cycles, whole), 6.28318530717958647f), &sn, &cs);
}

// Interpolated sample at `row[idx * stride]` (stride = frames), widened to FP32.  PACKED:
// complex quadratic taps in packed FP32x2, the same operations and order as the scalar form.
template <int S, int INTERP, bool PACKED = false>
__device__ __forceinline__ float2 tap_value(const typename Storage<S>::T* p, const TapPosition& tp, int stride) {
    using ST = Storage<S>;
    if constexpr (INTERP == kNearest) {
        return ST::load(p);
    } else if constexpr (INTERP == kLinear) {
        const float2 a = ST::load(p);
        const float2 b = ST::load(p + tp.step * stride);
        float2 r;
        r.x = __fmaf_rn(tp.w0, __fsub_rn(b.x, a.x), a.x);  // a + t (b - a), mach's lerp form
        r.y = ST::kComplex ? __fmaf_rn(tp.w0, __fsub_rn(b.y, a.y), a.y) : 0.f;
        return r;
    } else {
        const float2 a = ST::load(p - stride);
        const float2 b = ST::load(p);
        const float2 c = ST::load(p + stride);
        if constexpr (PACKED && ST::kComplex) {
            return __ffma2_rn(make_float2(tp.w2, tp.w2), c,
                              __ffma2_rn(make_float2(tp.w0, tp.w0), a, __fmul2_rn(make_float2(tp.w1, tp.w1), b)));
        }
        float2 r;
        r.x = __fmaf_rn(tp.w2, c.x, __fmaf_rn(tp.w0, a.x, __fmul_rn(tp.w1, b.x)));
        r.y = ST::kComplex ? __fmaf_rn(tp.w2, c.y, __fmaf_rn(tp.w0, a.y, __fmul_rn(tp.w1, b.y))) : 0.f;
        return r;
    }
}

// ---- vectorised frames (NF frames contiguous per sample, 16-byte aligned rows) ----

// float2 pairs holding NF frames: complex storage one pair per frame, real two frames per pair.
template <int S, int NF>
struct FramePairs {
    static constexpr int kValue = Storage<S>::kComplex ? NF : NF / 2;
};

// Widen 8 bytes of storage S into float2 pairs (same packing as the staged kernel's lanes).
template <int S>
__device__ __forceinline__ void widen8(uint2 r, float2* o);
template <>
__device__ __forceinline__ void widen8<kC64>(uint2 r, float2* o) {
    o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
}
template <>
__device__ __forceinline__ void widen8<kF32>(uint2 r, float2* o) {
    o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
}
template <>
__device__ __forceinline__ void widen8<kCF16>(uint2 r, float2* o) {
    o[0] = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    o[1] = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
}
template <>
__device__ __forceinline__ void widen8<kF16>(uint2 r, float2* o) {
    widen8<kCF16>(r, o);
}
template <>
__device__ __forceinline__ void widen8<kCBF16>(uint2 r, float2* o) {
    o[0] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.x));
    o[1] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.y));
}
template <>
__device__ __forceinline__ void widen8<kBF16>(uint2 r, float2* o) {
    widen8<kCBF16>(r, o);
}
// int16 pair of a 32-bit word -> exact floats without the conversion pipe: x + 32768 is
// placed in the mantissa of 2^23 (bit pattern 0x4B000000 | (x + 32768)) and 2^23 + 32768
// subtracted.  Low sample: (w & 0xFFFF) ^ 0x4B008000 (one LOP3); high sample: the arithmetic
// shift w >> 16 added to 0x4B008000 (measured on B200: 3-D 16 frames 67.2 -> 66.9 ms, Doppler
// int16 3.25 -> 3.20 ms against byte permutes of w ^ 0x80008000).
__device__ __forceinline__ float2 widen_i16x2(unsigned w) {
    const unsigned lo = (w & 0xFFFFu) ^ 0x4B008000u;
    const unsigned hi = static_cast<unsigned>(static_cast<int>(w) >> 16) + 0x4B008000u;
    return __fadd2_rn(make_float2(__uint_as_float(lo), __uint_as_float(hi)),
                      make_float2(-8421376.0f, -8421376.0f));  // exact
}
template <>
__device__ __forceinline__ void widen8<kCI16>(uint2 r, float2* o) {
    o[0] = widen_i16x2(r.x);
    o[1] = widen_i16x2(r.y);
}
template <>
__device__ __forceinline__ void widen8<kI16>(uint2 r, float2* o) {
    widen8<kCI16>(r, o);
}

// Load the NF frames of one sample (NF * sizeof(T) is a multiple of 16 bytes).  Rows of a
// multiple of 32 bytes are read with 256-bit loads, so that each lane's request covers whole
// 32-byte sectors (the planner only runs them on 32-byte aligned rows; measured on B200:
// Doppler complex64 in 8-frame chunks 5.7 -> 4.0 ms, FP16 3.45 -> 3.30 ms); others with
// 128-bit loads.
template <int S, int NF>
__device__ __forceinline__ void load_frames(const typename Storage<S>::T* p, float2* o) {
    constexpr int kBytes = NF * static_cast<int>(sizeof(typename Storage<S>::T));
    static_assert(kBytes % 16 == 0, "vector frames need 16-byte rows");
    constexpr int kPairsPer8 = FramePairs<S, NF>::kValue / (kBytes / 8);
    if constexpr (kBytes % 32 == 0) {
#pragma unroll
        for (int i = 0; i < kBytes / 32; ++i) {
            unsigned r[8];
            asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "l"(reinterpret_cast<const char*>(p) + 32 * i));
#pragma unroll
            for (int k = 0; k < 4; ++k) widen8<S>(make_uint2(r[2 * k], r[2 * k + 1]), o + (4 * i + k) * kPairsPer8);
        }
    } else {
        const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < kBytes / 16; ++i) {
            const uint4 r = __ldg(q + i);
            widen8<S>(make_uint2(r.x, r.y), o + (2 * i) * kPairsPer8);
            widen8<S>(make_uint2(r.z, r.w), o + (2 * i + 1) * kPairsPer8);
        }
    }
}

// Raw 32-bit words of the NF frames of one sample (NF * sizeof(T) bytes, a multiple of 16;
// 256-bit loads when a multiple of 32, as load_frames).
template <int S, int NF>
__device__ __forceinline__ void load_words(const typename Storage<S>::T* p, unsigned* w) {
    constexpr int kBytes = NF * static_cast<int>(sizeof(typename Storage<S>::T));
    static_assert(kBytes % 16 == 0, "vector frames need 16-byte rows");
    if constexpr (kBytes % 32 == 0) {
#pragma unroll
        for (int i = 0; i < kBytes / 32; ++i) {
            unsigned* r = w + 8 * i;
            asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "l"(reinterpret_cast<const char*>(p) + 32 * i));
        }
    } else {
        const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < kBytes / 16; ++i) {
            const uint4 r = __ldg(q + i);
            w[4 * i] = r.x;
            w[4 * i + 1] = r.y;
            w[4 * i + 2] = r.z;
            w[4 * i + 3] = r.w;
        }
    }
}

// Linear interpolation a + t (b - a) of one complex FP16 / BF16 sample pair (I, Q in one
// 32-bit word each for a and b), in FP32.  b - a is formed by the mixed-precision subtract
// (16-bit operand widened exactly inside the instruction), so only a is converted: the
// result is bit-identical to widening both and subtracting in FP32.
template <int S>
__device__ __forceinline__ float2 lerp_half_word(unsigned wa, unsigned wb, float t) {
    float2 r;
    if constexpr (S == kCF16) {
        asm("{\n\t.reg .b16 al, ah, bl, bh;\n\t.reg .f32 fa, fb, da, db;\n\t"
            "mov.b32 {al, ah}, %2;\n\tmov.b32 {bl, bh}, %3;\n\t"
            "cvt.f32.f16 fa, al;\n\tcvt.f32.f16 fb, ah;\n\t"
            "sub.rn.f32.f16 da, bl, fa;\n\tsub.rn.f32.f16 db, bh, fb;\n\t"
            "fma.rn.f32 %0, %4, da, fa;\n\tfma.rn.f32 %1, %4, db, fb;\n\t}"
            : "=f"(r.x), "=f"(r.y) : "r"(wa), "r"(wb), "f"(t));
    } else {
        asm("{\n\t.reg .b16 al, ah, bl, bh;\n\t.reg .f32 fa, fb, da, db;\n\t"
            "mov.b32 {al, ah}, %2;\n\tmov.b32 {bl, bh}, %3;\n\t"
            "cvt.f32.bf16 fa, al;\n\tcvt.f32.bf16 fb, ah;\n\t"
            "sub.rn.f32.bf16 da, bl, fa;\n\tsub.rn.f32.bf16 db, bh, fb;\n\t"
            "fma.rn.f32 %0, %4, da, fa;\n\tfma.rn.f32 %1, %4, db, fb;\n\t}"
            : "=f"(r.x), "=f"(r.y) : "r"(wa), "r"(wb), "f"(t));
    }
    return r;
}

// Receive-path Tukey weight.  The weight only scales a sample, so fast intrinsics are used
// (their ~1e-7 error is far inside the 1e-5 parity budget); the aperture decision itself is
// the exact FP32 test of kernel.cu:461.
__device__ __forceinline__ float fast_tukey(float h2, float radius, const DasArgs& a) {
    const float r = __fdividef(__fsqrt_rn(h2), radius);
    if ((r < 0.0f) || (r > 1.0f)) return 0.0f;
    if (r <= a.one_minus_alpha) return 1.0f;
    return __fmaf_rn(-0.5f, __cosf(__fdividef(kPi * (1.0f - r), a.alpha)), 0.5f);
}

// Voxel of thread j (0..127) of lane-voxel tile `tile`, or n_vox for none.  On a known grid a
// warp takes wf = 2^map_wlog neighbours along the contiguous axis times 32 / wf along the next
// one (a CTA wf x 128 / wf), so that the sample rows the 32 lanes of a load read lie close
// together in memory (few L1 lines per warp load); otherwise a tile is 128 consecutive voxels.
template <int VPC = kLaneVoxelThreads>
__device__ __forceinline__ int64_t lane_voxel_index(const DasArgs& a, int64_t tile, int j) {
    if (a.map_fast <= 0) return tile * VPC + j;
    const int lw = a.map_wlog;
    const int64_t tiles_fast = (a.map_fast + (1 << lw) - 1) >> lw;
    const int64_t per_outer = VPC >> lw;  // outer-axis voxels of a tile
    int64_t to, tf;                        // the tile's outer and fast-axis tile coordinates
    if (a.tile_rev) {
        const int64_t tiles_outer = (a.map_outer + per_outer - 1) / per_outer;
        const int64_t q = tile / tiles_outer;
        to = tile - q * tiles_outer;
        tf = tiles_fast - 1 - q;
    } else {
        to = tile / tiles_fast;
        tf = tile - to * tiles_fast;
    }
    const int64_t o = to * per_outer + (j >> lw);
    const int64_t f = (tf << lw) + (j & ((1 << lw) - 1));
    return (o < a.map_outer && f < a.map_fast) ? o * a.map_fast + f : a.n_vox;
}

// One CTA tile: voxels [tile * 128, tile * 128 + 128) of job `a`, all its transmits,
// elements and frames.  `smem_words` is the dynamic shared memory (tx_chunk x 128 words,
// x3 in split mode).  Shared by the per-job kernel and the persistent batch kernel.
// CS > 1 (one-frame jobs too small to fill the GPU): CS consecutive lanes share a voxel, each
// summing every CS-th candidate element, and their sums are added with warp shuffles; a CTA
// then covers 128 / CS voxels.
template <int S, int INTERP, int NF, bool SPLIT, int CS = 1>
__device__ __forceinline__ void lane_voxel_tile(const DasArgs& a, int64_t tile, float* smem_words, int chunk = 0) {
    static_assert(CS == 1 || NF == 1, "channel split: one-frame jobs only");
    using ST = Storage<S>;
    using T = typename ST::T;
    constexpr bool kCplx = ST::kComplex;
    constexpr unsigned kFull = 0xffffffffu;
    // [tx_chunk][kLaneVoxelThreads] arrivals; split mode: sample base, fraction, phase cycles
    float* const s_arrival = smem_words;
    int* const s_base = reinterpret_cast<int*>(s_arrival + a.tx_chunk * kLaneVoxelThreads);
    float* const s_cyc = s_arrival + 2 * a.tx_chunk * kLaneVoxelThreads;

    const int lane = threadIdx.x & 31;
    const int sub = threadIdx.x & (CS - 1);  // this lane's share of the voxel's elements
    const int64_t v = lane_voxel_index<kLaneVoxelThreads / CS>(a, tile, threadIdx.x / CS);
    const bool vox_ok = v < a.n_vox;
    const int n_frames = NF > 0 ? NF : a.n_frames;  // frames this thread sums
    // Frames per sample row, and this CTA's first frame: vector jobs with more frames than NF
    // run in chunks of NF frames.
    const int fstride = a.n_frames;
    const int f0 = NF >= 2 ? chunk * NF : 0;

    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (vox_ok) {
        vx = __ldg(a.scan + 3 * v + 0);
        vy = __ldg(a.scan + 3 * v + 1);
        vz = __ldg(a.scan + 3 * v + 2);
    }
    const float radius = __fdiv_rn(vz, a.two_f_number);  // kernel.cu:583
    const float radius_sq = __fmul_rn(radius, radius);

    float bx0 = vox_ok ? vx : INFINITY, bx1 = vox_ok ? vx : -INFINITY;
    float by0 = vox_ok ? vy : INFINITY, by1 = vox_ok ? vy : -INFINITY;
    float rmax = vox_ok ? fabsf(radius) : 0.f;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, off));
        bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, off));
        by0 = fminf(by0, __shfl_xor_sync(kFull, by0, off));
        by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, off));
        rmax = fmaxf(rmax, __shfl_xor_sync(kFull, rmax, off));
    }
    const float cand_r2 = rmax * rmax * 1.00001f + 1e-30f;

    // Vector path: NF frames per sample loaded as 16-byte vectors, accumulated as float2
    // pairs (complex: one frame per pair; real: two frames per pair).
    constexpr bool kVec = NF >= 2 && (NF * static_cast<int>(sizeof(T))) % 16 == 0;
    constexpr int kAcc = kVec ? FramePairs<S, NF>::kValue : (NF > 0 ? NF : 8);
    float2 acc[kAcc];
#pragma unroll
    for (int f = 0; f < kAcc; ++f) acc[f] = make_float2(0.f, 0.f);
    // One-frame complex jobs with FP32 delays: sum(c w x) and sum(s w x) in packed FP32x2; the
    // rotation sum((c + i s) w x) = sum(c w x) + i sum(s w x) is applied once after the loops
    // (compounding complex64 2.00 -> 1.91 ms on B200; with split delays it was slower).
    constexpr bool kDeferRot = NF == 1 && kCplx && !SPLIT;
    float2 acc_c = make_float2(0.f, 0.f), acc_s = make_float2(0.f, 0.f);

    const T* const channel = static_cast<const T*>(a.channel);
    const int row_len = a.n_samples * fstride;  // samples per (transmit, element) row
    const int tx_chunk = a.tx_chunk;

    for (int t0 = 0; t0 < a.n_tx; t0 += tx_chunk) {
        const int nt = min(tx_chunk, a.n_tx - t0);
        __syncthreads();
        for (int i = threadIdx.x; i < nt * kLaneVoxelThreads; i += kLaneVoxelThreads) {
            const int t = i / kLaneVoxelThreads;  // i - t * 128 is this thread's index: its own voxel
            const float txa = vox_ok ? __ldg(a.arrivals + static_cast<int64_t>(t0 + t) * a.n_vox + v) : 0.f;
            if constexpr (SPLIT) {
                // transmit part of the sample position and phase, per (voxel, transmit)
                const SplitPos sp = split_position((static_cast<double>(txa) - a.t0_d) * a.fs_d);
                s_base[i] = sp.base;
                s_arrival[i] = sp.frac;
                s_cyc[i] = reduced_cycles(static_cast<double>(txa) * a.fmod_d);
            } else {
                s_arrival[i] = txa;
            }
        }
        __syncthreads();

        for (int eb = a.e_begin; eb < a.e_end; eb += 32) {
            bool cand = false;
            {
                const int e = eb + lane;
                if (e < a.e_end) {
                    const float ex = __ldg(a.rx + 3 * e + 0);
                    const float ey = __ldg(a.rx + 3 * e + 1);
                    const float ddx = fmaxf(fmaxf(bx0 - ex, ex - bx1), 0.f);
                    const float ddy = fmaxf(fmaxf(by0 - ey, ey - by1), 0.f);
                    cand = ddx * ddx + ddy * ddy <= cand_r2;
                }
            }
            unsigned cmask = __ballot_sync(kFull, cand);
            // CS > 1: lane `sub` of a voxel takes the candidates e with e % CS == sub, so a
            // voxel's partial sums do not depend on which warp (tile) it is in.
            if constexpr (CS > 1) cmask &= (CS == 4 ? 0x11111111u : 0x55555555u) << sub;
            while (CS == 1 ? cmask != 0u : __any_sync(kFull, cmask != 0u)) {
                const bool e_ok = cmask != 0u;
                const int e = eb + (e_ok ? __ffs(cmask) - 1 : 0);
                cmask &= cmask - 1u;

                // Receive path (kernel.cu:444-483), reused for every transmit below.
                const float ex = __ldg(a.rx + 3 * e + 0), ey = __ldg(a.rx + 3 * e + 1), ez = __ldg(a.rx + 3 * e + 2);
                const float dx = __fsub_rn(ex, vx);
                const float dy = __fsub_rn(ey, vy);
                const float dz = __fsub_rn(ez, vz);
                const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                float dist = 0.f;
                SplitPos rx_pos{};
                float rx_cyc = 0.f;
                if constexpr (SPLIT) {
                    const double ddx = static_cast<double>(ex) - vx, ddy = static_cast<double>(ey) - vy,
                                 ddz = static_cast<double>(ez) - vz;
                    const double d = sqrt(fma(ddx, ddx, fma(ddy, ddy, ddz * ddz)));
                    rx_pos = split_position(d * a.fs_over_c);
                    rx_cyc = reduced_cycles(d * a.fmod_over_c);
                } else {
                    dist = __fsqrt_rn(__fmaf_rn(dz, dz, h2));
                }
                float weight = 1.0f;
                if (a.apod) weight = fast_tukey(h2, radius, a);
                const bool pair_ok = vox_ok && e_ok && !(h2 > radius_sq) && !(weight == 0.0f);
                if (!__any_sync(kFull, pair_ok)) continue;
                const float w = __fmul_rn(weight, a.scale);

                int row = (t0 * a.n_rx + e) * row_len;
                const int tx_step = a.n_rx * row_len;
                if constexpr (NF == 1) {
                    if (a.n_samples >= 3) {
                        // Two transmits at a time with no branch between them, so that the
                        // loads of both are in flight together.  A tap that is not taken reads
                        // sample 1 of its row (inside every row) and is not accumulated.
#pragma unroll 1
                        for (int t = 0; t < nt; t += 2, row += 2 * tx_step) {
                            float2 xv[2];
                            float cwv[2], swv[2];
                            bool okv[2];
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                const bool in = t + u < nt;
                                const int si = (in ? t + u : t) * kLaneVoxelThreads + threadIdx.x;
                                TapPosition tp{};
                                bool ok;
                                float cw = w, sw = 0.f;
                                if constexpr (SPLIT) {
                                    int base = s_base[si] + rx_pos.base;
                                    float frac = __fadd_rn(s_arrival[si], rx_pos.frac);
                                    if (frac >= 1.0f) {
                                        frac = __fsub_rn(frac, 1.0f);
                                        base += 1;
                                    }
                                    ok = in && pair_ok &&
                                         !(base < a.start_base || (base == a.start_base && frac < a.start_frac));
                                    const bool inside = split_tap_position<INTERP>(base, frac, a.n_samples, tp);
                                    ok = ok && inside;
                                    if (kCplx && a.rotate) {
                                        float sn, cs;
                                        split_phasor(__fadd_rn(s_cyc[si], rx_cyc), sn, cs);
                                        cw = __fmul_rn(cs, w);
                                        sw = __fmul_rn(sn, w);
                                    }
                                } else {
                                    const float tau = __fmaf_rn(dist, a.inv_c, s_arrival[si]);
                                    const float sp = __fmul_rn(__fsub_rn(tau, a.t0), a.fs);
                                    ok = in && pair_ok && !(tau < 0.0f);
                                    if constexpr (INTERP == kNearest) {
                                        ok = ok && (sp >= -0.5f) && (sp <= a.hi_nearest);
                                    } else if constexpr (INTERP == kLinear) {
                                        ok = ok && (sp >= 0.0f) && (sp <= a.hi_linear);
                                    } else {
                                        ok = ok && (sp >= 1.0f) && (sp <= a.hi_quadratic);
                                    }
                                    tp = tap_position<INTERP>(sp);
                                    if constexpr (INTERP == kNearest) ok = ok && tp.idx < a.n_samples;
                                    if (kCplx && a.rotate) {
                                        float sn, cs;
                                        __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
                                        cw = __fmul_rn(cs, w);
                                        sw = __fmul_rn(sn, w);
                                    }
                                }
                                if (!ok) {
                                    tp.idx = 1;
                                    tp.step = 0;
                                }
                                const int row_u = in ? row + u * tx_step : row;
                                xv[u] = tap_value<S, INTERP, kDeferRot>(channel + (row_u + tp.idx * n_frames), tp, n_frames);
                                cwv[u] = cw;
                                swv[u] = sw;
                                okv[u] = ok;
                            }
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                const float2 x = xv[u];
                                float2 r;
                                if constexpr (kDeferRot) {
                                    if (okv[u]) {
                                        acc_c = __ffma2_rn(make_float2(cwv[u], cwv[u]), x, acc_c);
                                        acc_s = __ffma2_rn(make_float2(swv[u], swv[u]), x, acc_s);
                                    }
                                    continue;
                                } else if constexpr (kCplx) {
                                    r.x = __fmaf_rn(x.x, cwv[u], __fmaf_rn(-x.y, swv[u], acc[0].x));
                                    r.y = __fmaf_rn(x.y, cwv[u], __fmaf_rn(x.x, swv[u], acc[0].y));
                                } else {
                                    r.x = __fmaf_rn(x.x, cwv[u], acc[0].x);
                                    r.y = acc[0].y;
                                }
                                acc[0] = okv[u] ? r : acc[0];
                            }
                        }
                        continue;
                    }
                }
#pragma unroll 2
                for (int t = 0; t < nt; ++t, row += tx_step) {
                    const int si = t * kLaneVoxelThreads + threadIdx.x;
                    TapPosition tp;
                    float cw = w, sw = 0.f;
                    if constexpr (SPLIT) {
                        // s = (tx part) + (receive part), as integer base + FP32 fraction
                        int base = s_base[si] + rx_pos.base;
                        float frac = __fadd_rn(s_arrival[si], rx_pos.frac);
                        if (frac >= 1.0f) {
                            frac = __fsub_rn(frac, 1.0f);
                            base += 1;
                        }
                        // tau < 0  <=>  s < -t0 * fs
                        bool ok = pair_ok && !(base < a.start_base || (base == a.start_base && frac < a.start_frac));
                        ok = ok && split_tap_position<INTERP>(base, frac, a.n_samples, tp);
                        if (!ok) continue;
                        if (kCplx && a.rotate) {
                            float sn, cs;
                            split_phasor(__fadd_rn(s_cyc[si], rx_cyc), sn, cs);
                            cw = __fmul_rn(cs, w);
                            sw = __fmul_rn(sn, w);
                        }
                    } else {
                        const float tau = __fmaf_rn(dist, a.inv_c, s_arrival[si]);
                        const float s = __fmul_rn(__fsub_rn(tau, a.t0), a.fs);
                        bool ok = pair_ok && !(tau < 0.0f);
                        if constexpr (INTERP == kNearest) {
                            ok = ok && (s >= -0.5f) && (s <= a.hi_nearest);
                        } else if constexpr (INTERP == kLinear) {
                            ok = ok && (s >= 0.0f) && (s <= a.hi_linear);
                        } else {
                            ok = ok && (s >= 1.0f) && (s <= a.hi_quadratic);
                        }
                        if (!ok) continue;
                        tp = tap_position<INTERP>(s);
                        if constexpr (INTERP == kNearest) {
                            if (tp.idx >= a.n_samples) continue;
                        }
                        if (kCplx && a.rotate) {
                            float sn, cs;
                            __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
                            cw = __fmul_rn(cs, w);
                            sw = __fmul_rn(sn, w);
                        }
                    }
                    const T* p = channel + (row + tp.idx * fstride + f0);
                    if constexpr (kVec && !kCplx && INTERP != kQuadratic) {
                        // Real frames in pairs: the interpolation weights folded into the
                        // apodisation weight, acc += (1 - t) w a + t w b in packed FP32x2.
                        float2 va[kAcc];
                        load_frames<S, NF>(p, va);
                        if constexpr (INTERP == kLinear) {
                            float2 vb[kAcc];
                            load_frames<S, NF>(p + tp.step * fstride, vb);
                            const float wb = __fmul_rn(tp.w0, cw);
                            const float wa = __fsub_rn(cw, wb);
#pragma unroll
                            for (int q = 0; q < kAcc; ++q) {
                                acc[q] = __ffma2_rn(make_float2(wa, wa), va[q], acc[q]);
                                acc[q] = __ffma2_rn(make_float2(wb, wb), vb[q], acc[q]);
                            }
                        } else {
#pragma unroll
                            for (int q = 0; q < kAcc; ++q) acc[q] = __ffma2_rn(make_float2(cw, cw), va[q], acc[q]);
                        }
                        continue;
                    }
                    if constexpr (kVec && kCplx && INTERP == kLinear && (S == kCF16 || S == kCBF16)) {
                        unsigned wa[NF], wb[NF];  // one (I, Q) word per frame
                        load_words<S, NF>(p, wa);
                        load_words<S, NF>(p + tp.step * fstride, wb);
#pragma unroll
                        for (int q = 0; q < NF; ++q) {
                            const float2 x = lerp_half_word<S>(wa[q], wb[q], tp.w0);
                            acc[q].x = __fmaf_rn(x.x, cw, __fmaf_rn(-x.y, sw, acc[q].x));
                            acc[q].y = __fmaf_rn(x.y, cw, __fmaf_rn(x.x, sw, acc[q].y));
                        }
                        continue;
                    }
                    if constexpr (kVec) {
                        float2 va[kAcc], vb[kAcc], vc[kAcc];
                        if constexpr (INTERP == kNearest) {
                            load_frames<S, NF>(p, va);
                        } else if constexpr (INTERP == kLinear) {
                            load_frames<S, NF>(p, va);
                            load_frames<S, NF>(p + tp.step * fstride, vb);
                        } else {
                            load_frames<S, NF>(p - fstride, va);
                            load_frames<S, NF>(p, vb);
                            load_frames<S, NF>(p + fstride, vc);
                        }
#pragma unroll
                        for (int q = 0; q < kAcc; ++q) {
                            float2 x;
                            if constexpr (INTERP == kNearest) {
                                x = va[q];
                            } else if constexpr (INTERP == kLinear) {
                                x.x = __fmaf_rn(tp.w0, __fsub_rn(vb[q].x, va[q].x), va[q].x);
                                x.y = __fmaf_rn(tp.w0, __fsub_rn(vb[q].y, va[q].y), va[q].y);
                            } else {
                                x.x = __fmaf_rn(tp.w2, vc[q].x, __fmaf_rn(tp.w0, va[q].x, __fmul_rn(tp.w1, vb[q].x)));
                                x.y = __fmaf_rn(tp.w2, vc[q].y, __fmaf_rn(tp.w0, va[q].y, __fmul_rn(tp.w1, vb[q].y)));
                            }
                            if constexpr (kCplx) {
                                acc[q].x = __fmaf_rn(x.x, cw, __fmaf_rn(-x.y, sw, acc[q].x));
                                acc[q].y = __fmaf_rn(x.y, cw, __fmaf_rn(x.x, sw, acc[q].y));
                            } else {
                                acc[q].x = __fmaf_rn(x.x, cw, acc[q].x);
                                acc[q].y = __fmaf_rn(x.y, cw, acc[q].y);
                            }
                        }
                        continue;
                    }
#pragma unroll
                    for (int f = 0; f < kAcc; ++f) {
                        if (NF > 0 || f < n_frames) {
                            const float2 x = tap_value<S, INTERP>(p + f, tp, n_frames);
                            if constexpr (kCplx) {
                                acc[f].x = __fmaf_rn(x.x, cw, __fmaf_rn(-x.y, sw, acc[f].x));
                                acc[f].y = __fmaf_rn(x.y, cw, __fmaf_rn(x.x, sw, acc[f].y));
                            } else {
                                acc[f].x = __fmaf_rn(x.x, cw, acc[f].x);
                            }
                        }
                    }
                }
            }
        }
    }

    if constexpr (kDeferRot) {
        acc[0].x = __fadd_rn(acc[0].x, __fsub_rn(acc_c.x, acc_s.y));
        acc[0].y = __fadd_rn(acc[0].y, __fadd_rn(acc_c.y, acc_s.x));
    }
    if constexpr (CS > 1) {  // add the lanes' partial sums of each voxel
#pragma unroll
        for (int off = 1; off < CS; off <<= 1) {
#pragma unroll
            for (int f = 0; f < kAcc; ++f) {
                acc[f].x = __fadd_rn(acc[f].x, __shfl_xor_sync(kFull, acc[f].x, off));
                acc[f].y = __fadd_rn(acc[f].y, __shfl_xor_sync(kFull, acc[f].y, off));
            }
        }
        if (sub != 0) return;
    }
    if (!vox_ok) return;
    if constexpr (kVec) {
#pragma unroll
        for (int q = 0; q < kAcc; ++q) {
            if constexpr (kCplx) {
                float2* out = static_cast<float2*>(a.out) + v * fstride + f0 + q;
                float2 r = acc[q];
                if (a.accumulate) {
                    const float2 prev = *out;
                    r.x = __fadd_rn(prev.x, r.x);
                    r.y = __fadd_rn(prev.y, r.y);
                }
                *out = r;
            } else {
                float* out = static_cast<float*>(a.out) + v * fstride + f0 + 2 * q;
                out[0] = a.accumulate ? __fadd_rn(out[0], acc[q].x) : acc[q].x;
                out[1] = a.accumulate ? __fadd_rn(out[1], acc[q].y) : acc[q].y;
            }
        }
        return;
    }
#pragma unroll
    for (int f = 0; f < kAcc; ++f) {
        if (NF > 0 || f < n_frames) {
            const int64_t o = v * n_frames + f;
            if constexpr (kCplx) {
                float2* out = static_cast<float2*>(a.out) + o;
                float2 r = acc[f];
                if (a.accumulate) {
                    const float2 prev = *out;
                    r.x = __fadd_rn(prev.x, r.x);
                    r.y = __fadd_rn(prev.y, r.y);
                }
                *out = r;
            } else {
                float* out = static_cast<float*>(a.out) + o;
                *out = a.accumulate ? __fadd_rn(*out, acc[f].x) : acc[f].x;
            }
        }
    }
}

// ---- per-point parameters shared by the warp-per-voxel kernel ----

// Receive path of one (voxel, element) pair in either delay mode.
struct PairRx {
    float dist;    // reference mode: FP32 distance (kernel.cu:467)
    SplitPos pos;  // split mode: receive part of the sample position
    float cyc;     // split mode: receive part of the phase (cycles)
    float w;       // apodisation weight x storage scale
};

// SM: delay mode known at compile time (0 reference, 1 split), or -1 to read a.split.
template <int SM = -1>
__device__ __forceinline__ bool pair_receive(const DasArgs& a, float ex, float ey, float ez, float vx, float vy,
                                             float vz, float radius, float radius_sq, PairRx& rx) {
    const float dx = __fsub_rn(ex, vx);
    const float dy = __fsub_rn(ey, vy);
    const float dz = __fsub_rn(ez, vz);
    const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    if (SM < 0 ? a.split != 0 : SM != 0) {
        const double ddx = static_cast<double>(ex) - vx, ddy = static_cast<double>(ey) - vy,
                     ddz = static_cast<double>(ez) - vz;
        const double d = sqrt(fma(ddx, ddx, fma(ddy, ddy, ddz * ddz)));
        rx.pos = split_position(d * a.fs_over_c);
        rx.cyc = reduced_cycles(d * a.fmod_over_c);
    } else {
        rx.dist = __fsqrt_rn(__fmaf_rn(dz, dz, h2));
    }
    float weight = 1.0f;
    if (a.apod) weight = fast_tukey(h2, radius, a);
    rx.w = __fmul_rn(weight, a.scale);
    return !(h2 > radius_sq) && !(weight == 0.0f);  // kernel.cu:461, 634
}

// Transmit part of one point: tap index, interpolation parameter (linear: t, quadratic: x
// from the centre tap) and the weighted phasor.  Returns false when the point is skipped.
template <int INTERP, bool CPLX, int SM = -1>
__device__ __forceinline__ bool point_taps(const DasArgs& a, const PairRx& rx, float txa, int& idx, float& w,
                                           float& cw, float& sw) {
    TapPosition tp{};
    float sn = 0.f, cs = 1.f;
    bool ok;
    if (SM < 0 ? a.split != 0 : SM != 0) {
        const SplitPos tx = split_position((static_cast<double>(txa) - a.t0_d) * a.fs_d);
        int base = tx.base + rx.pos.base;
        float frac = __fadd_rn(tx.frac, rx.pos.frac);
        if (frac >= 1.0f) {
            frac = __fsub_rn(frac, 1.0f);
            base += 1;
        }
        ok = !(base < a.start_base || (base == a.start_base && frac < a.start_frac));
        ok = ok && split_tap_position<INTERP>(base, frac, a.n_samples, tp);
        if (ok) w = INTERP == kQuadratic ? __fsub_rn(frac, static_cast<float>(tp.idx - base)) : tp.w0;
        if (ok && CPLX && a.rotate) split_phasor(__fadd_rn(reduced_cycles(static_cast<double>(txa) * a.fmod_d), rx.cyc), sn, cs);
    } else {
        const float tau = __fmaf_rn(rx.dist, a.inv_c, txa);
        const float s = __fmul_rn(__fsub_rn(tau, a.t0), a.fs);
        ok = !(tau < 0.0f);
        if constexpr (INTERP == kNearest) {
            ok = ok && (s >= -0.5f) && (s <= a.hi_nearest);
        } else if constexpr (INTERP == kLinear) {
            ok = ok && (s >= 0.0f) && (s <= a.hi_linear);
        } else {
            ok = ok && (s >= 1.0f) && (s <= a.hi_quadratic);
        }
        tp = tap_position<INTERP>(s);
        if constexpr (INTERP == kNearest) ok = ok && tp.idx < a.n_samples;
        if (ok) w = INTERP == kQuadratic ? __fsub_rn(s, static_cast<float>(tp.idx)) : tp.w0;
        if (ok && CPLX && a.rotate) __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
    }
    idx = tp.idx;
    cw = rx.w;
    sw = 0.f;
    if (ok && CPLX && a.rotate) {
        cw = __fmul_rn(cs, rx.w);
        sw = __fmul_rn(sn, rx.w);
    }
    return ok;
}

// Interpolated sample from tap index `idx` and parameter `w` (see point_taps); `row`
// already points at the frame, samples are `stride` apart.
template <int S, int INTERP>
__device__ __forceinline__ float2 gather_taps(const typename Storage<S>::T* row, int idx, float w, int64_t stride) {
    using ST = Storage<S>;
    const typename ST::T* p = row + static_cast<int64_t>(idx) * stride;
    if constexpr (INTERP == kNearest) {
        return ST::load(p);
    } else if constexpr (INTERP == kLinear) {
        const float2 lo = ST::load(p);
        const float2 hi = ST::load(p + (w > 0.0f ? stride : 0));
        return make_float2(__fmaf_rn(w, __fsub_rn(hi.x, lo.x), lo.x),
                           ST::kComplex ? __fmaf_rn(w, __fsub_rn(hi.y, lo.y), lo.y) : 0.f);
    } else {
        const float hx = __fmul_rn(0.5f, w);
        const float q = __fmul_rn(hx, w);
        const float wm = __fsub_rn(q, hx), w0 = __fmaf_rn(-2.0f, q, 1.0f), wp = __fadd_rn(q, hx);
        const float2 dm = ST::load(p - stride);
        const float2 d0 = ST::load(p);
        const float2 dp = ST::load(p + stride);
        return make_float2(__fmaf_rn(wp, dp.x, __fmaf_rn(wm, dm.x, __fmul_rn(w0, d0.x))),
                           ST::kComplex ? __fmaf_rn(wp, dp.y, __fmaf_rn(wm, dm.y, __fmul_rn(w0, d0.y))) : 0.f);
    }
}

template <int S, int INTERP, int NF, bool SPLIT, int CS = 1>
__global__ void __launch_bounds__(kLaneVoxelThreads, NF == 16 ? 4 : 8)
    das_lane_voxel_kernel(const __grid_constant__ DasArgs a) {
    extern __shared__ float smem_words[];
    if (NF >= 2 && a.frame_chunks > 1) {  // consecutive CTAs: the chunks of one tile, which share rows
        const int64_t tile = blockIdx.x / a.frame_chunks;
        lane_voxel_tile<S, INTERP, NF, SPLIT, CS>(a, tile, smem_words,
                                                  static_cast<int>(blockIdx.x - tile * a.frame_chunks));
    } else {
        lane_voxel_tile<S, INTERP, NF, SPLIT, CS>(a, blockIdx.x, smem_words);
    }
}

}  // namespace mach_b200
