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

// Interpolated sample at `row[idx * stride]` (stride = frames), widened to FP32.
template <int S, int INTERP>
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
        float2 r;
        r.x = __fmaf_rn(tp.w2, c.x, __fmaf_rn(tp.w0, a.x, __fmul_rn(tp.w1, b.x)));
        r.y = ST::kComplex ? __fmaf_rn(tp.w2, c.y, __fmaf_rn(tp.w0, a.y, __fmul_rn(tp.w1, b.y))) : 0.f;
        return r;
    }
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

template <int S, int INTERP, int NF>
__global__ void __launch_bounds__(kLaneVoxelThreads, 8) das_lane_voxel_kernel(const __grid_constant__ DasArgs a) {
    using ST = Storage<S>;
    using T = typename ST::T;
    constexpr bool kCplx = ST::kComplex;
    constexpr unsigned kFull = 0xffffffffu;
    extern __shared__ float s_arrival[];  // [tx_chunk][kLaneVoxelThreads]

    const int lane = threadIdx.x & 31;
    const int64_t v = static_cast<int64_t>(blockIdx.x) * kLaneVoxelThreads + threadIdx.x;
    const bool vox_ok = v < a.n_vox;
    const int n_frames = NF > 0 ? NF : a.n_frames;

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

    constexpr int kAcc = NF > 0 ? NF : 8;
    float2 acc[kAcc];
#pragma unroll
    for (int f = 0; f < kAcc; ++f) acc[f] = make_float2(0.f, 0.f);

    const T* const channel = static_cast<const T*>(a.channel);
    const int row_len = a.n_samples * n_frames;  // samples per (transmit, element) row
    const int tx_chunk = a.tx_chunk;

    for (int t0 = 0; t0 < a.n_tx; t0 += tx_chunk) {
        const int nt = min(tx_chunk, a.n_tx - t0);
        __syncthreads();
        for (int i = threadIdx.x; i < nt * kLaneVoxelThreads; i += kLaneVoxelThreads) {
            const int t = i / kLaneVoxelThreads;
            const int64_t vv = static_cast<int64_t>(blockIdx.x) * kLaneVoxelThreads + (i - t * kLaneVoxelThreads);
            s_arrival[i] = vv < a.n_vox ? __ldg(a.arrivals + static_cast<int64_t>(t0 + t) * a.n_vox + vv) : 0.f;
        }
        __syncthreads();

        for (int eb = 0; eb < a.n_rx; eb += 32) {
            bool cand = false;
            {
                const int e = eb + lane;
                if (e < a.n_rx) {
                    const float ex = __ldg(a.rx + 3 * e + 0);
                    const float ey = __ldg(a.rx + 3 * e + 1);
                    const float ddx = fmaxf(fmaxf(bx0 - ex, ex - bx1), 0.f);
                    const float ddy = fmaxf(fmaxf(by0 - ey, ey - by1), 0.f);
                    cand = ddx * ddx + ddy * ddy <= cand_r2;
                }
            }
            unsigned cmask = __ballot_sync(kFull, cand);
            while (cmask) {
                const int e = eb + __ffs(cmask) - 1;
                cmask &= cmask - 1u;

                // Receive path (kernel.cu:444-483), reused for every transmit below.
                const float dx = __fsub_rn(__ldg(a.rx + 3 * e + 0), vx);
                const float dy = __fsub_rn(__ldg(a.rx + 3 * e + 1), vy);
                const float dz = __fsub_rn(__ldg(a.rx + 3 * e + 2), vz);
                const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                const float dist = __fsqrt_rn(__fmaf_rn(dz, dz, h2));
                float weight = 1.0f;
                if (a.apod) weight = fast_tukey(h2, radius, a);
                const bool pair_ok = vox_ok && !(h2 > radius_sq) && !(weight == 0.0f);
                if (!__any_sync(kFull, pair_ok)) continue;
                const float w = __fmul_rn(weight, a.scale);

                int row = (t0 * a.n_rx + e) * row_len;
                const int tx_step = a.n_rx * row_len;
#pragma unroll 2
                for (int t = 0; t < nt; ++t, row += tx_step) {
                    const float tau = __fmaf_rn(dist, a.inv_c, s_arrival[t * kLaneVoxelThreads + threadIdx.x]);
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
                    const TapPosition tp = tap_position<INTERP>(s);
                    if constexpr (INTERP == kNearest) {
                        if (tp.idx >= a.n_samples) continue;
                    }
                    float cw = w, sw = 0.f;
                    if (kCplx && a.rotate) {
                        float sn, cs;
                        __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
                        cw = __fmul_rn(cs, w);
                        sw = __fmul_rn(sn, w);
                    }
                    const T* p = channel + (row + tp.idx * n_frames);
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

    if (!vox_ok) return;
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

}  // namespace mach_b200
