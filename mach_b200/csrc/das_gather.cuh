// The delay-and-sum gather kernel (templated on storage, interpolation and lane shape).
//
// Work decomposition (one launch covers every transmit, element and frame):
//   * a warp owns G = 32 / LPV voxels; the LPV lanes of a voxel split its frames
//     (lane `sub` handles frames sub, sub + LPV, ... within the CTA's frame chunk);
//   * elements are visited in blocks of 32; a block is skipped unless some element
//     in it can be inside the f-number aperture of some voxel of the warp
//     (a conservative bounding-box test, then the exact per-pair test);
//   * within a block, chunks of LPV elements are processed: lane (voxel g, sub)
//     computes the receive path of pair (g, element chunk+sub) once -- distance,
//     Tukey weight, aperture test -- and reuses it for every transmit;
//   * for each transmit the lane turns that into a fractional sample index and a
//     weighted phasor, and the LPV lanes of the voxel group broadcast them with
//     warp shuffles so every lane gathers its own frames;
//   * transmits are processed in groups of TX_GROUP so the channel data in flight
//     across the GPU stays within L2; their arrival times live in registers;
//   * sums stay in registers across elements, transmits and frames and are written
//     once -- no atomics, no second pass.
#pragma once

#include "das_lane_voxel.cuh"

namespace mach_b200 {

constexpr int kThreadsPerBlock = 128;
constexpr int kTxGroup = 8;

template <int S, int INTERP, int LPV, int MAXP>
__global__ void __launch_bounds__(kThreadsPerBlock) das_gather_kernel(const __grid_constant__ DasArgs a) {
    using ST = Storage<S>;
    using T = typename ST::T;
    constexpr bool kCplx = ST::kComplex;
    constexpr int G = 32 / LPV;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr unsigned kLaneMask = LPV == 32 ? kFull : ((1u << (LPV & 31)) - 1u);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = lane / LPV;
    const int sub = lane - g * LPV;
    const int64_t v = (static_cast<int64_t>(blockIdx.x) * (kThreadsPerBlock / 32) + warp) * G + g;
    const bool vox_ok = v < a.n_vox;
    const int passes = a.frame_passes;
    const int frame0 = static_cast<int>(blockIdx.y) * (LPV * passes) + sub;

    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (vox_ok) {
        vx = __ldg(a.scan + 3 * v + 0);
        vy = __ldg(a.scan + 3 * v + 1);
        vz = __ldg(a.scan + 3 * v + 2);
    }
    // kernel.cu:583-584
    const float radius = __fdiv_rn(vz, a.two_f_number);
    const float radius_sq = __fmul_rn(radius, radius);

    // Bounding box of the warp's voxels in the array plane, and the largest aperture radius.
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
    // Superset margin: FP32 rounding of h2 and R^2 is far below 1e-5 relative.
    const float cand_r2 = rmax * rmax * 1.00001f + 1e-30f;

    float2 acc[MAXP];
#pragma unroll
    for (int p = 0; p < MAXP; ++p) acc[p] = make_float2(0.f, 0.f);

    const T* const channel = static_cast<const T*>(a.channel);
    const int64_t n_frames = a.n_frames;

    for (int tg = 0; tg < a.n_tx; tg += kTxGroup) {
        float txa[kTxGroup];
#pragma unroll
        for (int j = 0; j < kTxGroup; ++j) {
            txa[j] = (vox_ok && tg + j < a.n_tx) ? __ldg(a.arrivals + static_cast<int64_t>(tg + j) * a.n_vox + v) : 0.f;
        }

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
            const unsigned cmask = __ballot_sync(kFull, cand);
            if (cmask == 0u) continue;

#pragma unroll 1
            for (int c0 = 0; c0 < 32; c0 += LPV) {
                const unsigned chunk_mask = (cmask >> c0) & kLaneMask;
                if (chunk_mask == 0u) continue;

                // Receive path of this lane's pair (voxel g, element eb + c0 + sub).
                const int pe = eb + c0 + sub;
                bool pair_ok = vox_ok && pe < a.n_rx && ((chunk_mask >> sub) & 1u);
                PairRx rx{};
                if (pair_ok) {
                    pair_ok = pair_receive(a, __ldg(a.rx + 3 * pe + 0), __ldg(a.rx + 3 * pe + 1),
                                           __ldg(a.rx + 3 * pe + 2), vx, vy, vz, radius, radius_sq, rx);
                }
                const bool any_pair = __any_sync(kFull, pair_ok);
                if (!any_pair) continue;

#pragma unroll
                for (int j = 0; j < kTxGroup; ++j) {
                    const int tx = tg + j;
                    if (tx >= a.n_tx) continue;
                    int idx = 0;
                    float w = 0.f, cw = 0.f, sw = 0.f;
                    const bool ok = pair_ok && point_taps<INTERP, kCplx>(a, rx, txa[j], idx, w, cw, sw);
                    const T* const tx_base = channel + static_cast<int64_t>(tx) * a.n_rx * a.row_stride;

                    if constexpr (LPV == 1) {
                        if (ok) {
                            const T* row = tx_base + static_cast<int64_t>(pe) * a.row_stride;
#pragma unroll
                            for (int p = 0; p < MAXP; ++p) {
                                if (p < passes && frame0 + p < n_frames) {
                                    const float2 x = gather_taps<S, INTERP>(row + frame0 + p, idx, w, n_frames);
                                    if constexpr (kCplx) {
                                        acc[p].x = __fmaf_rn(x.x, cw, __fmaf_rn(-x.y, sw, acc[p].x));
                                        acc[p].y = __fmaf_rn(x.y, cw, __fmaf_rn(x.x, sw, acc[p].y));
                                    } else {
                                        acc[p].x = __fmaf_rn(x.x, cw, acc[p].x);
                                    }
                                }
                            }
                        }
                    } else {
                        // Which chunk positions k are valid for at least one voxel group of the warp.
                        unsigned vmask = __ballot_sync(kFull, ok);
                        unsigned kmask = 0u;
#pragma unroll
                        for (int gg = 0; gg < G; ++gg) kmask |= (vmask >> ((gg * LPV) & 31)) & kLaneMask;
                        while (kmask) {
                            const int k = __ffs(kmask) - 1;
                            kmask &= kmask - 1u;
                            const int idxk = __shfl_sync(kFull, idx, k, LPV);
                            const float wk = __shfl_sync(kFull, w, k, LPV);
                            const float cwk = __shfl_sync(kFull, cw, k, LPV);
                            const float swk = kCplx ? __shfl_sync(kFull, sw, k, LPV) : 0.f;
                            const bool okk = (vmask >> (g * LPV + k)) & 1u;
                            if (okk) {
                                const T* row = tx_base + static_cast<int64_t>(eb + c0 + k) * a.row_stride;
#pragma unroll
                                for (int p = 0; p < MAXP; ++p) {
                                    const int f = frame0 + p * LPV;
                                    if (p < passes && f < n_frames) {
                                        const float2 x = gather_taps<S, INTERP>(row + f, idxk, wk, n_frames);
                                        if constexpr (kCplx) {
                                            acc[p].x = __fmaf_rn(x.x, cwk, __fmaf_rn(-x.y, swk, acc[p].x));
                                            acc[p].y = __fmaf_rn(x.y, cwk, __fmaf_rn(x.x, swk, acc[p].y));
                                        } else {
                                            acc[p].x = __fmaf_rn(x.x, cwk, acc[p].x);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }

    if (!vox_ok) return;
#pragma unroll
    for (int p = 0; p < MAXP; ++p) {
        const int f = LPV == 1 ? frame0 + p : frame0 + p * LPV;
        if (p < passes && f < n_frames) {
            const int64_t o = v * n_frames + f;
            if constexpr (kCplx) {
                float2* out = static_cast<float2*>(a.out) + o;
                float2 r = acc[p];
                if (a.accumulate) {
                    const float2 prev = *out;
                    r.x = __fadd_rn(prev.x, r.x);
                    r.y = __fadd_rn(prev.y, r.y);
                }
                *out = r;
            } else {
                float* out = static_cast<float*>(a.out) + o;
                *out = a.accumulate ? __fadd_rn(*out, acc[p].x) : acc[p].x;
            }
        }
    }
}

}  // namespace mach_b200
