// Frame-lane gather kernel for long ensembles (Doppler, many-frame 3-D): lanes hold frames,
// and a warp walks a run of G neighbouring voxels, loading each element's sample rows once for
// all of them.
//
// The work of an ensemble is, per (voxel, element, transmit) point, two sample rows of all
// frames (linear taps s and s + 1) weighted by one complex coefficient each.  Delays and
// weights do not depend on the frame, and neighbouring voxels along the lateral axes read
// nearly the same rows (a 0.125 mm lateral step moves a delay by less than one sample inside
// an f# >= 1 aperture).  So:
//   * a warp owns G voxels of one run along a lateral grid axis and a chunk of 32 J lane
//     words of frames (complex storage: one frame per lane word; real storage: two);
//   * per (transmit, element batch) the 32 lanes compute the parameters of 32 (voxel,
//     element) pairs -- mach's FP32 delay, aperture and Tukey arithmetic, or the split FP64
//     base + FP32 fraction -- into shared memory: tap row, whether the second tap is used,
//     and the interpolation weights folded into the weighted phasor.  The next batch's
//     parameters are computed before this batch's points are summed;
//   * per element, the warp takes the rows its in-aperture voxels need, [rmin, rmax], and
//     when they span at most kFrameLaneRows rows loads all of them at once (every load of
//     the element in flight together, one memory latency per element rather than per point),
//     then adds each voxel's taps from the row registers by a static index.  On the Doppler
//     configuration the union is 0.78 rows per point instead of 2 (measured on its
//     geometry).  Wider spans load each voxel's rows in turn.  Every decision is
//     warp-uniform because every lane works on the same voxel;
//   * the accumulation is packed FP32x2 (FFMA2): complex storage keeps two accumulator pairs
//     per frame, sum(cw (I, Q)) and sum(sw (I, Q)), combined into the rotated sum at the end;
//     real storage keeps one pair per two frames;
//   * sums stay in registers for the whole job and are written once, coalesced; the
//     power-Doppler epilogue adds sum over frames of |x|^2 with one atomic per voxel and
//     chunk instead.
// There are no waits on other warps and no barriers beyond __syncwarp.
#pragma once

#include "das_ensemble.cuh"  // LaneWord<S>

namespace mach_b200 {

constexpr int kFrameLaneWarps = 4;
constexpr int kFrameLaneThreads = 32 * kFrameLaneWarps;
constexpr int kFrameLaneRows = 4;  // rows of one element held at once

// Run mapping and frame chunking of one frame-lane launch.
struct FrameLaneArgs {
    int64_t run_len;       // voxels along the run axis (n_vox without a grid)
    int64_t run_stride;    // voxel-index stride along the run axis (1 without a grid)
    int64_t n_across;      // lines along the other lateral axis (1 for a 2-D grid)
    int64_t across_stride; // voxel-index stride of that axis
    int64_t n_fast;        // voxels along the contiguous axis (1 without a grid)
    int64_t runs_per_line; // ceil(run_len / G)
    int64_t n_runs;        // runs_per_line * n_across * n_fast
    int32_t words;         // lane words per sample row: n_frames (complex) or n_frames / 2 (real)
    int32_t n_chunks;      // ceil(words / (32 J))
};

// Shared memory of one warp: the parameters of two batches (tap rows, then coefficients).
template <int KCOEF>
__host__ __device__ constexpr int frame_lane_warp_bytes() {
    return 2 * 32 * 4 + 2 * 32 * 16 * KCOEF;
}

// Voxel i of run `run`, or -1 when the run is shorter than G there.
__device__ __forceinline__ int64_t frame_lane_voxel(const FrameLaneArgs& fl, int64_t run, int G, int i) {
    const int64_t ry = run % fl.runs_per_line;
    const int64_t rest = run / fl.runs_per_line;
    const int64_t xa = rest % fl.n_across;
    const int64_t z = rest / fl.n_across;
    const int64_t y = ry * G + i;
    if (y >= fl.run_len || z >= fl.n_fast) return -1;
    return xa * fl.across_stride + y * fl.run_stride + z;
}

constexpr int kActTwo = 1;   // the second tap (row + 1) is used
constexpr int kActShift = 1; // the tap row, shifted

// One CTA block of a frame-lane launch: four warps, runs 4 block / n_chunks .. + 3, frame chunk
// block % n_chunks.  Shared by the per-job kernel and the persistent batch kernel; returns
// (per warp) when done.  SPLIT is the delay mode (the FP64 split path costs registers, so it is
// compiled only where it is used).  FULL: the chunk holds 32 J lane words of every row (no
// partial column), so no lane checks.
template <int S, int INTERP, int J, int G, bool SPLIT, bool FULL>
__device__ __forceinline__ void frame_lane_block_impl(const DasArgs& a, const FrameLaneArgs& fl, int64_t block,
                                                      unsigned char* smem_raw) {
    static_assert(32 % G == 0 && G <= 32, "G divides the warp");
    static_assert(INTERP == kNearest || INTERP == kLinear, "two-tap interpolators only");
    using LW = LaneWord<S>;
    using W = typename LW::W;
    constexpr bool kCplx = Storage<S>::kComplex;
    constexpr int kEB = 32 / G;                    // elements per parameter batch
    constexpr unsigned kGMask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
    constexpr int kCoef = kCplx ? 2 : 1;           // float4 coefficient words per pair
    constexpr int kSM = SPLIT ? 1 : 0;
    constexpr int U = kFrameLaneRows;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int* const s_act = reinterpret_cast<int*>(smem_raw + warp * frame_lane_warp_bytes<kCoef>());  // [2][32]
    float4* const s_coef = reinterpret_cast<float4*>(s_act + 2 * 32);                             // [2][32][kCoef]

    const int64_t run = (block / fl.n_chunks) * kFrameLaneWarps + warp;
    const int chunk = static_cast<int>(block % fl.n_chunks);
    if (run >= fl.n_runs) return;  // whole warp: no CTA-wide barrier below
    const int w0 = chunk * 32 * J;                                // first lane word of this chunk
    const int nj = FULL ? J : min(J, (fl.words - w0 + 31) >> 5);  // columns holding frames
    const W* const channel = static_cast<const W*>(a.channel);

    // This lane's parameter role: voxel i = lane % G of the run, element eb + lane / G.
    const int pi = lane % G;
    const int pe = lane / G;
    const int64_t pv = frame_lane_voxel(fl, run, G, pi);
    const bool pv_ok = pv >= 0;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (pv_ok) {
        vx = __ldg(a.scan + 3 * pv + 0);
        vy = __ldg(a.scan + 3 * pv + 1);
        vz = __ldg(a.scan + 3 * pv + 2);
    }
    const float radius = __fdiv_rn(vz, a.two_f_number);  // kernel.cu:583
    const float radius_sq = __fmul_rn(radius, radius);

    // Accumulators: complex -> (sum cw*(I,Q), sum sw*(I,Q)) per frame; real -> one pair per
    // two frames.
    float2 acc0[G][J], acc1[G][kCplx ? J : 1];
#pragma unroll
    for (int i = 0; i < G; ++i) {
#pragma unroll
        for (int j = 0; j < J; ++j) {
            acc0[i][j] = make_float2(0.f, 0.f);
            if constexpr (kCplx) acc1[i][j] = make_float2(0.f, 0.f);
        }
    }

    auto load_row = [&](float2 (&Rr)[J], int row) {
        const W* p = channel + static_cast<int64_t>(row) * fl.words + w0 + lane;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            if (FULL || (j < nj && w0 + 32 * j + lane < fl.words)) Rr[j] = LW::widen(__ldg(p + 32 * j));
        }
    };
    // acc[i] += cA * RA + cB * RB (two taps), or cA * RA (one tap).
    auto mac2 = [&](float2 (&A0)[J], float2 (&A1)[kCplx ? J : 1], const float2 (&RA)[J], const float2 (&RB)[J],
                    const float4& ca, const float4& cb) {
#pragma unroll
        for (int j = 0; j < J; ++j) {
            if (FULL || j < nj) {
                if constexpr (kCplx) {
                    A0[j] = __ffma2_rn(make_float2(ca.x, ca.y), RA[j], A0[j]);
                    A1[j] = __ffma2_rn(make_float2(ca.z, ca.w), RA[j], A1[j]);
                    A0[j] = __ffma2_rn(make_float2(cb.x, cb.y), RB[j], A0[j]);
                    A1[j] = __ffma2_rn(make_float2(cb.z, cb.w), RB[j], A1[j]);
                } else {
                    A0[j] = __ffma2_rn(make_float2(ca.x, ca.y), RA[j], A0[j]);
                    A0[j] = __ffma2_rn(make_float2(ca.z, ca.w), RB[j], A0[j]);
                }
            }
        }
    };
    auto mac1 = [&](float2 (&A0)[J], float2 (&A1)[kCplx ? J : 1], const float2 (&RA)[J], const float4& ca) {
#pragma unroll
        for (int j = 0; j < J; ++j) {
            if (FULL || j < nj) {
                A0[j] = __ffma2_rn(make_float2(ca.x, ca.y), RA[j], A0[j]);
                if constexpr (kCplx) A1[j] = __ffma2_rn(make_float2(ca.z, ca.w), RA[j], A1[j]);
            }
        }
    };
    // Taps of one point from rows R[o], R[o + 1] (o static), parameters of slot p.
    auto point = [&](float2 (&A0)[J], float2 (&A1)[kCplx ? J : 1], const float2 (&R)[U][J], int buf, int p,
                     int o) {
        const int act = s_act[buf * 32 + p];
        const float4 ca = s_coef[(buf * 32 + p) * kCoef];
        const float4 cb = kCplx ? s_coef[(buf * 32 + p) * kCoef + kCoef - 1] : ca;
        if (INTERP == kLinear && (act & kActTwo)) {
            // complex: ca = (a cw, a cw, a sw, a sw), cb = (b cw, ...); real: ca = (a w, a w, b w, b w)
            switch (o) {
                case 0: mac2(A0, A1, R[0], R[1], ca, kCplx ? cb : ca); break;
                case 1: mac2(A0, A1, R[1], R[2], ca, kCplx ? cb : ca); break;
                default: mac2(A0, A1, R[2], R[3], ca, kCplx ? cb : ca); break;
            }
        } else {
            switch (o) {
                case 0: mac1(A0, A1, R[0], ca); break;
                case 1: mac1(A0, A1, R[1], ca); break;
                case 2: mac1(A0, A1, R[2], ca); break;
                default: mac1(A0, A1, R[3], ca); break;
            }
        }
    };
    // The points of element eo of batch buffer `buf` (voxel bits m): its rows once, then each
    // voxel's taps.
    auto element = [&](int buf, int eo, unsigned m) {
        float2 R[U][J];  // rows rmin .. rmin + U - 1 (only the element's own rows are read)
        if constexpr (!FULL) {  // lanes past the row's end read nothing: keep them finite
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int j = 0; j < J; ++j) R[u][j] = make_float2(0.f, 0.f);
            }
        }
        int rmin = 0x7fffffff, rmax = -1;
#pragma unroll
        for (int i = 0; i < G; ++i) {
            if ((m >> i) & 1u) {
                const int act = s_act[buf * 32 + eo * G + i];
                rmin = min(rmin, act >> kActShift);
                rmax = max(rmax, (act >> kActShift) + (act & kActTwo));
            }
        }
        const int span = rmax - rmin + 1;
        if (span <= U) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (u < span) load_row(R[u], rmin + u);
            }
#pragma unroll
            for (int i = 0; i < G; ++i) {
                if ((m >> i) & 1u) {
                    const int p = eo * G + i;
                    point(acc0[i], acc1[i], R, buf, p, (s_act[buf * 32 + p] >> kActShift) - rmin);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < G; ++i) {
                if ((m >> i) & 1u) {
                    const int p = eo * G + i;
                    const int act = s_act[buf * 32 + p];
                    load_row(R[0], act >> kActShift);
                    if (INTERP == kLinear && (act & kActTwo)) load_row(R[1], (act >> kActShift) + 1);
                    point(acc0[i], acc1[i], R, buf, p, 0);
                }
            }
        }
    };

    // ---- one parameter batch: (transmit, 32 / G elements) x the G voxels of the run
    const int n_eb = (a.n_rx + kEB - 1) / kEB;
    const int n_batches = a.n_tx * n_eb;
    auto params = [&](int bi, int buf) -> unsigned {
        const int t = bi / n_eb;
        const int e = (bi - t * n_eb) * kEB + pe;
        bool ok = false;
        int act = 0;
        float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0;
        if (pv_ok && e < a.n_rx) {
            const float ex = __ldg(a.rx + 3 * e + 0), ey = __ldg(a.rx + 3 * e + 1), ez = __ldg(a.rx + 3 * e + 2);
            PairRx rx;
            if (pair_receive<kSM>(a, ex, ey, ez, vx, vy, vz, radius, radius_sq, rx)) {
                const float txa = __ldg(a.arrivals + static_cast<int64_t>(t) * a.n_vox + pv);
                int idx;
                float frac = 0.f, cw, sw;
                ok = point_taps<INTERP, kCplx, kSM>(a, rx, txa, idx, frac, cw, sw);
                if (ok) {
                    const int row = (t * a.n_rx + e) * a.n_samples + idx;
                    const bool two = INTERP == kLinear && frac > 0.0f;
                    act = (row << kActShift) | (two ? kActTwo : 0);
                    const float fa = two ? __fsub_rn(1.0f, frac) : 1.0f;
                    const float fb = two ? frac : 0.0f;
                    if constexpr (kCplx) {
                        const float acw = __fmul_rn(fa, cw), asw = __fmul_rn(fa, sw);
                        const float bcw = __fmul_rn(fb, cw), bsw = __fmul_rn(fb, sw);
                        c0 = make_float4(acw, acw, asw, asw);
                        c1 = make_float4(bcw, bcw, bsw, bsw);
                    } else {
                        const float aw = __fmul_rn(fa, cw), bw = __fmul_rn(fb, cw);
                        c0 = make_float4(aw, aw, bw, bw);
                    }
                }
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        s_act[buf * 32 + lane] = act;
        s_coef[(buf * 32 + lane) * kCoef] = c0;
        if constexpr (kCplx) s_coef[(buf * 32 + lane) * kCoef + 1] = c1;
        __syncwarp();
        return mask;
    };

    int buf = 0;
    unsigned mask = n_batches > 0 ? params(0, 0) : 0u;
    for (int bi = 0; bi < n_batches; ++bi) {
        // the next batch's parameters, ahead of this batch's points
        const unsigned next = bi + 1 < n_batches ? params(bi + 1, buf ^ 1) : 0u;
        while (mask != 0u) {
            const int eo = (__ffs(mask) - 1) / G;
            const unsigned m = (mask >> (eo * G)) & kGMask;
            mask &= ~(kGMask << (eo * G));
            element(buf, eo, m);
        }
        __syncwarp();  // this buffer's parameters are rewritten two batches on
        buf ^= 1;
        mask = next;
    }

    // Write the sums (or the power-Doppler epilogue).
#pragma unroll
    for (int i = 0; i < G; ++i) {
        const int64_t v = frame_lane_voxel(fl, run, G, i);
        if (v < 0) continue;  // uniform: v does not depend on the lane
        float power = 0.f;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int w = w0 + 32 * j + lane;
            if (j >= nj || w >= fl.words) continue;
            float2 r;
            if constexpr (kCplx) {
                r.x = __fsub_rn(acc0[i][j].x, acc1[i][j].y);  // sum cw I - sw Q
                r.y = __fadd_rn(acc0[i][j].y, acc1[i][j].x);  // sum cw Q + sw I
            } else {
                r = acc0[i][j];
            }
            if (a.power) {
                power = __fmaf_rn(r.x, r.x, power);
                power = __fmaf_rn(r.y, r.y, power);
                continue;
            }
            float2* o = reinterpret_cast<float2*>(static_cast<char*>(a.out) +
                                                  (v * a.n_frames + static_cast<int64_t>(w) * LW::kFrames) * 4 *
                                                      (kCplx ? 2 : 1));
            if (a.accumulate) {
                const float2 prev = *o;
                r.x = __fadd_rn(prev.x, r.x);
                r.y = __fadd_rn(prev.y, r.y);
            }
            *o = r;
        }
        if (a.power) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) power += __shfl_xor_sync(0xffffffffu, power, off);
            if (lane == 0) atomicAdd(static_cast<float*>(a.out) + v, power);
        }
    }
}

template <int S, int INTERP, int J, int G, bool SPLIT>
__device__ __forceinline__ void frame_lane_block(const DasArgs& a, const FrameLaneArgs& fl, int64_t block,
                                                 unsigned char* smem_raw) {
    const int w0 = static_cast<int>(block % fl.n_chunks) * 32 * J;
    if (fl.words - w0 >= 32 * J) {
        frame_lane_block_impl<S, INTERP, J, G, SPLIT, true>(a, fl, block, smem_raw);
    } else {
        frame_lane_block_impl<S, INTERP, J, G, SPLIT, false>(a, fl, block, smem_raw);
    }
}

template <int S, int INTERP, int J, int G, bool SPLIT>
__global__ void __launch_bounds__(kFrameLaneThreads, 4)
    das_frame_lane_kernel(const __grid_constant__ DasArgs a, const __grid_constant__ FrameLaneArgs fl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    frame_lane_block<S, INTERP, J, G, SPLIT>(a, fl, blockIdx.x, smem_raw);
}

}  // namespace mach_b200
