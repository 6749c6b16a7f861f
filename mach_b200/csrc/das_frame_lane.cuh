// Frame-lane gather kernel for long ensembles (Doppler, many-frame 3-D): lanes hold frames,
// and a warp walks a run of G neighbouring voxels while keeping sample rows in registers.
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
//     and the interpolation weights folded into the weighted phasor;
//   * the warp steps through the in-aperture pairs element by element, voxel by voxel.  It
//     holds two sample rows of its frame chunk in registers (slots R0, R1: one lane word per
//     lane and column) and loads a row only when the step needs one that neither slot holds.
//     On the Doppler configuration that is 0.78 row loads per point instead of 2 (measured on
//     its geometry); every decision is warp-uniform because every lane works on the same voxel;
//   * ring mode (rows of a multiple of 16 bytes, 16-byte aligned channel data): the rows a
//     batch will load are known once its parameters are: a planning pass runs the two-slot
//     window over the batch and lists them, and lane 0 streams them one batch ahead into a
//     ring of K shared-memory row buffers with bulk copies (cp.async.bulk, mbarrier
//     completion, no multicast).  A step that needs a row waits on its buffer's mbarrier
//     (bounded wait) and reads it with conflict-free shared-memory loads, so L2 latency is
//     hidden behind the steps before it.  Direct mode loads the rows from global memory;
//   * the accumulation is packed FP32x2 (FFMA2): complex storage keeps two accumulator pairs
//     per frame, sum(cw (I, Q)) and sum(sw (I, Q)), combined into the rotated sum at the end;
//     real storage keeps one pair per two frames;
//   * sums stay in registers for the whole job and are written once, coalesced; the
//     power-Doppler epilogue adds sum over frames of |x|^2 with one atomic per voxel and
//     chunk instead.
// Every mbarrier wait is bounded; on a timeout the warp stops, waits (bounded) for its copies
// in flight and sets the status word, and its voxels' output is not written.
#pragma once

#include "das_ensemble.cuh"  // LaneWord<S>, mbarrier helpers

namespace mach_b200 {

constexpr int kFrameLaneWarps = 4;
constexpr int kFrameLaneThreads = 32 * kFrameLaneWarps;
constexpr int kFrameLaneList = 128;  // row-list entries per warp (two batches of at most 64 loads)

// Run mapping, frame chunking and ring layout of one frame-lane launch.
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
    int32_t ring_slots;    // K: row buffers per warp (a power of two), ring mode
    int32_t ring_log2;     // log2(K)
    int32_t slot_bytes;    // bytes of one row buffer: 32 J lane words
    int32_t warp_bytes;    // dynamic shared memory per warp (128-byte multiple)
    int32_t* status;       // device status word: set when a bounded wait gives up
};

// Dynamic shared memory of one warp: ring buffers, then mbarriers, the row list, and the
// parameters of two batches.
template <int KCOEF>
__host__ __device__ constexpr int frame_lane_warp_bytes(int slots, int slot_bytes) {
    return ((slots * slot_bytes + slots * 8 + kFrameLaneList * 4 + 2 * 32 * 4 + 2 * 32 * 16 * KCOEF) + 127) & ~127;
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

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Action bits of a planned step (ring mode), stored with the tap row (row << kActShift).
constexpr int kActTwo = 1;   // second tap (row + 1) used
constexpr int kActL0 = 2;    // slot R0 is loaded from the next ring entry
constexpr int kActL1 = 4;    // slot R1 is loaded from the next ring entry (after R0's)
constexpr int kActRin0 = 8;  // slot R0 holds the first tap's row
constexpr int kActShift = 4;

// One CTA block of a frame-lane launch: four warps, runs 4 block / n_chunks .. + 3, frame chunk
// block % n_chunks.  Shared by the per-job kernel and the persistent batch kernel; returns
// (per warp) when done.  SPLIT is the delay mode (the FP64 split path costs registers, so it is
// compiled only where it is used).
// Bounded wait on a ring buffer's mbarrier: try_wait polls without a suspend hint (a buffer is
// usually full, or nearly, when a step needs it); gives up after 2^31 SM clock cycles (about
// a second at B200 clocks).
__device__ __forceinline__ bool ring_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

// FULL: the chunk holds 32 J lane words of every row (no partial column), so no lane checks.
template <int S, int INTERP, int J, int G, bool SPLIT, bool RING, bool FULL>
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

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned char* const wsm = smem_raw + warp * fl.warp_bytes;
    const int K = RING ? fl.ring_slots : 0;
    unsigned char* const ring = wsm;
    uint64_t* const bars = reinterpret_cast<uint64_t*>(wsm + K * fl.slot_bytes);
    int* const list = reinterpret_cast<int*>(bars + K);
    int* const s_act = list + kFrameLaneList;                              // [2][32]
    float4* const s_coef = reinterpret_cast<float4*>(s_act + 2 * 32);      // [2][32][kCoef]

    const int64_t run = (block / fl.n_chunks) * kFrameLaneWarps + warp;
    const int chunk = static_cast<int>(block % fl.n_chunks);
    if (run >= fl.n_runs) return;  // whole warp: no CTA-wide barrier below
    const int w0 = chunk * 32 * J;                                // first lane word of this chunk
    const int nj = FULL ? J : min(J, (fl.words - w0 + 31) >> 5);  // columns holding frames
    const uint32_t copy_bytes = static_cast<uint32_t>(min(32 * J, fl.words - w0)) * sizeof(W);
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

    if constexpr (RING) {
        if (lane == 0) {
            for (int k = 0; k < K; ++k) mbar_init(bars + k, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
    }

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
    float2 R0[J], R1[J];
#pragma unroll
    for (int j = 0; j < J; ++j) R0[j] = R1[j] = make_float2(0.f, 0.f);

    // ---- rows: direct loads, or the ring (head: entries consumed, tail: copies issued,
    // planned: entries listed)
    int q0 = -1, q1 = -1, lru = 0;  // window state (direct mode: consumer; ring mode: planner)
    int head = 0, tail = 0, planned = 0;
    bool failed = false;

    auto load_row = [&](float2 (&R)[J], int row) {
        const W* p = channel + static_cast<int64_t>(row) * fl.words + w0 + lane;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            if (FULL || (j < nj && w0 + 32 * j + lane < fl.words)) R[j] = LW::widen(__ldg(p + 32 * j));
        }
    };
    // Lane 0 streams listed rows into free ring buffers.
    auto issue = [&]() {
        if (tail < planned && tail - head < K) {
            __syncwarp();  // every lane has read the buffers that are reused below
            while (tail < planned && tail - head < K) {
                const int slot = tail & (K - 1);
                if (lane == 0) {
                    const int row = list[tail & (kFrameLaneList - 1)];
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_expect_tx(bars + slot, copy_bytes);
                    bulk_load(ring + slot * fl.slot_bytes, channel + static_cast<int64_t>(row) * fl.words + w0,
                              copy_bytes, bars + slot);
                }
                ++tail;
            }
        }
    };
    auto consume = [&](float2 (&R)[J]) {
        if (tail <= head) issue();  // (never needed by the refill rule; keeps every wait on an issued copy)
        const int slot = head & (K - 1);
        const bool ok = ring_wait(bars + slot, static_cast<uint32_t>(head >> fl.ring_log2) & 1u);
        if (__any_sync(0xffffffffu, !ok)) failed = true;
        const W* p = reinterpret_cast<const W*>(ring + slot * fl.slot_bytes) + lane;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            if (FULL || (j < nj && w0 + 32 * j + lane < fl.words)) R[j] = LW::widen(p[32 * j]);
        }
        ++head;
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
    // Ring mode: run the two-slot window over the batch's steps (in consumption order), list
    // the rows to load and record each step's actions.
    auto plan = [&](int buf, unsigned mask) {
        while (mask != 0u) {
            const int p = __ffs(mask) - 1;
            mask &= mask - 1u;
            int act = s_act[buf * 32 + p];
            const int r = act >> kActShift;
            const bool two = (act & kActTwo) != 0;
            const bool have_r = q0 == r || q1 == r;
            const bool have_r1 = !two || q0 == r + 1 || q1 == r + 1;
            int l0 = -1, l1 = -1;  // rows loaded into R0 / R1 at this step
            if (!have_r && !have_r1) {
                l0 = r;
                l1 = r + 1;
            } else if (!have_r) {
                const int s = two ? (q0 == r + 1 ? 1 : 0) : lru;
                (s == 0 ? l0 : l1) = r;
            } else if (!have_r1) {
                (q0 == r ? l1 : l0) = r + 1;
            }
            if (l0 >= 0) {
                if (lane == 0) list[planned & (kFrameLaneList - 1)] = l0;
                ++planned;
                q0 = l0;
                act |= kActL0;
                lru = 1;
            }
            if (l1 >= 0) {
                if (lane == 0) list[planned & (kFrameLaneList - 1)] = l1;
                ++planned;
                q1 = l1;
                act |= kActL1;
                lru = 0;
            }
            if (q0 == r) act |= kActRin0;
            if (lane == 0) s_act[buf * 32 + p] = act;
        }
        __syncwarp();
    };
    // One (voxel i, element) point from slot p of batch buffer `buf`.
    auto step = [&](float2 (&A0)[J], float2 (&A1)[kCplx ? J : 1], int buf, int p) {
        const int act = s_act[buf * 32 + p];
        const float4 ca = s_coef[(buf * 32 + p) * kCoef];
        const float4 cb = kCplx ? s_coef[(buf * 32 + p) * kCoef + kCoef - 1] : ca;
        bool rin0;
        if constexpr (RING) {
            if (act & kActL0) consume(R0);
            if (act & kActL1) consume(R1);
            if ((act & (kActL0 | kActL1)) && tail - head <= K / 2) issue();  // refill half a ring at a time
            rin0 = (act & kActRin0) != 0;
        } else {
            const int r = act >> kActShift;
            if (act & kActTwo) {
                rin0 = q0 == r || (q1 != r && q0 != r + 1);
                if (rin0) {
                    if (q0 != r) { load_row(R0, r); q0 = r; }
                    if (q1 != r + 1) { load_row(R1, r + 1); q1 = r + 1; }
                } else {
                    if (q1 != r) { load_row(R1, r); q1 = r; }
                    if (q0 != r + 1) { load_row(R0, r + 1); q0 = r + 1; }
                }
            } else {
                if (q0 != r && q1 != r) { load_row(R0, r); q0 = r; }
                rin0 = q0 == r;
            }
        }
        if (INTERP == kLinear && (act & kActTwo)) {
            // complex: ca = (a cw, a cw, a sw, a sw), cb = (b cw, ...); real: ca = (a w, a w, b w, b w)
            if (rin0) {
                if constexpr (kCplx) mac2(A0, A1, R0, R1, ca, cb);
                else mac2(A0, A1, R0, R1, ca, ca);
            } else {
                if constexpr (kCplx) mac2(A0, A1, R1, R0, ca, cb);
                else mac2(A0, A1, R1, R0, ca, ca);
            }
        } else {
            if (rin0) mac1(A0, A1, R0, ca);
            else mac1(A0, A1, R1, ca);
        }
    };

    int buf = 0;
    unsigned mask = n_batches > 0 ? params(0, 0) : 0u;
    if constexpr (RING) {
        plan(0, mask);
        issue();
    }
    for (int bi = 0; bi < n_batches && !failed; ++bi) {
        unsigned next = 0u;
        if (bi + 1 < n_batches) {  // the next batch's parameters and copies, ahead of this batch's steps
            next = params(bi + 1, buf ^ 1);
            if constexpr (RING) {
                plan(buf ^ 1, next);
                issue();
            }
        }
        while (mask != 0u && !failed) {
            const int eo = (__ffs(mask) - 1) / G;
            const unsigned m = (mask >> (eo * G)) & kGMask;
            mask &= ~(kGMask << (eo * G));
#pragma unroll
            for (int i = 0; i < G; ++i) {
                if ((m >> i) & 1u) step(acc0[i], acc1[i], buf, eo * G + i);
            }
        }
        __syncwarp();  // this buffer's parameters are rewritten two batches on
        buf ^= 1;
        mask = next;
    }
    if constexpr (RING) {
        if (failed) {
            // Give the copies in flight a bounded chance to land before the warp moves on.
            for (; head < tail; ++head) ring_wait(bars + (head & (K - 1)), static_cast<uint32_t>(head >> fl.ring_log2) & 1u);
        }
        __syncwarp();
        if (lane == 0) {
            for (int k = 0; k < K; ++k) mbar_inval(bars + k);  // re-initialised by the next block
            if (failed) atomicOr(fl.status, 1);
        }
        __syncwarp();
        if (failed) return;
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

template <int S, int INTERP, int J, int G, bool SPLIT, bool RING>
__device__ __forceinline__ void frame_lane_block(const DasArgs& a, const FrameLaneArgs& fl, int64_t block,
                                                 unsigned char* smem_raw) {
    const int w0 = static_cast<int>(block % fl.n_chunks) * 32 * J;
    if (fl.words - w0 >= 32 * J) {
        frame_lane_block_impl<S, INTERP, J, G, SPLIT, RING, true>(a, fl, block, smem_raw);
    } else {
        frame_lane_block_impl<S, INTERP, J, G, SPLIT, RING, false>(a, fl, block, smem_raw);
    }
}

template <int S, int INTERP, int J, int G, bool SPLIT, bool RING>
__global__ void __launch_bounds__(kFrameLaneThreads, 4)
    das_frame_lane_kernel(const __grid_constant__ DasArgs a, const __grid_constant__ FrameLaneArgs fl) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    frame_lane_block<S, INTERP, J, G, SPLIT, RING>(a, fl, blockIdx.x, smem_raw);
}

}  // namespace mach_b200
