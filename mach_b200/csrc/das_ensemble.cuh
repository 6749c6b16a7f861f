// Ensemble kernel: multi-frame (Doppler / ensemble) gather with the sample window held in
// tensor memory.
//
// Work item = (voxel tile of 128, block of 32 lanes of frames).  Each CTA has four teams of
// four warps; team q is warps {q, q+4, q+8, q+12}, i.e. the warps of SM sub-partition q,
// and it owns TMEM lanes [32q, 32q + 32).  Lane l of every warp of the team stands for
// frame l of the block (complex storage) or frames 2l, 2l+1 (real storage), so a tap row of
// the window is one TMEM column pair per lane and every lane of a warp reads the SAME
// column for a voxel: a gather with a warp-uniform column address, which tcgen05.ld does
// without touching shared memory.  Per (element, transmit) step of a team:
//   a. each team thread turns its voxel's delay into a tap row, fraction and weights
//      (mach's FP32 arithmetic, or the split FP64 base + FP32 fraction), and the team's
//      row window [lo, hi] is reduced;
//   b. thread 0 of the team streams the window rows [lo, lo + W) x the frame block in
//      with one TMA 2-D tile copy (cp.async.bulk.tensor, mbarrier completion);
//   c. the team's warps widen the rows to FP32 and store them into TMEM (tcgen05.st);
//   d. each warp gathers its 32 voxels: one tcgen05.ld (both taps, both components) per
//      voxel, then lerp, rotation and accumulation in FP32 registers.
// Steps are pipelined: parameters and the window copy run two steps ahead of the gather
// (three shared-memory windows, four parameter slots, two TMEM windows), with one named
// barrier per team and step.  Teams take items from a device counter, heaviest first
// (deep tiles have the widest aperture), so the tail of a launch is made of light items.  A step whose rows do not fit the window gathers
// straight from global memory.  All mbarrier waits are bounded; on a timeout the team
// records an error in the status word and stops.  Every CTA frees its tensor memory
// before it exits.
#pragma once

#include <cuda.h>

#include "das_staged.cuh"

namespace mach_b200 {

constexpr int kEnsTeams = 4;
constexpr int kEnsTeamThreads = 128;
constexpr int kEnsThreads = kEnsTeams * kEnsTeamThreads;  // 512
constexpr int kEnsTileVoxels = 128;                      // one voxel per team thread
constexpr int kEnsMaxPrefetchTx = 16;                    // arrivals of <= 16 transmits staged per item
constexpr int kEnsMaxWindow = 64;

constexpr int kEnsWindows = 3;  // shared-memory windows in flight
constexpr int kEnsSlots = 4;    // parameter slots (steps k .. k + 2 plus one being read)

struct EnsembleArgs {
    int* counter;         // work-item counter, zero at launch
    int32_t window_rows;  // W: rows per window, a multiple of 16 in [16, 64]
    int32_t n_tiles;      // voxel tiles
    int32_t n_fblocks;    // frame blocks (32 lanes each)
    int32_t box_x;        // TMA box width in tensor-map elements (one frame block)
    uint32_t tmem_cols;   // TMEM columns allocated per CTA (power of two >= 32)
    int32_t team_bytes;   // dynamic shared memory per team
};

// ------------------------------------------------------------------ lane words

// One lane's sample of one row: a complex frame, or a pair of real frames.
template <int S>
struct LaneWord;
template <>
struct LaneWord<kC64> {
    using W = uint2;
    static constexpr int kFrames = 1;
    __device__ __forceinline__ static float2 widen(W w) { return make_float2(__uint_as_float(w.x), __uint_as_float(w.y)); }
};
template <>
struct LaneWord<kF32> {
    using W = uint2;
    static constexpr int kFrames = 2;
    __device__ __forceinline__ static float2 widen(W w) { return make_float2(__uint_as_float(w.x), __uint_as_float(w.y)); }
};
template <>
struct LaneWord<kCF16> {
    using W = uint32_t;
    static constexpr int kFrames = 1;
    __device__ __forceinline__ static float2 widen(W w) { return __half22float2(*reinterpret_cast<const __half2*>(&w)); }
};
template <>
struct LaneWord<kF16> : LaneWord<kCF16> {
    static constexpr int kFrames = 2;
};
template <>
struct LaneWord<kCBF16> {
    using W = uint32_t;
    static constexpr int kFrames = 1;
    __device__ __forceinline__ static float2 widen(W w) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
    }
};
template <>
struct LaneWord<kBF16> : LaneWord<kCBF16> {
    static constexpr int kFrames = 2;
};
template <>
struct LaneWord<kCI16> {
    using W = uint32_t;
    static constexpr int kFrames = 1;
    __device__ __forceinline__ static float2 widen(W w) { return i16x2_to_float2(w); }
};
template <>
struct LaneWord<kI16> : LaneWord<kCI16> {
    static constexpr int kFrames = 2;
};

// ------------------------------------------------------------------ tensor memory, team barriers

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Four rows (8 words) of this lane at columns [col, col + 8).
__device__ __forceinline__ void tmem_st8(uint32_t col, const float2 (&v)[4]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(col),
                 "r"(__float_as_uint(v[0].x)), "r"(__float_as_uint(v[0].y)), "r"(__float_as_uint(v[1].x)),
                 "r"(__float_as_uint(v[1].y)), "r"(__float_as_uint(v[2].x)), "r"(__float_as_uint(v[2].y)),
                 "r"(__float_as_uint(v[3].x)), "r"(__float_as_uint(v[3].y))
                 : "memory");
}
// Four loads of (row, row + 1) at columns c0..c3 and the wait for them, in one statement:
// the outputs are only defined once tcgen05.wait::ld has retired the loads.  No memory
// clobber: tensor memory is not addressable memory, and the statement stays ordered after
// the tcgen05.st and fence statements of the copy (all volatile), so shared-memory loads of
// the next voxels may be scheduled around it.
__device__ __forceinline__ void tmem_ld4x4(const uint32_t (&c)[4], uint32_t (&r)[4][4]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%16];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%4, %5, %6, %7}, [%17];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%8, %9, %10, %11}, [%18];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%12, %13, %14, %15}, [%19];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0][0]), "=r"(r[0][1]), "=r"(r[0][2]), "=r"(r[0][3]), "=r"(r[1][0]), "=r"(r[1][1]), "=r"(r[1][2]),
          "=r"(r[1][3]), "=r"(r[2][0]), "=r"(r[2][1]), "=r"(r[2][2]), "=r"(r[2][3]), "=r"(r[3][0]), "=r"(r[3][1]),
          "=r"(r[3][2]), "=r"(r[3][3])
        : "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]));
}
// Same for one row (nearest taps); the second row of each result repeats the first.
__device__ __forceinline__ void tmem_ld4x2(const uint32_t (&c)[4], uint32_t (&r)[4][4]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%8];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%9];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4, %5}, [%10];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%6, %7}, [%11];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0][0]), "=r"(r[0][1]), "=r"(r[1][0]), "=r"(r[1][1]), "=r"(r[2][0]), "=r"(r[2][1]), "=r"(r[3][0]),
          "=r"(r[3][1])
        : "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        r[i][2] = r[i][0];
        r[i][3] = r[i][1];
    }
}

__device__ __forceinline__ void team_sync(int team) {
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(kEnsTeamThreads) : "memory");
}
// Team barrier that also ORs a flag over the team.
__device__ __forceinline__ bool team_sync_or(int team, bool flag) {
    uint32_t r;
    asm volatile(
        "{ .reg .pred pi, po; setp.ne.u32 pi, %1, 0; bar.red.or.pred po, %2, %3, pi; selp.u32 %0, 1, 0, po; }"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(flag)), "r"(team + 1), "r"(kEnsTeamThreads)
        : "memory");
    return r != 0;
}

// ------------------------------------------------------------------ shared memory per team

struct EnsembleTeamSmem {
    unsigned char* win;  // [kEnsWindows][W][32] lane words
    StepParam* param;    // [kEnsSlots][128]
    int2* lohi;          // [kEnsSlots][4] per-warp window partials (lo, hi)
    unsigned* valid;     // [kEnsSlots][4] per-warp validity ballots
    int* count;          // [4]
    float* bbox;         // [4][5]
    float* arr;          // [n_pref][128]
    int64_t* vox;        // [128] voxel index of each tile slot (-1 outside the grid)
    int* cand;           // [128] candidate elements of the current element block
    int* item;           // [2] current work item
    uint64_t* bar;       // [kEnsWindows]
};

__host__ __device__ inline int ensemble_team_bytes(int window_rows, int lane_word_bytes, int n_pref) {
    int b = kEnsWindows * window_rows * 32 * lane_word_bytes;  // windows
    b += kEnsSlots * kEnsTileVoxels * static_cast<int>(sizeof(StepParam));
    b += (kEnsSlots * 4 * 2 + kEnsSlots * 4 + 4) * 4 + 4 * 5 * 4;  // partials, ballots, counts, bbox
    b += n_pref * kEnsTileVoxels * 4;                          // arrivals
    b += kEnsTileVoxels * 8;                                   // voxel indices
    b += kEnsTileVoxels * 4;                                   // candidates
    b += 2 * 4;                                                // work item
    b = (b + 7) & ~7;
    b += kEnsWindows * 8;                                      // mbarriers
    return (b + 127) & ~127;
}

__device__ __forceinline__ EnsembleTeamSmem team_smem(unsigned char* base, int window_rows, int lwb, int n_pref) {
    EnsembleTeamSmem s;
    unsigned char* p = base;
    s.win = p;
    p += kEnsWindows * window_rows * 32 * lwb;
    s.param = reinterpret_cast<StepParam*>(p);
    p += kEnsSlots * kEnsTileVoxels * sizeof(StepParam);
    s.lohi = reinterpret_cast<int2*>(p);  // 16-byte aligned: read as two int4 per slot
    p += kEnsSlots * 4 * 2 * 4;
    s.valid = reinterpret_cast<unsigned*>(p);
    p += kEnsSlots * 4 * 4;
    s.count = reinterpret_cast<int*>(p);
    p += 4 * 4;
    s.bbox = reinterpret_cast<float*>(p);
    p += 4 * 5 * 4;
    s.arr = reinterpret_cast<float*>(p);
    p += n_pref * kEnsTileVoxels * 4;
    s.vox = reinterpret_cast<int64_t*>(p);
    p += kEnsTileVoxels * 8;
    s.cand = reinterpret_cast<int*>(p);
    p += kEnsTileVoxels * 4;
    s.item = reinterpret_cast<int*>(p);
    p += 2 * 4;
    p = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t{7});
    s.bar = reinterpret_cast<uint64_t*>(p);
    return s;
}

// ------------------------------------------------------------------ the kernel

constexpr int kEnsModeEmpty = 0, kEnsModeWindow = 1, kEnsModeDirect = 2;

template <int S, int INTERP, bool SPLIT>
__global__ void __launch_bounds__(kEnsThreads, 1)
    das_ensemble_kernel(const __grid_constant__ DasArgs a, const __grid_constant__ StagedArgs st,
                        const __grid_constant__ EnsembleArgs ea, const __grid_constant__ CUtensorMap tmap) {
    static_assert(INTERP == kNearest || INTERP == kLinear, "ensemble kernel: nearest or linear taps");
    using LW = LaneWord<S>;
    using Word = typename LW::W;
    constexpr bool kCplx = Storage<S>::kComplex;
    constexpr int kLwb = sizeof(Word);
    constexpr unsigned kFull = 0xffffffffu;

    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t s_tmem;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int team = warp & 3;  // sub-partition = TMEM lane quadrant
    const int tw = warp >> 2;   // warp within the team
    const int tt = tw * 32 + lane;
    const int W = ea.window_rows;
    const int n_pref = a.n_tx <= kEnsMaxPrefetchTx ? a.n_tx : 0;
    EnsembleTeamSmem s = team_smem(smem + team * ea.team_bytes, W, kLwb, n_pref);

    if (tt == 0) {
#pragma unroll
        for (int i = 0; i < kEnsWindows; ++i) mbar_init(&s.bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&s_tmem, ea.tmem_cols);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tbase = s_tmem + (static_cast<uint32_t>(team * 32) << 16);

    const int64_t n_frames = a.n_frames;
    const int64_t row_words = static_cast<int64_t>(a.n_frames) / LW::kFrames;  // lane words per sample row
    const int n_items = ea.n_tiles * ea.n_fblocks;
    uint32_t phase = 0u;    // bit b: parity of the next completion of buffer b's mbarrier
    uint32_t pending = 0u;  // bit b: a copy was issued on buffer b and has not been waited for
    bool dead = false;

    for (;;) {
        team_sync(team);  // the previous item's shared state is consumed
        if (tt == 0) s.item[0] = atomicAdd(ea.counter, 1);
        team_sync(team);
        const int item = s.item[0];
        if (item >= n_items) break;
        // Tiles in reverse order: for a scan ordered depth-fastest the deepest (widest
        // aperture, most candidate elements) come first.
        const int tile = ea.n_tiles - 1 - item % ea.n_tiles;
        const int fb = item / ea.n_tiles;
        const int64_t word0 = static_cast<int64_t>(fb) * 32 + lane;  // this lane's word within a row
        const bool lane_ok = word0 < row_words;

        // ---- this thread's voxel, its arrivals, the tile bounding box
        // Team thread (tw, lane) owns tile slot 4 * (4 * (lane >> 2) + tw) + (lane & 3): each warp
        // holds every fourth column of 4-voxel runs along the contiguous axis, so the four
        // warps see similar apertures and finish their gathers together.
        const int64_t pv = tile_voxel(a, st, tile, 4 * (4 * (lane >> 2) + tw) + (lane & 3));
        s.vox[tt] = pv;
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (pv >= 0) {
            vx = __ldg(a.scan + 3 * pv + 0);
            vy = __ldg(a.scan + 3 * pv + 1);
            vz = __ldg(a.scan + 3 * pv + 2);
        }
        const float radius = __fdiv_rn(vz, a.two_f_number);  // kernel.cu:583
        const float radius_sq = __fmul_rn(radius, radius);
        for (int t = 0; t < n_pref; ++t) {
            s.arr[t * kEnsTileVoxels + tt] = pv >= 0 ? __ldg(a.arrivals + static_cast<int64_t>(t) * a.n_vox + pv) : 0.f;
        }
        {
            float b[5] = {pv >= 0 ? vx : INFINITY, pv >= 0 ? -vx : INFINITY, pv >= 0 ? vy : INFINITY,
                          pv >= 0 ? -vy : INFINITY, pv >= 0 ? -fabsf(radius) : INFINITY};
#pragma unroll
            for (int k = 0; k < 5; ++k) {
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) b[k] = fminf(b[k], __shfl_xor_sync(kFull, b[k], off));
            }
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < 5; ++k) s.bbox[tw * 5 + k] = b[k];
            }
        }
        team_sync(team);
        float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY, rmax = 0.f;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            bx0 = fminf(bx0, s.bbox[w * 5 + 0]);
            bx1 = fmaxf(bx1, -s.bbox[w * 5 + 1]);
            by0 = fminf(by0, s.bbox[w * 5 + 2]);
            by1 = fmaxf(by1, -s.bbox[w * 5 + 3]);
            rmax = fmaxf(rmax, -s.bbox[w * 5 + 4]);
        }
        const float cand_r2 = rmax * rmax * 1.00001f + 1e-30f;

        float2 acc[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = make_float2(0.f, 0.f);

        // receive-path state of this thread's voxel (reused across the transmits of an element)
        int rx_elem = -1;
        float dist = 0.f, weight_scaled = 0.f;
        bool pair_ok = false;
        SplitPos rx_pos{};
        float rx_cyc = 0.f;

        for (int eb = 0; eb < a.n_rx && !dead; eb += kEnsTileVoxels) {
            // ---- candidate elements of this block, compacted in element order
            bool cand = false;
            const int e_test = eb + tt;
            if (e_test < a.n_rx) {
                const float ex = __ldg(a.rx + 3 * e_test + 0);
                const float ey = __ldg(a.rx + 3 * e_test + 1);
                const float ddx = fmaxf(fmaxf(bx0 - ex, ex - bx1), 0.f);
                const float ddy = fmaxf(fmaxf(by0 - ey, ey - by1), 0.f);
                cand = ddx * ddx + ddy * ddy <= cand_r2;
            }
            const unsigned m = __ballot_sync(kFull, cand);
            team_sync(team);  // the previous block's candidates are consumed
            if (lane == 0) s.count[tw] = __popc(m);
            team_sync(team);
            int base = 0, total = 0;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int c = s.count[w];
                base += w < tw ? c : 0;
                total += c;
            }
            if (cand) s.cand[base + __popc(m & ((1u << lane) - 1u))] = e_test;
            team_sync(team);
            if (total == 0) continue;
            const int n_steps = total * a.n_tx;

            // ---- parameters of one step for this thread's voxel into slot `slot`
            int p_ci = 0, p_t = 0;  // step cursor of the parameter phase
            auto make_params = [&](int slot) {
                const int e = s.cand[p_ci];
                const int t = p_t;
                if (++p_t == a.n_tx) {
                    p_t = 0;
                    ++p_ci;
                }
                if (e != rx_elem) {
                    rx_elem = e;
                    const float ex = __ldg(a.rx + 3 * e + 0), ey = __ldg(a.rx + 3 * e + 1), ez = __ldg(a.rx + 3 * e + 2);
                    const float dx = __fsub_rn(ex, vx);
                    const float dy = __fsub_rn(ey, vy);
                    const float dz = __fsub_rn(ez, vz);
                    const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                    if (SPLIT) {
                        const double ddx = static_cast<double>(ex) - vx, ddy = static_cast<double>(ey) - vy,
                                     ddz = static_cast<double>(ez) - vz;
                        const double d = sqrt(fma(ddx, ddx, fma(ddy, ddy, ddz * ddz)));
                        rx_pos = split_position(d * a.fs_over_c);
                        rx_cyc = reduced_cycles(d * a.fmod_over_c);
                    } else {
                        dist = __fsqrt_rn(__fmaf_rn(dz, dz, h2));  // kernel.cu:467
                    }
                    float weight = 1.0f;
                    if (a.apod) weight = fast_tukey(h2, radius, a);
                    pair_ok = pv >= 0 && !(h2 > radius_sq) && !(weight == 0.0f);
                    weight_scaled = __fmul_rn(weight, a.scale);
                }
                StepParam p{-(1 << 28), 0.f, 0.f, 0.f};
                int lo = 0x7fffffff, hi = -1;
                bool ok = false;
                if (pair_ok) {
                    const float txa = n_pref ? s.arr[t * kEnsTileVoxels + tt]
                                             : __ldg(a.arrivals + static_cast<int64_t>(t) * a.n_vox + pv);
                    TapPosition tp{};
                    float sn = 0.f, cs = 1.f;
                    if (SPLIT) {
                        const SplitPos tx_pos = split_position((static_cast<double>(txa) - a.t0_d) * a.fs_d);
                        int sbase = tx_pos.base + rx_pos.base;
                        float frac = __fadd_rn(tx_pos.frac, rx_pos.frac);
                        if (frac >= 1.0f) {
                            frac = __fsub_rn(frac, 1.0f);
                            sbase += 1;
                        }
                        ok = !(sbase < a.start_base || (sbase == a.start_base && frac < a.start_frac));
                        ok = ok && split_tap_position<INTERP>(sbase, frac, a.n_samples, tp);
                        if (ok && kCplx && a.rotate) {
                            split_phasor(__fadd_rn(reduced_cycles(static_cast<double>(txa) * a.fmod_d), rx_cyc), sn, cs);
                        }
                    } else {
                        const float tau = __fmaf_rn(dist, a.inv_c, txa);  // kernel.cu:470
                        const float sp = __fmul_rn(__fsub_rn(tau, a.t0), a.fs);  // kernel.cu:637
                        ok = !(tau < 0.0f);                                     // kernel.cu:634
                        if constexpr (INTERP == kNearest) {
                            ok = ok && (sp >= -0.5f) && (sp <= a.hi_nearest);
                        } else {
                            ok = ok && (sp >= 0.0f) && (sp <= a.hi_linear);
                        }
                        tp = tap_position<INTERP>(sp);
                        if constexpr (INTERP == kNearest) ok = ok && tp.idx < a.n_samples;
                        if (ok && kCplx && a.rotate) {
                            __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
                        }
                    }
                    if (ok) {
                        p.row = tp.idx;
                        p.w = INTERP == kLinear ? tp.w0 : 0.f;
                        p.cw = weight_scaled;
                        if (kCplx && a.rotate) {
                            p.cw = __fmul_rn(cs, weight_scaled);
                            p.sw = __fmul_rn(sn, weight_scaled);
                        }
                        lo = tp.idx;
                        hi = INTERP == kLinear ? tp.idx + 1 : tp.idx;  // both linear taps are always staged
                    }
                }
                s.param[slot * kEnsTileVoxels + tt] = p;
                const unsigned vmask = __ballot_sync(kFull, ok);
                lo = __reduce_min_sync(kFull, lo);
                hi = __reduce_max_sync(kFull, hi);
                if (lane == 0) {
                    s.lohi[slot * 4 + tw] = make_int2(lo, hi);
                    s.valid[slot * 4 + tw] = vmask;
                }
            };
            // ---- after the team barrier: step k's window and mode (every thread), copy start (thread 0)
            int w_ci = 0, w_t = 0;  // step cursor of the window phase
            auto plan_window = [&](int slot, int b, int& lo_out) -> int {
                const int4 q0 = reinterpret_cast<const int4*>(s.lohi + slot * 4)[0];
                const int4 q1 = reinterpret_cast<const int4*>(s.lohi + slot * 4)[1];
                const int lo = min(min(q0.x, q0.z), min(q1.x, q1.z));
                const int hi = max(max(q0.y, q0.w), max(q1.y, q1.w));
                const int e = s.cand[w_ci];
                const int t = w_t;
                if (++w_t == a.n_tx) {
                    w_t = 0;
                    ++w_ci;
                }
                lo_out = lo;
                int mode = kEnsModeEmpty;
                if (hi >= lo) mode = (st.use_tma && hi - lo + 1 <= W) ? kEnsModeWindow : kEnsModeDirect;
                if (mode == kEnsModeWindow && tt == 0) {
                    const int row0 = (t * a.n_rx + e) * a.n_samples + lo;
                    mbar_expect_tx(&s.bar[b], static_cast<uint32_t>(W * 32 * kLwb));
                    tma_load_2d(s.win + b * W * 32 * kLwb, &tmap, fb * ea.box_x, row0, &s.bar[b]);
                }
                if (mode == kEnsModeWindow) pending |= 1u << b;
                return mode;
            };

            // Planned steps k and k + 1: window start, mode, element, transmit.
            int q_lo[2] = {0, 0}, q_mode[2] = {kEnsModeEmpty, kEnsModeEmpty}, q_e[2] = {0, 0}, q_t[2] = {0, 0};
            make_params(0);
            if (n_steps > 1) make_params(1);
            tmem_fence_before();
            team_sync(team);
            tmem_fence_after();
            q_e[0] = s.cand[w_ci];
            q_t[0] = w_t;
            q_mode[0] = plan_window(0, 0, q_lo[0]);
            if (n_steps > 1) {
                q_e[1] = s.cand[w_ci];
                q_t[1] = w_t;
                q_mode[1] = plan_window(1, 1, q_lo[1]);
            }

            int wb = 0;  // shared-memory window of step k (k % 3)
            for (int k = 0; k < n_steps; ++k) {
                const int slot = k & (kEnsSlots - 1);
                const int tb = k & 1;  // TMEM window of step k
                const int wb2 = wb == 0 ? 2 : wb - 1;  // window of step k + 2
                const int cur_lo = q_lo[0], cur_mode = q_mode[0], cur_e = q_e[0], cur_t = q_t[0];
                if (k + 2 < n_steps) make_params((k + 2) & (kEnsSlots - 1));
                // ---- window k: wait for its copy, widen its rows into TMEM (this warp's quarter)
                bool timed_out = false;
                const int b = wb;
                if (cur_mode == kEnsModeWindow) {
                    if (mbar_wait(&s.bar[b], (phase >> b) & 1u)) {
                        phase ^= 1u << b;
                        pending &= ~(1u << b);
                    } else {
                        timed_out = true;  // the copy stays pending; the exit path waits for it once more
                    }
                    // tcgen05.st is warp-collective: the whole warp copies or none of it does.
                    timed_out = __any_sync(kFull, timed_out);
                    if (!timed_out) {
                        // This warp's quarter of the rows, four rows (one 8-column store) at a time;
                        // W / 4 is a multiple of 4 and at most 16.
                        const int rows = W >> 2;
                        const int r0 = tw * rows;
                        const Word* src = reinterpret_cast<const Word*>(s.win + b * W * 32 * kLwb) + r0 * 32 + lane;
                        const uint32_t col0 = tbase + static_cast<uint32_t>(tb * 2 * W + 2 * r0);
#pragma unroll
                        for (int j = 0; j < kEnsMaxWindow / 16; ++j) {
                            if (4 * j < rows) {
                                float2 v[4];
#pragma unroll
                                for (int q = 0; q < 4; ++q) v[q] = LW::widen(src[(4 * j + q) * 32]);
                                tmem_st8(col0 + static_cast<uint32_t>(8 * j), v);
                            }
                        }
                        tmem_wait_st();
                    }
                }
                tmem_fence_before();
                if (team_sync_or(team, timed_out)) {
                    dead = true;
                    break;
                }
                tmem_fence_after();
                // ---- start the copy of step k + 2
                int n_lo = 0, n_mode = kEnsModeEmpty, n_e = 0, n_t = 0;
                if (k + 2 < n_steps) {
                    n_e = s.cand[w_ci];
                    n_t = w_t;
                    n_mode = plan_window((k + 2) & (kEnsSlots - 1), wb2, n_lo);
                }
                // ---- gather step k
                const unsigned vm = s.valid[slot * 4 + tw];
                const StepParam* prm = s.param + slot * kEnsTileVoxels + tw * 32;
                if (cur_mode == kEnsModeWindow && vm != 0u) {
                    const int colb = static_cast<int>(tbase) + tb * 2 * W;  // column of row lo
                    const int cb = colb - 2 * cur_lo;
#pragma unroll
                    for (int g = 0; g < 8; ++g) {
                        if (((vm >> (4 * g)) & 0xfu) == 0u) continue;
                        StepParam p[4];
                        uint32_t r[4][4], col[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            p[i] = prm[4 * g + i];
                            col[i] = static_cast<uint32_t>(max(2 * p[i].row + cb, colb));
                        }
                        if constexpr (INTERP == kLinear) {
                            tmem_ld4x4(col, r);
                        } else {
                            tmem_ld4x2(col, r);
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float ax = __uint_as_float(r[i][0]), ay = __uint_as_float(r[i][1]);
                            float vx_, vy_;
                            if constexpr (INTERP == kLinear) {
                                const float bx = __uint_as_float(r[i][2]), by = __uint_as_float(r[i][3]);
                                vx_ = __fmaf_rn(p[i].w, __fsub_rn(bx, ax), ax);  // a + t (b - a)
                                vy_ = __fmaf_rn(p[i].w, __fsub_rn(by, ay), ay);
                            } else {
                                vx_ = ax;
                                vy_ = ay;
                            }
                            float2& o = acc[4 * g + i];
                            if constexpr (kCplx) {
                                o.x = __fmaf_rn(vx_, p[i].cw, __fmaf_rn(-vy_, p[i].sw, o.x));
                                o.y = __fmaf_rn(vy_, p[i].cw, __fmaf_rn(vx_, p[i].sw, o.y));
                            } else {
                                o.x = __fmaf_rn(vx_, p[i].cw, o.x);
                                o.y = __fmaf_rn(vy_, p[i].cw, o.y);
                            }
                        }
                    }
                } else if (cur_mode == kEnsModeDirect && vm != 0u && lane_ok) {
                    const Word* grow = static_cast<const Word*>(a.channel) +
                                       static_cast<int64_t>(cur_t * a.n_rx + cur_e) * a.n_samples * row_words + word0;
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        if (!((vm >> i) & 1u)) continue;
                        const StepParam p = prm[i];
                        const Word* q = grow + static_cast<int64_t>(p.row) * row_words;
                        const float2 va = LW::widen(__ldg(q));
                        float2 v = va;
                        if constexpr (INTERP == kLinear) {
                            const float2 vb = LW::widen(__ldg(q + (p.w > 0.0f ? row_words : 0)));
                            v.x = __fmaf_rn(p.w, __fsub_rn(vb.x, va.x), va.x);
                            v.y = __fmaf_rn(p.w, __fsub_rn(vb.y, va.y), va.y);
                        }
                        float2& o = acc[i];
                        if constexpr (kCplx) {
                            o.x = __fmaf_rn(v.x, p.cw, __fmaf_rn(-v.y, p.sw, o.x));
                            o.y = __fmaf_rn(v.y, p.cw, __fmaf_rn(v.x, p.sw, o.y));
                        } else {
                            o.x = __fmaf_rn(v.x, p.cw, o.x);
                            o.y = __fmaf_rn(v.y, p.cw, o.y);
                        }
                    }
                }
                q_lo[0] = q_lo[1];
                q_mode[0] = q_mode[1];
                q_e[0] = q_e[1];
                q_t[0] = q_t[1];
                q_lo[1] = n_lo;
                q_mode[1] = n_mode;
                q_e[1] = n_e;
                q_t[1] = n_t;
                wb = wb == 2 ? 0 : wb + 1;
            }
        }
        if (dead) break;

        // ---- power-Doppler epilogue: |x|^2 summed over this frame block (the warp's lanes),
        // one atomic add per voxel (frame blocks of a voxel add in any order)
        if (a.power) {
            float mine = 0.f;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                float pw = lane_ok ? __fmaf_rn(acc[i].x, acc[i].x, __fmul_rn(acc[i].y, acc[i].y)) : 0.f;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) pw += __shfl_xor_sync(kFull, pw, off);
                if (lane == i) mine = pw;
            }
            const int64_t v = s.vox[tw * 32 + lane];
            if (v >= 0) atomicAdd(static_cast<float*>(a.out) + v, mine);
            continue;
        }
        // ---- write this item's sums: lane word `word0` of each of this warp's 32 voxels
        if (lane_ok) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int64_t v = s.vox[tw * 32 + i];
                if (v < 0) continue;
                float2 res = acc[i];
                if constexpr (kCplx) {
                    float2* o = static_cast<float2*>(a.out) + v * n_frames + word0;
                    if (a.accumulate) {
                        const float2 prev = *o;
                        res.x = __fadd_rn(prev.x, res.x);
                        res.y = __fadd_rn(prev.y, res.y);
                    }
                    *o = res;
                } else {
                    float2* o = reinterpret_cast<float2*>(static_cast<float*>(a.out) + v * n_frames + 2 * word0);
                    if (a.accumulate) {
                        const float2 prev = *o;
                        res.x = __fadd_rn(prev.x, res.x);
                        res.y = __fadd_rn(prev.y, res.y);
                    }
                    *o = res;
                }
            }
        }
    }

    if (dead) {
        // Give copies still in flight a bounded chance to land before the CTA exits.
#pragma unroll
        for (int i = 0; i < kEnsWindows; ++i) {
            if ((pending >> i) & 1u) mbar_wait(&s.bar[i], (phase >> i) & 1u);
        }
        if (tt == 0) atomicOr(st.status, 1);
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    if (warp == 0) tmem_dealloc(s_tmem, ea.tmem_cols);
}

}  // namespace mach_b200
