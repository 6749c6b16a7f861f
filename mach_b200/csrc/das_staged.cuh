// Staged multi-frame gather kernel (ensembles: Doppler, multi-frame 3-D).
//
// With many frames per (voxel, element, transmit) point the delay arithmetic is amortised
// and the cost is moving samples: every point reads 2-3 taps x frames.  Neighbouring
// voxels read overlapping sample rows, so a CTA works on a compact tile of 128 voxels
// (a block of the voxel grid when its shape is known) and a chunk of frames, and for
// each (element, transmit) step:
//   1. threads 0-127 turn their voxel's delay into a tap row and weights (receive path
//      reused across transmits), and the row window [lo, hi] the tile needs is reduced;
//   2. one thread issues a TMA 2-D tile copy (cp.async.bulk.tensor) of rows [lo, lo + W)
//      x the frame chunk into shared memory, completing on an mbarrier;
//   3. every warp gathers its voxels' taps from shared memory (lane = frames, 8-byte
//      vector per lane), interpolates and rotates with packed FP32x2 FMAs, accumulating
//      in registers.
// Steps are software-pipelined: the window for step k+1 streams in while step k computes
// (window double-buffered, parameters triple-buffered, one __syncthreads per step).  A
// step whose window is taller than W reads its taps straight from global memory instead.
// All waits on the mbarrier are bounded; on timeout the kernel records an error in the
// status word and leaves the tile's output untouched.
#pragma once

#include <cuda.h>

#include "das_lane_voxel.cuh"

namespace mach_b200 {

constexpr int kStagedThreads = 256;
constexpr int kTileVoxels = 128;
constexpr int kStagedWarps = kStagedThreads / 32;
constexpr int kVoxelsPerWarp = kTileVoxels / kStagedWarps;  // 16
constexpr int kMaxElemBlock = 256;                           // elements tested per candidate pass

struct StagedArgs {
    int32_t use_tma;          // 1: stage windows with TMA; 0: gather from global memory
    int32_t window_rows;      // TMA box height (rows of samples per window)
    int32_t grid_fast;        // voxel grid extents, fast (contiguous) axis first; 0 = 1-D tiling
    int32_t grid_mid;
    int32_t grid_slow;
    int32_t tile_fast;        // tile extents (tile_fast * tile_mid * tile_slow == 128)
    int32_t tile_mid;
    int32_t tile_slow;
    int32_t tiles_fast;       // number of tiles along the fast and mid axes
    int32_t tiles_mid;
    int32_t* status;          // device status word: 1 = an mbarrier wait timed out
};

// ------------------------------------------------------------------ packed FP32x2 helpers

__device__ __forceinline__ unsigned long long pk(float2 v) {
    return (static_cast<unsigned long long>(__float_as_uint(v.y)) << 32) | __float_as_uint(v.x);
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
    return make_float2(__uint_as_float(static_cast<unsigned>(r)), __uint_as_float(static_cast<unsigned>(r >> 32)));
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}

// ------------------------------------------------------------------ 8-byte lane vectors

// One lane reads 8 bytes per tap: 1 complex64, 2 float32 / complex half / complex int16
// samples, or 4 half / bfloat16 / int16 samples.  unpack() widens them to float2 pairs
// (complex: (I, Q) per frame; real: two consecutive frames).
template <int S>
struct Vec8;

// int16 pair (low, high) of a 32-bit word -> exact floats without the conversion pipe:
// x + 32768 placed in the mantissa of 2^23, minus (2^23 + 32768).
__device__ __forceinline__ float2 i16x2_to_float2(unsigned w) {
    const unsigned u = w ^ 0x80008000u;
    const float lo = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7610));
    const float hi = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7632));
    return sub2(make_float2(lo, hi), make_float2(8421376.0f, 8421376.0f));
}

template <>
struct Vec8<kC64> {
    static constexpr int kPairs = 1;
    __device__ __forceinline__ static void unpack(uint2 r, float2* o) {
        o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
    }
};
template <>
struct Vec8<kF32> {
    static constexpr int kPairs = 1;
    __device__ __forceinline__ static void unpack(uint2 r, float2* o) {
        o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
    }
};
template <>
struct Vec8<kCF16> {
    static constexpr int kPairs = 2;
    __device__ __forceinline__ static void unpack(uint2 r, float2* o) {
        o[0] = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
        o[1] = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    }
};
template <>
struct Vec8<kF16> : Vec8<kCF16> {};
template <>
struct Vec8<kCBF16> {
    static constexpr int kPairs = 2;
    __device__ __forceinline__ static void unpack(uint2 r, float2* o) {
        o[0] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.x));
        o[1] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.y));
    }
};
template <>
struct Vec8<kBF16> : Vec8<kCBF16> {};
template <>
struct Vec8<kCI16> {
    static constexpr int kPairs = 2;
    __device__ __forceinline__ static void unpack(uint2 r, float2* o) {
        o[0] = i16x2_to_float2(r.x);
        o[1] = i16x2_to_float2(r.y);
    }
};
template <>
struct Vec8<kI16> : Vec8<kCI16> {};

// ------------------------------------------------------------------ mbarrier / TMA

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// Bounded wait: each try suspends for at most ~10 us, 2^16 tries bound the wait to well
// under a second; returns false if the phase did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < (1 << 16); ++it) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity), "r"(10000)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// ------------------------------------------------------------------ tile -> voxel index

__device__ __forceinline__ int64_t tile_voxel(const DasArgs& a, const StagedArgs& st, int tile, int local) {
    if (st.grid_fast <= 0) {
        const int64_t v = static_cast<int64_t>(tile) * kTileVoxels + local;
        return v < a.n_vox ? v : -1;
    }
    const int tf = tile % st.tiles_fast;
    const int rest = tile / st.tiles_fast;
    const int tm = rest % st.tiles_mid;
    const int ts = rest / st.tiles_mid;
    const int lf = local % st.tile_fast;
    const int lrest = local / st.tile_fast;
    const int lm = lrest % st.tile_mid;
    const int ls = lrest / st.tile_mid;
    const int f = tf * st.tile_fast + lf;
    const int m = tm * st.tile_mid + lm;
    const int s = ts * st.tile_slow + ls;
    if (f >= st.grid_fast || m >= st.grid_mid || s >= st.grid_slow) return -1;
    return (static_cast<int64_t>(s) * st.grid_mid + m) * st.grid_fast + f;
}

// Per-voxel step parameters in shared memory (16 bytes, one broadcast load per round).
struct alignas(16) StepParam {
    int row;   // tap row (TMA mode: absolute sample index, the window start is subtracted later)
    float w;   // linear: fraction t; quadratic: offset x from the centre tap; nearest: unused
    float cw;  // weight x cos(phase) (real data: the weight)
    float sw;  // weight x sin(phase)
};

constexpr int kMaxPrefetchTx = 32;  // transmit arrivals of the tile staged once in shared memory

// One CTA tile: the tile's 128 voxels x frame chunk `chunk` of job `a`.  `tmap` must live in
// parameter, constant or global memory.  Shared by the per-job and persistent kernels.
template <int S, int INTERP, int LV>
// Returns false if a wait timed out (the caller must then stop using this CTA).
__device__ __forceinline__ bool staged_tile(const DasArgs& a, const StagedArgs& st, const CUtensorMap* tmap,
                                            int tile, int chunk, unsigned char* smem) {
    using ST = Storage<S>;
    using T = typename ST::T;
    constexpr bool kCplx = ST::kComplex;
    constexpr int kEsz = sizeof(T);
    constexpr int VF = 8 / kEsz;                // frames per lane
    constexpr int NP = Vec8<S>::kPairs;         // float2 pairs per lane per tap
    constexpr int G = 32 / LV;                  // voxel streams per warp
    constexpr int ROUNDS = kVoxelsPerWarp / G;  // voxels per stream
    constexpr int FC = LV * VF;                 // frames per CTA
    constexpr int kRowBytes = FC * kEsz;        // one window row
    constexpr unsigned kFull = 0xffffffffu;
    constexpr unsigned kGroupMask = (1u << G) - 1u;
    static_assert(kVoxelsPerWarp % G == 0, "lane shape");

    const int W = st.window_rows;
    const int window_bytes = W * kRowBytes;
    unsigned char* s_window = smem;                                                // [2][W][FC] of T
    StepParam* s_param = reinterpret_cast<StepParam*>(smem + 2 * window_bytes);  // [3][128]
    float* s_arr = reinterpret_cast<float*>(s_param + 3 * kTileVoxels);           // [n_pref][128]
    const int n_pref = a.n_tx <= kMaxPrefetchTx ? a.n_tx : 0;
    int* s_cand = reinterpret_cast<int*>(s_arr + n_pref * kTileVoxels);           // [kMaxElemBlock]
    int* s_lohi = s_cand + kMaxElemBlock;  // [3][4][2] per-parameter-warp window partials
    unsigned* s_valid = reinterpret_cast<unsigned*>(s_lohi + 3 * 4 * 2);  // [3][4] validity ballots
    int* s_lo = reinterpret_cast<int*>(s_valid + 3 * 4);                 // [3] window start per step
    int* s_mode = s_lo + 3;                                               // [3] 0 empty, 1 TMA, 2 direct
    int* s_count = s_mode + 3;                                            // [kStagedWarps] compaction
    float* s_bbox = reinterpret_cast<float*>(s_count + kStagedWarps);     // [kStagedWarps][5]
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(s_bbox + kStagedWarps * 5) + 7) & ~uintptr_t{7});  // [2]

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = lane / LV;
    const int sub = lane - g * LV;
    const int frame0 = chunk * FC + sub * VF;
    const bool frames_ok = frame0 < a.n_frames;
    const T* const channel = static_cast<const T*>(a.channel);
    const int64_t n_frames = a.n_frames;
    const int64_t row_len = static_cast<int64_t>(a.n_samples);

    // ---- the parameter thread's voxel (threads 0..127)
    const bool is_param = tid < kTileVoxels;
    const int64_t pv = is_param ? tile_voxel(a, st, tile, tid) : -1;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (pv >= 0) {
        vx = __ldg(a.scan + 3 * pv + 0);
        vy = __ldg(a.scan + 3 * pv + 1);
        vz = __ldg(a.scan + 3 * pv + 2);
    }
    const float radius = __fdiv_rn(vz, a.two_f_number);  // kernel.cu:583
    const float radius_sq = __fmul_rn(radius, radius);

    // ---- stage the tile's transmit arrivals; tile bounding box for the candidate test
    for (int i = tid; i < n_pref * kTileVoxels; i += kStagedThreads) {
        const int t = i / kTileVoxels;
        const int64_t vv = tile_voxel(a, st, tile, i - t * kTileVoxels);
        s_arr[i] = vv >= 0 ? __ldg(a.arrivals + static_cast<int64_t>(t) * a.n_vox + vv) : 0.f;
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
            for (int k = 0; k < 5; ++k) s_bbox[warp * 5 + k] = b[k];
        }
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY, rmax = 0.f;
#pragma unroll
    for (int w = 0; w < kStagedWarps; ++w) {
        bx0 = fminf(bx0, s_bbox[w * 5 + 0]);
        bx1 = fmaxf(bx1, -s_bbox[w * 5 + 1]);
        by0 = fminf(by0, s_bbox[w * 5 + 2]);
        by1 = fmaxf(by1, -s_bbox[w * 5 + 3]);
        rmax = fmaxf(rmax, -s_bbox[w * 5 + 4]);
    }
    const float cand_r2 = rmax * rmax * 1.00001f + 1e-30f;

    float2 acc[ROUNDS][NP];
#pragma unroll
    for (int r = 0; r < ROUNDS; ++r)
#pragma unroll
        for (int q = 0; q < NP; ++q) acc[r][q] = make_float2(0.f, 0.f);

    uint32_t phase[2] = {0u, 0u};
    bool timed_out = false;

    // Parameter-thread state: receive path of (pv, current element).
    int rx_elem = -1;
    float dist = 0.f, weight_scaled = 0.f;
    bool pair_ok = false;
    SplitPos rx_pos{};
    float rx_cyc = 0.f;

    for (int eb = 0; eb < a.n_rx; eb += kMaxElemBlock) {
        // ---- candidate elements of this block (compacted, in element order)
        bool cand = false;
        const int e_test = eb + tid;
        if (tid < kMaxElemBlock && e_test < a.n_rx) {
            const float ex = __ldg(a.rx + 3 * e_test + 0);
            const float ey = __ldg(a.rx + 3 * e_test + 1);
            const float ddx = fmaxf(fmaxf(bx0 - ex, ex - bx1), 0.f);
            const float ddy = fmaxf(fmaxf(by0 - ey, ey - by1), 0.f);
            cand = ddx * ddx + ddy * ddy <= cand_r2;
        }
        const unsigned m = __ballot_sync(kFull, cand);
        __syncthreads();  // the previous block's s_cand is fully consumed
        if (lane == 0) s_count[warp] = __popc(m);
        __syncthreads();
        int base = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kStagedWarps; ++w) {
            const int c = s_count[w];
            base += w < warp ? c : 0;
            total += c;
        }
        if (cand) s_cand[base + __popc(m & ((1u << lane) - 1u))] = e_test;
        __syncthreads();
        if (total == 0) continue;
        const int n_steps = total * a.n_tx;

        // ---- parameters of step k into slot k % 3 (parameter threads), window partials, ballots
        auto make_params = [&](int k) {
            if (!is_param) return;
            const int ci = k / a.n_tx;
            const int t = k - ci * a.n_tx;
            const int e = s_cand[ci];
            const int slot = k % 3;
            if (e != rx_elem) {
                rx_elem = e;
                const float ex = __ldg(a.rx + 3 * e + 0), ey = __ldg(a.rx + 3 * e + 1), ez = __ldg(a.rx + 3 * e + 2);
                const float dx = __fsub_rn(ex, vx);
                const float dy = __fsub_rn(ey, vy);
                const float dz = __fsub_rn(ez, vz);
                const float h2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                if (a.split) {
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
            StepParam p{-1, 0.f, 0.f, 0.f};
            int lo = 0x7fffffff, hi = -1;
            bool ok = false;
            if (pair_ok) {
                const float txa = n_pref ? s_arr[t * kTileVoxels + tid]
                                         : __ldg(a.arrivals + static_cast<int64_t>(t) * a.n_vox + pv);
                TapPosition tp{};
                float sn = 0.f, cs = 1.f;
                if (a.split) {
                    const SplitPos tx_pos = split_position((static_cast<double>(txa) - a.t0_d) * a.fs_d);
                    int sbase = tx_pos.base + rx_pos.base;
                    float frac = __fadd_rn(tx_pos.frac, rx_pos.frac);
                    if (frac >= 1.0f) {
                        frac = __fsub_rn(frac, 1.0f);
                        sbase += 1;
                    }
                    ok = !(sbase < a.start_base || (sbase == a.start_base && frac < a.start_frac));
                    ok = ok && split_tap_position<INTERP>(sbase, frac, a.n_samples, tp);
                    if (INTERP == kQuadratic && ok) tp.w0 = __fsub_rn(frac, static_cast<float>(tp.idx - sbase));
                    if (ok && kCplx && a.rotate) {
                        split_phasor(__fadd_rn(reduced_cycles(static_cast<double>(txa) * a.fmod_d), rx_cyc), sn, cs);
                    }
                } else {
                    const float tau = __fmaf_rn(dist, a.inv_c, txa);
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
                    if constexpr (INTERP == kQuadratic) tp.w0 = __fsub_rn(s, static_cast<float>(tp.idx));
                    if (ok && kCplx && a.rotate) {
                        __sincosf(__fmul_rn(a.mod_rad, tau), &sn, &cs);  // kernel.cu:656-658
                    }
                }
                if (ok) {
                    p.row = tp.idx;
                    p.w = tp.w0;  // linear: t; quadratic: x (weights rebuilt in the gather)
                    p.cw = weight_scaled;
                    if (kCplx && a.rotate) {
                        p.cw = __fmul_rn(cs, weight_scaled);
                        p.sw = __fmul_rn(sn, weight_scaled);
                    }
                    lo = INTERP == kQuadratic ? tp.idx - 1 : tp.idx;
                    hi = INTERP == kQuadratic ? tp.idx + 1 : (INTERP == kLinear ? tp.idx + tp.step : tp.idx);
                }
            }
            s_param[slot * kTileVoxels + tid] = p;
            const unsigned vmask = __ballot_sync(kFull, ok);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                lo = min(lo, __shfl_xor_sync(kFull, lo, off));
                hi = max(hi, __shfl_xor_sync(kFull, hi, off));
            }
            if (lane == 0) {
                s_lohi[(slot * 4 + warp) * 2 + 0] = lo;
                s_lohi[(slot * 4 + warp) * 2 + 1] = hi;
                s_valid[slot * 4 + warp] = vmask;
            }
        };
        // ---- after the barrier: decide how step k reads its taps, and start its window copy
        auto start_window = [&](int k) {
            if (tid != 0) return;
            const int slot = k % 3;
            int lo = 0x7fffffff, hi = -1;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                lo = min(lo, s_lohi[(slot * 4 + w) * 2 + 0]);
                hi = max(hi, s_lohi[(slot * 4 + w) * 2 + 1]);
            }
            int mode = 0;
            if (hi >= lo) mode = (st.use_tma && hi - lo + 1 <= W) ? 1 : 2;
            s_lo[slot] = lo;
            s_mode[slot] = mode;
            if (mode == 1) {
                const int ci = k / a.n_tx;
                const int t = k - ci * a.n_tx;
                const int e = s_cand[ci];
                const int b = k & 1;
                const int row0 = (t * a.n_rx + e) * a.n_samples + lo;
                mbar_expect_tx(&s_bar[b], static_cast<uint32_t>(window_bytes));
                tma_load_2d(s_window + b * window_bytes, tmap, chunk * FC, row0, &s_bar[b]);
            }
        };

        make_params(0);
        __syncthreads();
        start_window(0);
        for (int k = 0; k < n_steps; ++k) {
            if (k + 1 < n_steps) make_params(k + 1);
            __syncthreads();
            if (k + 1 < n_steps) start_window(k + 1);

            const int slot = k % 3;
            const int mode = s_mode[slot];
            if (mode == 0) continue;
            const int b = k & 1;
            if (mode == 1) {
                // After a timeout a thread stops waiting and computing but keeps taking every
                // barrier, so the CTA never diverges on __syncthreads.
                if (!timed_out && !mbar_wait(&s_bar[b], phase[b])) timed_out = true;
                phase[b] ^= 1u;
            }
            if (timed_out || !frames_ok) continue;
            // This warp's 16 voxels are bits [16 (warp & 1), +16) of parameter warp warp / 2.
            const unsigned wmask = (s_valid[slot * 4 + (warp >> 1)] >> ((warp & 1) * 16)) & 0xffffu;
            if (wmask == 0u) continue;
            const int ci = k / a.n_tx;
            const int t = k - ci * a.n_tx;
            const int e = s_cand[ci];
            const int lo = s_lo[slot];
            const unsigned char* win = s_window + b * window_bytes + sub * VF * kEsz;
            const T* grow = channel + static_cast<int64_t>(t * a.n_rx + e) * row_len * n_frames + frame0;
            const StepParam* prm = s_param + slot * kTileVoxels + warp * kVoxelsPerWarp + g;
#pragma unroll
            for (int r = 0; r < ROUNDS; ++r) {
                if (((wmask >> (r * G)) & kGroupMask) == 0u) continue;  // no voxel of this round is valid
                if (!((wmask >> (r * G + g)) & 1u)) continue;
                const StepParam p = prm[r * G];
                uint2 ta, tb, tc;
                if (mode == 1) {
                    const unsigned char* q = win + (p.row - lo) * kRowBytes;
                    if constexpr (INTERP == kNearest) {
                        ta = *reinterpret_cast<const uint2*>(q);
                    } else if constexpr (INTERP == kLinear) {
                        ta = *reinterpret_cast<const uint2*>(q);
                        tb = *reinterpret_cast<const uint2*>(q + (p.w > 0.0f ? kRowBytes : 0));
                    } else {
                        ta = *reinterpret_cast<const uint2*>(q - kRowBytes);
                        tb = *reinterpret_cast<const uint2*>(q);
                        tc = *reinterpret_cast<const uint2*>(q + kRowBytes);
                    }
                } else {
                    const T* q = grow + static_cast<int64_t>(p.row) * n_frames;
                    if constexpr (INTERP == kNearest) {
                        ta = __ldg(reinterpret_cast<const uint2*>(q));
                    } else if constexpr (INTERP == kLinear) {
                        ta = __ldg(reinterpret_cast<const uint2*>(q));
                        tb = __ldg(reinterpret_cast<const uint2*>(q + (p.w > 0.0f ? n_frames : 0)));
                    } else {
                        ta = __ldg(reinterpret_cast<const uint2*>(q - n_frames));
                        tb = __ldg(reinterpret_cast<const uint2*>(q));
                        tc = __ldg(reinterpret_cast<const uint2*>(q + n_frames));
                    }
                }
                float2 va[NP], vb[NP], vc[NP];
                Vec8<S>::unpack(ta, va);
                if constexpr (INTERP != kNearest) Vec8<S>::unpack(tb, vb);
                if constexpr (INTERP == kQuadratic) Vec8<S>::unpack(tc, vc);
                float wm = 0.f, w0 = 0.f, wp = 0.f;
                if constexpr (INTERP == kQuadratic) {
                    const float hx = __fmul_rn(0.5f, p.w);
                    const float qq = __fmul_rn(hx, p.w);
                    wm = __fsub_rn(qq, hx);
                    w0 = __fmaf_rn(-2.0f, qq, 1.0f);
                    wp = __fadd_rn(qq, hx);
                }
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    float2 v;
                    if constexpr (INTERP == kNearest) {
                        v = va[q];
                    } else if constexpr (INTERP == kLinear) {
                        if constexpr (kCplx) {
                            v.x = __fmaf_rn(p.w, __fsub_rn(vb[q].x, va[q].x), va[q].x);  // a + t (b - a)
                            v.y = __fmaf_rn(p.w, __fsub_rn(vb[q].y, va[q].y), va[q].y);
                        } else {
                            v = fma2(make_float2(p.w, p.w), sub2(vb[q], va[q]), va[q]);
                        }
                    } else {
                        if constexpr (kCplx) {
                            v.x = __fmaf_rn(wp, vc[q].x, __fmaf_rn(wm, va[q].x, __fmul_rn(w0, vb[q].x)));
                            v.y = __fmaf_rn(wp, vc[q].y, __fmaf_rn(wm, va[q].y, __fmul_rn(w0, vb[q].y)));
                        } else {
                            v = fma2(make_float2(wp, wp), vc[q],
                                     fma2(make_float2(wm, wm), va[q], mul2(make_float2(w0, w0), vb[q])));
                        }
                    }
                    if constexpr (kCplx) {
                        acc[r][q].x = __fmaf_rn(v.x, p.cw, __fmaf_rn(-v.y, p.sw, acc[r][q].x));
                        acc[r][q].y = __fmaf_rn(v.y, p.cw, __fmaf_rn(v.x, p.sw, acc[r][q].y));
                    } else {
                        acc[r][q] = fma2(v, make_float2(p.cw, p.cw), acc[r][q]);
                    }
                }
            }
        }
    }

    if (__syncthreads_or(timed_out)) {
        // Give the last copy on each buffer a bounded chance to land before the CTA exits,
        // record the failure and leave this tile's output untouched.
        mbar_wait(&s_bar[0], phase[0] ^ 1u);
        mbar_wait(&s_bar[1], phase[1] ^ 1u);
        if (tid == 0) atomicOr(st.status, 1);
        return false;
    }
    // No copy is in flight: retire the barriers so the next tile of a persistent CTA can
    // initialise them again.
    if (tid == 0) {
        mbar_inval(&s_bar[0]);
        mbar_inval(&s_bar[1]);
    }

    // ---- write the tile's sums: lane (g, sub) holds frames frame0 .. frame0 + VF - 1
    if (!frames_ok) return true;
#pragma unroll
    for (int r = 0; r < ROUNDS; ++r) {
        const int64_t v = tile_voxel(a, st, tile, warp * kVoxelsPerWarp + r * G + g);
        if (v < 0) continue;
        if constexpr (kCplx) {
            float2* o = static_cast<float2*>(a.out) + v * n_frames + frame0;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                float2 res = acc[r][q];
                if (a.accumulate) {
                    const float2 prev = o[q];
                    res.x = __fadd_rn(prev.x, res.x);
                    res.y = __fadd_rn(prev.y, res.y);
                }
                o[q] = res;
            }
        } else {
            float* o = static_cast<float*>(a.out) + v * n_frames + frame0;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                float2 res = acc[r][q];
                if (a.accumulate) {
                    res.x = __fadd_rn(o[2 * q], res.x);
                    res.y = __fadd_rn(o[2 * q + 1], res.y);
                }
                o[2 * q] = res.x;
                o[2 * q + 1] = res.y;
            }
        }
    }
    return true;
}

template <int S, int INTERP, int LV>
__global__ void __launch_bounds__(kStagedThreads, 3)
    das_staged_kernel(const __grid_constant__ DasArgs a, const __grid_constant__ StagedArgs st,
                      const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(128) unsigned char smem[];
    staged_tile<S, INTERP, LV>(a, st, &tmap, blockIdx.x, blockIdx.y, smem);
}

// Shared memory needed by one CTA.
inline size_t staged_smem_bytes(int window_rows, int frame_chunk, int esz, int n_tx) {
    const size_t window = static_cast<size_t>(window_rows) * frame_chunk * esz;
    const size_t pref = n_tx <= kMaxPrefetchTx ? static_cast<size_t>(n_tx) * kTileVoxels * sizeof(float) : 0;
    return 2 * window + 3 * kTileVoxels * sizeof(StepParam) + pref + kMaxElemBlock * sizeof(int) +
           (3 * 4 * 2 + 3 * 4 + 3 + 3 + kStagedWarps) * sizeof(int) + kStagedWarps * 5 * sizeof(float) + 8 +
           2 * sizeof(uint64_t);
}

}  // namespace mach_b200
