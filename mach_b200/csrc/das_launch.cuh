// Kernel selection and launch for one storage type.
#pragma once

#include <algorithm>

#include "das_batch.cuh"
#include "das_ensemble.cuh"
#include "das_frame_lane.cuh"
#include "das_gather.cuh"
#include "das_lane_voxel.cuh"
#include "das_staged.cuh"

namespace mach_b200 {

enum KernelKind : int {
    kKindLaneVoxel1 = 0,   // das_lane_voxel_kernel, exactly one frame
    kKindLaneVoxelN = 1,   // das_lane_voxel_kernel, 2..8 frames per lane
    kKindWarpHalf = 2,     // das_gather_kernel, 16 lanes per voxel
    kKindWarp = 3,         // das_gather_kernel, 32 lanes per voxel
    kKindStaged = 4,       // das_staged_kernel, windows staged in shared memory (TMA or direct)
    kKindLaneVoxel16 = 5,  // das_lane_voxel_kernel, exactly 16 frames loaded as 16-byte vectors
    kKindEnsemble = 6,     // das_ensemble_kernel, windows in tensor memory, lanes = frames
    kKindLaneVoxel8 = 7,   // das_lane_voxel_kernel, chunks of 8 frames (grid.y) of a longer ensemble
    kKindFrameLane = 8,    // das_frame_lane_kernel, lanes = frames, rows reused along voxel runs
};

struct LaunchPlan {
    int kind;
    int lanes_per_voxel;  // staged kernel: 4, 8, 16 or 32; one-frame lane-voxel kernel: 1, 2 or 4 lanes per voxel
    int passes;       // frames per lane (multi-frame kernels)
    int tx_chunk;     // arrivals staged per pass (lane-voxel kernels)
    dim3 grid;
    dim3 block;
    size_t smem;
    int map_fast;       // lane-voxel kernels: grid tiling (DasArgs::map_*), 0 = linear tiles
    int map_wlog;
    int64_t map_outer;
    int tile_rev;       // lane-voxel kernels on a grid: far end of the contiguous axis first (DasArgs::tile_rev)
    int frame_chunks;   // lane-voxel 8-frame chunks per tile (DasArgs::frame_chunks)
    int element_block;  // lane-voxel kernels: elements per launch (0 = all), so that one launch's
                        // channel data stays resident in L2
    int frame_slots;    // frame-lane kernel: J, lane-word columns per warp (1, 2 or 4)
    int run_voxels;     // frame-lane kernel: G, voxels per warp run (J * G = 16)
};

// Opt a kernel into more than 48 KB of dynamic shared memory (once per instance is enough,
// repeating it is harmless).
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <int S, int I, int LV>
cudaError_t launch_staged(const DasArgs& a, const StagedArgs& st, const CUtensorMap& map, const LaunchPlan& p,
                          cudaStream_t stream) {
    const cudaError_t e = allow_smem(das_staged_kernel<S, I, LV>, p.smem);
    if (e != cudaSuccess) return e;
    das_staged_kernel<S, I, LV><<<p.grid, p.block, p.smem, stream>>>(a, st, map);
    return cudaGetLastError();
}

// Storage types with two float2 pairs per 8-byte lane vector stop at 16 lanes per voxel
// (32 would need 64 accumulator registers per thread); the planner never asks for more.
template <int S>
constexpr int max_lanes_per_voxel() {
    return Vec8<S>::kPairs == 2 ? 16 : 32;
}

template <int S, int I>
cudaError_t launch_staged_lv(const DasArgs& a, const StagedArgs& st, const CUtensorMap& map, const LaunchPlan& p,
                             cudaStream_t stream) {
    switch (p.lanes_per_voxel) {
        case 4: return launch_staged<S, I, 4>(a, st, map, p, stream);
        case 8: return launch_staged<S, I, 8>(a, st, map, p, stream);
        case 16: return launch_staged<S, I, 16>(a, st, map, p, stream);
        default: return launch_staged<S, I, max_lanes_per_voxel<S>()>(a, st, map, p, stream);
    }
}

template <int S>
cudaError_t launch_das_staged(const DasArgs& a, const StagedArgs& st, const CUtensorMap& map, int interp,
                              const LaunchPlan& p, cudaStream_t stream) {
    switch (interp) {
        case kNearest: return launch_staged_lv<S, kNearest>(a, st, map, p, stream);
        case kLinear: return launch_staged_lv<S, kLinear>(a, st, map, p, stream);
        default: return launch_staged_lv<S, kQuadratic>(a, st, map, p, stream);
    }
}

template <int S>
cudaError_t launch_das(const DasArgs& a, int interp, const LaunchPlan& p, cudaStream_t stream) {
#define MACH_B200_LV(I, NF)                                                                   \
    do {                                                                                      \
        if (a.split) das_lane_voxel_kernel<S, I, NF, true><<<p.grid, p.block, p.smem, stream>>>(a);  \
        else das_lane_voxel_kernel<S, I, NF, false><<<p.grid, p.block, p.smem, stream>>>(a);         \
    } while (0)
#define MACH_B200_LV_CS(I, CS)                                                                           \
    do {                                                                                                 \
        if (a.split) das_lane_voxel_kernel<S, I, 1, true, CS><<<p.grid, p.block, p.smem, stream>>>(a);   \
        else das_lane_voxel_kernel<S, I, 1, false, CS><<<p.grid, p.block, p.smem, stream>>>(a);          \
    } while (0)
#define MACH_B200_WG(I, L, P) das_gather_kernel<S, I, L, P><<<p.grid, p.block, 0, stream>>>(a)
#define MACH_B200_KINDS(I)                                   \
    switch (p.kind) {                                        \
        case kKindLaneVoxel1:                                \
            if (p.lanes_per_voxel == 4) MACH_B200_LV_CS(I, 4); \
            else if (p.lanes_per_voxel == 2) MACH_B200_LV_CS(I, 2); \
            else MACH_B200_LV(I, 1);                         \
            break;                                           \
        case kKindLaneVoxelN: MACH_B200_LV(I, 0); break;     \
        case kKindLaneVoxel16: MACH_B200_LV(I, 16); break;   \
        case kKindLaneVoxel8: MACH_B200_LV(I, 8); break;     \
        case kKindWarpHalf: MACH_B200_WG(I, 16, 4); break;   \
        default: MACH_B200_WG(I, 32, 8); break;              \
    }
    switch (interp) {
        case kNearest: MACH_B200_KINDS(kNearest); break;
        case kLinear: MACH_B200_KINDS(kLinear); break;
        default: MACH_B200_KINDS(kQuadratic); break;
    }
#undef MACH_B200_KINDS
#undef MACH_B200_WG
#undef MACH_B200_LV_CS
#undef MACH_B200_LV
    return cudaGetLastError();
}

// Frame-lane kernel: (J, G) pairs with J * G = 16 (64 accumulator registers for complex storage).
template <int S, int I, int J, bool SPLIT>
cudaError_t launch_frame_lane_k(const DasArgs& a, const FrameLaneArgs& fl, const LaunchPlan& p, cudaStream_t stream) {
    das_frame_lane_kernel<S, I, J, 16 / J, SPLIT><<<p.grid, p.block, p.smem, stream>>>(a, fl);
    return cudaGetLastError();
}

template <int S, int I, bool SPLIT>
cudaError_t launch_frame_lane_i(const DasArgs& a, const FrameLaneArgs& fl, const LaunchPlan& p, cudaStream_t stream) {
    switch (p.frame_slots) {
        case 1: return launch_frame_lane_k<S, I, 1, SPLIT>(a, fl, p, stream);
        case 2: return launch_frame_lane_k<S, I, 2, SPLIT>(a, fl, p, stream);
        default: return launch_frame_lane_k<S, I, 4, SPLIT>(a, fl, p, stream);
    }
}

template <int S>
cudaError_t launch_das_frame_lane(const DasArgs& a, const FrameLaneArgs& fl, int interp, const LaunchPlan& p,
                                  cudaStream_t stream) {
    if (interp == kNearest) {
        return a.split ? launch_frame_lane_i<S, kNearest, true>(a, fl, p, stream)
                       : launch_frame_lane_i<S, kNearest, false>(a, fl, p, stream);
    }
    return a.split ? launch_frame_lane_i<S, kLinear, true>(a, fl, p, stream)
                   : launch_frame_lane_i<S, kLinear, false>(a, fl, p, stream);
}

// ---------------------------------------------------------------- persistent batch launches

struct PersistentLaunch {
    const BatchHeader* hdr;
    const BatchJob* jobs;
    const int64_t* item_begin;
    unsigned long long* counter;
    size_t smem;
    int max_items;  // grid is min(max_items, resident CTAs)
};

template <typename K>
cudaError_t launch_persistent(K kernel, int threads, const PersistentLaunch& pl, cudaStream_t stream) {
    cudaError_t e = allow_smem(kernel, pl.smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&device)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, pl.smem)) != cudaSuccess) return e;
    const int grid = std::max(1, std::min(pl.max_items, std::max(1, per_sm) * sms));
    kernel<<<grid, threads, pl.smem, stream>>>(pl.hdr, pl.jobs, pl.item_begin, pl.counter);
    return cudaGetLastError();
}

// Lane-voxel family: frame class 1 (one frame), 12 / 14 (one frame, 2 / 4 lanes per voxel),
// 0 (2..8 frames), 16 (sixteen, vectorised), 8 (chunks of 8 frames of a longer ensemble).
template <int S>
cudaError_t launch_lane_voxel_persistent(int interp, int frame_class, bool split, const PersistentLaunch& pl,
                                         cudaStream_t stream) {
#define MACH_B200_PLV(I, NF, CS)                                                                              \
    return split ? launch_persistent(das_lane_voxel_persistent<S, I, NF, true, CS>, kLaneVoxelThreads, pl, stream) \
                 : launch_persistent(das_lane_voxel_persistent<S, I, NF, false, CS>, kLaneVoxelThreads, pl, stream)
#define MACH_B200_PLV_NF(I)                         \
    switch (frame_class) {                          \
        case 1: MACH_B200_PLV(I, 1, 1);             \
        case 12: MACH_B200_PLV(I, 1, 2);            \
        case 14: MACH_B200_PLV(I, 1, 4);            \
        case 16: MACH_B200_PLV(I, 16, 1);           \
        case 8: MACH_B200_PLV(I, 8, 1);             \
        default: MACH_B200_PLV(I, 0, 1);            \
    }
    switch (interp) {
        case kNearest: MACH_B200_PLV_NF(kNearest)
        case kLinear: MACH_B200_PLV_NF(kLinear)
        default: MACH_B200_PLV_NF(kQuadratic)
    }
#undef MACH_B200_PLV_NF
#undef MACH_B200_PLV
}

// Frame-lane family: variant = J (1, 2, 4).
template <int S>
cudaError_t launch_frame_lane_persistent(int interp, int variant, bool split, const PersistentLaunch& pl,
                                         cudaStream_t stream) {
#define MACH_B200_PFL(I, J)                                                                                    \
    return split ? launch_persistent(das_frame_lane_persistent<S, I, J, true>, kFrameLaneThreads, pl, stream) \
                 : launch_persistent(das_frame_lane_persistent<S, I, J, false>, kFrameLaneThreads, pl, stream)
#define MACH_B200_PFL_V(I)           \
    switch (variant) {               \
        case 1: MACH_B200_PFL(I, 1); \
        case 2: MACH_B200_PFL(I, 2); \
        default: MACH_B200_PFL(I, 4); \
    }
    if (interp == kNearest) {
        MACH_B200_PFL_V(kNearest)
    }
    MACH_B200_PFL_V(kLinear)
#undef MACH_B200_PFL_V
#undef MACH_B200_PFL
}

template <int S>
cudaError_t launch_staged_persistent(int interp, int lanes, const PersistentLaunch& pl, cudaStream_t stream) {
#define MACH_B200_PST(I, LV) return launch_persistent(das_staged_persistent<S, I, LV>, kStagedThreads, pl, stream)
#define MACH_B200_PST_LV(I)                                    \
    switch (lanes) {                                           \
        case 4: MACH_B200_PST(I, 4);                           \
        case 8: MACH_B200_PST(I, 8);                           \
        case 16: MACH_B200_PST(I, 16);                         \
        default: MACH_B200_PST(I, max_lanes_per_voxel<S>());   \
    }
    switch (interp) {
        case kNearest: MACH_B200_PST_LV(kNearest)
        case kLinear: MACH_B200_PST_LV(kLinear)
        default: MACH_B200_PST_LV(kQuadratic)
    }
#undef MACH_B200_PST_LV
#undef MACH_B200_PST
}

// Channel-data ingest (das_ingest.cu): (n_s, n_e, n_w, n_frames) -> (n_w, n_e, n_s, n_frames),
// converted from storage `src_code` to `dst_code` (both real or both complex), times `scale`.
cudaError_t launch_ingest(int src_code, const void* src, int dst_code, void* dst, int n_s, int n_e, int n_w,
                          int n_frames, float scale, cudaStream_t st);

// Analytic signal along the sample axis (das_hilbert.cu).  Column c of the real source splits
// into (c2, c1, c0) with c0 = c % n0, c1 = (c / n0) % n1, c2 = c / (n0 n1); its sample s sits at
// element sum(c_i * src_stride[i]) + s * src_sample, and its complex result at
// sum(c_i * dst_stride[i]) + s * dst_sample (in complex elements).
constexpr int kHilMaxStages = 32;
constexpr int kHilRoots = 256;  // shared-memory roots of the odd register radices (float2)
struct HilbertArgs {
    const void* src;
    void* dst;
    int n;                    // samples per column: the transform length
    int n_stages;             // Stockham stages; radix[s] of each
    int radix[kHilMaxStages];
    float inv_n;              // 1 / n
    float scale;              // both parts of the result are multiplied by it before rounding
    int64_t n_cols;
    int cols_log2;            // 1..4: a CTA takes 2^cols_log2 columns, transformed in pairs
    int pair_stride;          // float2 between the shared-memory buffers of two column pairs
    int x_in_smem;            // 1: the group's samples are kept in shared memory for the output
    int load_cols_fast;       // 1: consecutive threads read consecutive columns of one sample
    int store_cols_fast;      // 1: consecutive threads write consecutive columns of one sample
    int64_t n0, n1;
    int64_t src_stride[3];
    int64_t src_sample;
    int64_t dst_stride[3];
    int64_t dst_sample;
};

// Radices of the Stockham stages for length n (16, 8, 4, 2 first, then odd primes); -1 if
// more than max_stages.
int hilbert_plan(int n, int* radix, int max_stages);

// Real storage src_code (kF32/kF16/kBF16/kI16) to complex dst_code (kC64/kCF16/kCBF16/kCI16);
// `smem` = 8 (n + kHilRoots + 2^cols_log2 pair_stride) bytes (two buffers of pair_stride float2
// per column pair), plus 4 n 2^cols_log2 with x_in_smem.  A persistent grid of at most the
// resident CTAs.
cudaError_t launch_hilbert(int src_code, int dst_code, const HilbertArgs& g, size_t smem, cudaStream_t st);

// Transmit arrivals of a plane (model 1) or spherical (model 2) wave table (das_transmit.cu):
// out[t][v] for t < n_tx, v < n_scan; params [n_tx][8] FP64, scan [n_scan][3] FP32, all
// device memory.
cudaError_t launch_tx_arrivals(int model, const double* params, const float* scan, int64_t n_scan, int n_tx,
                               double sound_speed, float* out, cudaStream_t st);

// Power-Doppler epilogue (das_power.cu): out[v] (+)= sum over frames of |in[v][f]|^2.
cudaError_t launch_power_epilogue(const void* in, float* out, int64_t n_vox, int n_frames, bool cplx, bool accumulate,
                                  cudaStream_t stream);

// Ensemble kernel: persistent grid of at most one CTA per SM (its 512 threads use the whole
// register file), each CTA running four teams over the (tile, frame block) items.
template <int S, int I, bool SPLIT>
cudaError_t launch_ensemble(const DasArgs& a, const StagedArgs& st, const EnsembleArgs& ea, const CUtensorMap& map,
                            size_t smem, cudaStream_t stream) {
    auto kernel = das_ensemble_kernel<S, I, SPLIT>;
    cudaError_t e = allow_smem(kernel, smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&device)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kEnsThreads, smem)) != cudaSuccess) return e;
    const int items = ea.n_tiles * ea.n_fblocks;
    const int grid = std::max(1, std::min((items + kEnsTeams - 1) / kEnsTeams, std::max(1, per_sm) * sms));
    kernel<<<grid, kEnsThreads, smem, stream>>>(a, st, ea, map);
    return cudaGetLastError();
}

template <int S>
cudaError_t launch_das_ensemble(const DasArgs& a, const StagedArgs& st, const EnsembleArgs& ea, const CUtensorMap& map,
                                int interp, size_t smem, cudaStream_t stream) {
    if (interp == kNearest) {
        return a.split ? launch_ensemble<S, kNearest, true>(a, st, ea, map, smem, stream)
                       : launch_ensemble<S, kNearest, false>(a, st, ea, map, smem, stream);
    }
    return a.split ? launch_ensemble<S, kLinear, true>(a, st, ea, map, smem, stream)
                   : launch_ensemble<S, kLinear, false>(a, st, ea, map, smem, stream);
}

}  // namespace mach_b200
