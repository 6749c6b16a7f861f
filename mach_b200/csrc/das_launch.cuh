// Kernel selection and launch for one storage type.
#pragma once

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
};

struct LaunchPlan {
    int kind;
    int lanes_per_voxel;  // staged kernel: 4, 8, 16 or 32
    int passes;       // frames per lane (multi-frame kernels)
    int tx_chunk;     // arrivals staged per pass (lane-voxel kernels)
    dim3 grid;
    dim3 block;
    size_t smem;
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

template <int S, int I>
cudaError_t launch_staged_lv(const DasArgs& a, const StagedArgs& st, const CUtensorMap& map, const LaunchPlan& p,
                             cudaStream_t stream) {
    switch (p.lanes_per_voxel) {
        case 4: return launch_staged<S, I, 4>(a, st, map, p, stream);
        case 8: return launch_staged<S, I, 8>(a, st, map, p, stream);
        case 16: return launch_staged<S, I, 16>(a, st, map, p, stream);
        default: return launch_staged<S, I, 32>(a, st, map, p, stream);
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
#define MACH_B200_LV(I, NF) das_lane_voxel_kernel<S, I, NF><<<p.grid, p.block, p.smem, stream>>>(a)
#define MACH_B200_WG(I, L, P) das_gather_kernel<S, I, L, P><<<p.grid, p.block, 0, stream>>>(a)
#define MACH_B200_KINDS(I)                                   \
    switch (p.kind) {                                        \
        case kKindLaneVoxel1: MACH_B200_LV(I, 1); break;     \
        case kKindLaneVoxelN: MACH_B200_LV(I, 0); break;     \
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
#undef MACH_B200_LV
    return cudaGetLastError();
}

}  // namespace mach_b200
