// Gather kernels for f32 channel-data storage (one translation unit per storage type
// so the library compiles in parallel).
#include "das_launch.cuh"

namespace mach_b200 {
template cudaError_t launch_das<kF32>(const DasArgs&, int, const LaunchPlan&, cudaStream_t);
template cudaError_t launch_das_staged<kF32>(const DasArgs&, const StagedArgs&, const CUtensorMap&, int,
                                             const LaunchPlan&, cudaStream_t);
template cudaError_t launch_lane_voxel_persistent<kF32>(int, int, bool, const PersistentLaunch&, cudaStream_t);
template cudaError_t launch_staged_persistent<kF32>(int, int, const PersistentLaunch&, cudaStream_t);
template cudaError_t launch_das_ensemble<kF32>(const DasArgs&, const StagedArgs&, const EnsembleArgs&,
                                               const CUtensorMap&, int, size_t, cudaStream_t);
template cudaError_t launch_das_frame_lane<kF32>(const DasArgs&, const FrameLaneArgs&, int, const LaunchPlan&,
                                                cudaStream_t);
template cudaError_t launch_frame_lane_persistent<kF32>(int, int, bool, const PersistentLaunch&, cudaStream_t);
}  // namespace mach_b200
