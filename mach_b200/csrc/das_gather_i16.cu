// Gather kernels for i16 channel-data storage (one translation unit per storage type
// so the library compiles in parallel).
#include "das_gather.cuh"

namespace mach_b200 {
template cudaError_t launch_das_gather<kI16>(const DasArgs&, int, int, dim3, cudaStream_t);
}  // namespace mach_b200
