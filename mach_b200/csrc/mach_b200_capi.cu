// C ABI of mach_b200 (declared in include/mach_b200.h): argument checks, host-buffer
// staging, launch planning (kernel family, tiling, TMA descriptor) and dispatch.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <vector>

#include "das_launch.cuh"
#include "das_split.h"
#include "mach_b200.h"

#ifndef MACH_B200_NVCC_VERSION
#define MACH_B200_NVCC_VERSION "0.0.0"
#endif
#define MACH_B200_VERSION "0.2.0"

namespace mach_b200 {
// Instantiated once per storage type in das_gather_<storage>.cu.
#define MACH_B200_EXTERN(S)                                                                                  \
    extern template cudaError_t launch_das<S>(const DasArgs&, int, const LaunchPlan&, cudaStream_t);         \
    extern template cudaError_t launch_das_staged<S>(const DasArgs&, const StagedArgs&, const CUtensorMap&, \
                                                     int, const LaunchPlan&, cudaStream_t);                 \
    extern template cudaError_t launch_das_frame_lane<S>(const DasArgs&, const FrameLaneArgs&, int,         \
                                                         const LaunchPlan&, cudaStream_t);                   \
    extern template cudaError_t launch_das_ensemble<S>(const DasArgs&, const StagedArgs&,                  \
                                                       const EnsembleArgs&, const CUtensorMap&, int, size_t,  \
                                                       cudaStream_t);                                         \
    extern template cudaError_t launch_lane_voxel_persistent<S>(int, int, bool, const PersistentLaunch&,    \
                                                                cudaStream_t);                               \
    extern template cudaError_t launch_staged_persistent<S>(int, int, const PersistentLaunch&, cudaStream_t); \
    extern template cudaError_t launch_frame_lane_persistent<S>(int, int, bool, const PersistentLaunch&,    \
                                                                cudaStream_t);
MACH_B200_EXTERN(kF32)
MACH_B200_EXTERN(kC64)
MACH_B200_EXTERN(kF16)
MACH_B200_EXTERN(kCF16)
MACH_B200_EXTERN(kBF16)
MACH_B200_EXTERN(kCBF16)
MACH_B200_EXTERN(kI16)
MACH_B200_EXTERN(kCI16)
#undef MACH_B200_EXTERN
}  // namespace mach_b200

// Status word written by kernels whose bounded waits time out (one per device).
__device__ int g_mach_b200_status;

// Work-item counters of mach_b200_beamform_ensemble_noalloc: one per launch (a launch covers
// fewer than 2^31 channel samples), kNoAllocLaunches at most: 256 bytes held on every device
// that loads the library.  Every call shares them; each call zeroes the ones it uses.
constexpr int kNoAllocLaunches = 64;
static __device__ __align__(256) int g_noalloc_counters[kNoAllocLaunches];

namespace {

using namespace mach_b200;

thread_local std::string g_error;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define MACH_B200_CUDA_TRY(expr)                                                                \
    do {                                                                                        \
        cudaError_t err_ = (expr);                                                              \
        if (err_ != cudaSuccess) {                                                              \
            return fail(MACH_B200_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(err_)); \
        }                                                                                       \
    } while (0)

size_t storage_bytes(int storage) {
    switch (storage) {
        case kF32: return 4;
        case kC64: return 8;
        case kF16: case kBF16: case kI16: return 2;
        default: return 4;  // cf16, cbf16, ci16
    }
}

enum Residency { kOnDevice, kHostPinned, kHostPageable };

// Where does `p` live?  Device pointers must belong to `device`.
int residency(const void* p, int device, Residency* r, const char* name) {
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *r = kHostPageable;
        return MACH_B200_OK;
    }
    switch (attr.type) {
        case cudaMemoryTypeDevice:
        case cudaMemoryTypeManaged:
            if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
                return fail(MACH_B200_ERR_DEVICE, "%s is on CUDA device %d but the current device is %d", name,
                            attr.device, device);
            }
            *r = kOnDevice;
            return MACH_B200_OK;
        case cudaMemoryTypeHost:
            *r = kHostPinned;
            return MACH_B200_OK;
        default:
            *r = kHostPageable;
            return MACH_B200_OK;
    }
}

// ---------------------------------------------------------------- per-device state

constexpr int kMaxDevices = 64;

struct DeviceState {
    std::once_flag once;
    cudaError_t init_error = cudaSuccess;
    int* status = nullptr;  // device address of g_mach_b200_status
    std::once_flag pool_once;
    cudaError_t pool_error = cudaSuccess;
    std::atomic<cudaMemPool_t> pool{nullptr};  // the library's own stream-ordered pool for staging buffers
};
DeviceState g_devices[kMaxDevices];

// First call on a device (that device current): look up the status word.  Nothing else of the
// process's CUDA state is touched (its default memory pool keeps its settings).
int device_state(int device, DeviceState** out) {
    if (device < 0 || device >= kMaxDevices) return fail(MACH_B200_ERR_DEVICE, "device %d out of range", device);
    DeviceState& d = g_devices[device];
    std::call_once(d.once, [&d]() {
        void* p = nullptr;
        d.init_error = cudaGetSymbolAddress(&p, g_mach_b200_status);
        d.status = static_cast<int*>(p);
    });
    if (d.init_error != cudaSuccess) {
        return fail(MACH_B200_ERR_CUDA, "device setup failed: %s", cudaGetErrorString(d.init_error));
    }
    *out = &d;
    return MACH_B200_OK;
}

// Memory pool of the library's temporary device buffers on `device`, created on first use.
// It keeps up to kPoolKeepBytes of freed memory cached between calls (host-staged jobs
// allocate the same buffers call after call); beyond that, freed memory goes back to the
// driver at the next synchronisation.
constexpr uint64_t kPoolKeepBytes = uint64_t{2} << 30;

cudaError_t library_pool(int device, cudaMemPool_t* pool) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    DeviceState& d = g_devices[device];
    std::call_once(d.pool_once, [&d, device]() {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t created = nullptr;
        d.pool_error = cudaMemPoolCreate(&created, &props);
        if (d.pool_error == cudaSuccess) {
            uint64_t keep = kPoolKeepBytes;
            d.pool_error = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
            d.pool.store(created);
        }
    });
    *pool = d.pool.load();
    return d.pool_error;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        }
    });
    return fn;
}

// ---------------------------------------------------------------- launch planning

// Lane-voxel kernel: transmits whose arrivals a CTA stages at once (40 x 128 voxels x 4 B = 20 KB,
// nine CTAs per SM; split delays stage three words per entry, so 32).  A job of n_tx transmits
// runs in ceil(n_tx / cap) equal passes over its elements (75 transmits: 2 passes of 38 and 37;
// measured on B200, compounding 1.64 ms against 1.71 ms with 3 passes of 25).
constexpr int kMaxTxChunk = 40;
constexpr int kMaxTxChunkSplit = 32;

struct Plan {
    LaunchPlan lp{};
    StagedArgs st{};
    EnsembleArgs ea{};
    FrameLaneArgs fl{};
    bool staged = false;
    bool ensemble = false;
    bool frame_lane = false;
};

int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Tile extents for a voxel grid (fast axis first); the product is exactly 128.
void choose_tile(const mach_b200_options& o, StagedArgs& st) {
    const int slow = o.grid_shape[0], mid = o.grid_shape[1], fast = o.grid_shape[2];
    st.grid_fast = fast;
    st.grid_mid = mid;
    st.grid_slow = slow;
    if (mid <= 1) {  // 2-D grid: 8 along the contiguous axis x 16 across
        st.tile_fast = 8;
        st.tile_mid = 1;
        st.tile_slow = 16;
    } else {  // 3-D grid: 8 x 4 x 4
        st.tile_fast = 8;
        st.tile_mid = 4;
        st.tile_slow = 4;
    }
    st.tiles_fast = (fast + st.tile_fast - 1) / st.tile_fast;
    st.tiles_mid = (mid + st.tile_mid - 1) / st.tile_mid;
}

bool grid_matches(const mach_b200_options& o, uint64_t n_vox) {
    const int64_t a = o.grid_shape[0], b = o.grid_shape[1], c = o.grid_shape[2];
    return a > 0 && b > 0 && c > 0 && static_cast<uint64_t>(a * b * c) == n_vox;
}

// Ensemble kernel plan (lanes = frames, windows in tensor memory), or false when the job
// does not meet its conditions: nearest / linear taps, a TMA-able channel (16-byte aligned
// base, row pitch a multiple of 16 bytes), fewer than 2^31 voxels.
bool plan_ensemble(int storage, int interp, uint64_t n_vox, uint32_t n_frames, uint32_t n_tx, const void* channel,
                   bool channel_on_device, const mach_b200_options& o, Plan& p) {
    const int esz = static_cast<int>(storage_bytes(storage));
    const bool cplx = (storage & 1) != 0;
    if (interp != kNearest && interp != kLinear) return false;
    if (n_vox == 0 || n_vox > 0x7fffffffull || n_frames == 0) return false;
    if ((static_cast<uint64_t>(n_frames) * esz) % 16 != 0) return false;
    if (channel_on_device && reinterpret_cast<uintptr_t>(channel) % 16 != 0) return false;
    if (tensor_map_encoder() == nullptr) return false;
    const int lwb = (storage == kC64 || storage == kF32) ? 8 : 4;  // bytes of one lane word
    const int frames_per_lane = cplx ? 1 : 2;
    int w = o.window_rows > 0 ? o.window_rows : 48;
    w = std::min(kEnsMaxWindow, std::max(16, (w + 15) & ~15));
    EnsembleArgs& ea = p.ea;
    ea.window_rows = w;
    ea.n_fblocks = static_cast<int32_t>((n_frames + 32u * frames_per_lane - 1) / (32u * frames_per_lane));
    ea.box_x = 32 * lwb / esz;
    ea.tmem_cols = static_cast<uint32_t>(std::max(32, next_pow2(4 * w)));
    StagedArgs& st = p.st;
    if (grid_matches(o, n_vox)) {
        st.grid_slow = o.grid_shape[0];
        st.grid_mid = o.grid_shape[1];
        st.grid_fast = o.grid_shape[2];
        st.tile_fast = 4;  // along the contiguous axis (depth, for a scan ordered depth-fastest)
        st.tile_mid = st.grid_mid <= 1 ? 1 : 4;
        st.tile_slow = st.grid_mid <= 1 ? 32 : 8;
        st.tiles_fast = (st.grid_fast + st.tile_fast - 1) / st.tile_fast;
        st.tiles_mid = (st.grid_mid + st.tile_mid - 1) / st.tile_mid;
        const int64_t tiles = static_cast<int64_t>(st.tiles_fast) * st.tiles_mid *
                              ((st.grid_slow + st.tile_slow - 1) / st.tile_slow);
        ea.n_tiles = static_cast<int32_t>(tiles);
    } else {
        st.grid_fast = 0;
        ea.n_tiles = static_cast<int32_t>((n_vox + kEnsTileVoxels - 1) / kEnsTileVoxels);
    }
    if (static_cast<int64_t>(ea.n_tiles) * ea.n_fblocks > 0x7fffffffll) return false;
    const int n_pref = n_tx <= static_cast<uint32_t>(kEnsMaxPrefetchTx) ? static_cast<int>(n_tx) : 0;
    // Four teams' buffers must fit the 227 KB a CTA may use.
    while (w > 16 && kEnsTeams * ensemble_team_bytes(w, lwb, n_pref) > 227 * 1024) w -= 16;
    ea.window_rows = w;
    ea.tmem_cols = static_cast<uint32_t>(std::max(32, next_pow2(4 * w)));
    st.use_tma = 1;
    st.window_rows = w;
    ea.team_bytes = ensemble_team_bytes(w, lwb, n_pref);
    p.ensemble = true;
    p.staged = false;
    p.lp.kind = kKindEnsemble;
    p.lp.block = dim3(kEnsThreads, 1, 1);
    p.lp.grid = dim3(1, 1, 1);  // persistent; the launcher sizes it
    p.lp.passes = 1;
    p.lp.tx_chunk = 1;
    p.lp.lanes_per_voxel = 32;
    p.lp.smem = static_cast<size_t>(kEnsTeams) * ea.team_bytes;
    return true;
}

// Frame-lane kernel plan (lanes = frames, sample rows reused in registers along runs of
// neighbouring voxels), or false when the job does not meet its conditions: nearest / linear
// taps, an even frame count for real storage, lane words aligned, at least one full column of
// 32 lane words per sample row.  Runs lie along the mid axis of a 3-D grid and the slow axis of
// a 2-D one (the lateral axes, where delays change least from voxel to voxel); without a grid
// they are runs of consecutive voxels.
bool plan_frame_lane(int storage, int interp, uint64_t n_vox, uint32_t n_frames, const void* channel,
                     bool channel_on_device, const mach_b200_options& o, Plan& p) {
    const bool cplx = (storage & 1) != 0;
    const int word_bytes = (storage == kC64 || storage == kF32) ? 8 : 4;
    if (interp != kNearest && interp != kLinear) return false;
    if (n_vox == 0 || n_frames == 0 || (!cplx && n_frames % 2 != 0)) return false;
    if (channel_on_device && reinterpret_cast<uintptr_t>(channel) % word_bytes != 0) return false;
    const int64_t words = cplx ? n_frames : n_frames / 2;
    if (words < 32) return false;
    int J = o.frame_slots;
    if (J != 1 && J != 2 && J != 4) J = words <= 32 ? 1 : (words <= 64 ? 2 : 4);
    const int G = 16 / J;
    const int coef = cplx ? 2 : 1;
    FrameLaneArgs& fl = p.fl;
    if (grid_matches(o, n_vox)) {
        const int64_t slow = o.grid_shape[0], mid = o.grid_shape[1], fast = o.grid_shape[2];
        fl.n_fast = fast;
        fl.run_stride = fast;
        if (mid > 1) {
            fl.run_len = mid;
            fl.n_across = slow;
            fl.across_stride = mid * fast;
        } else {
            fl.run_len = slow;
            fl.n_across = 1;
            fl.across_stride = 0;
        }
    } else {
        fl.run_len = static_cast<int64_t>(n_vox);
        fl.run_stride = 1;
        fl.n_across = 1;
        fl.across_stride = 0;
        fl.n_fast = 1;
    }
    fl.runs_per_line = (fl.run_len + G - 1) / G;
    fl.n_runs = fl.runs_per_line * fl.n_across * fl.n_fast;
    fl.words = static_cast<int32_t>(words);
    fl.n_chunks = static_cast<int32_t>((words + 32 * J - 1) / (32 * J));
    const int64_t ctas = (fl.n_runs + kFrameLaneWarps - 1) / kFrameLaneWarps * fl.n_chunks;
    if (ctas > 0x7fffffffll) return false;
    p.frame_lane = true;
    p.lp.kind = kKindFrameLane;
    p.lp.frame_slots = J;
    p.lp.run_voxels = G;
    p.lp.block = dim3(kFrameLaneThreads, 1, 1);
    p.lp.grid = dim3(static_cast<unsigned>(ctas), 1, 1);
    p.lp.passes = 1;
    p.lp.tx_chunk = 1;
    p.lp.lanes_per_voxel = 32;
    p.lp.smem = static_cast<size_t>(kFrameLaneWarps) *
                (coef == 2 ? frame_lane_warp_bytes<2>() : frame_lane_warp_bytes<1>());
    return true;
}

// interp < 0: a caller that runs neither the frame-lane nor the ensemble kernel; batch: a
// persistent batch, which runs the frame-lane kernel but not the ensemble kernel.
Plan plan_launch(int storage, uint64_t n_vox, uint32_t n_frames, uint32_t n_tx, const void* channel,
                 bool channel_on_device, const mach_b200_options& o, int interp = -1, bool batch = false,
                 uint32_t n_rx = 0, uint32_t n_samples = 0) {
    Plan p;
    const int esz = static_cast<int>(storage_bytes(storage));
    const int vf = 8 / esz;
    int kind = o.kernel;
    // Longer ensembles in chunks of 8 frames (one CTA per chunk and tile) of the voxel-per-lane
    // kernel: rows of 8 frames must be 16-byte vectors and every sample row a multiple of 16
    // bytes.
    // (8-frame rows of 32 or more bytes are read with 256-bit loads: 32-byte aligned channel data)
    const uintptr_t align8 = (8u * esz) % 32u == 0 ? 32 : 16;
    const bool lane8_ok = n_frames > 16 && n_frames % 8 == 0 && (8u * esz) % 16u == 0 &&
                          (static_cast<uint64_t>(n_frames) * esz) % 16u == 0 &&
                          (!channel_on_device || reinterpret_cast<uintptr_t>(channel) % align8 == 0);
    // Measured on B200 (200-frame Doppler): for 4-byte complex storage (cf16, cbf16, ci16) the
    // 8-frame chunks beat the ensemble kernel (3.5 vs 5.5 ms); for complex64 and real storage
    // the ensemble kernel wins.
    // Measured on B200 (200-frame Doppler): the 8-frame chunks beat the ensemble kernel for
    // complex storage -- 3.3 vs 5.6 ms (cf16), 4.0 vs 4.8 ms (complex64, 256-bit row loads).
    if (kind == MACH_B200_KERNEL_AUTO && lane8_ok && (esz == 4 || esz == 8) && (storage & 1) &&
        grid_matches(o, n_vox)) {
        kind = MACH_B200_KERNEL_LANE_VOXEL;
    }
    // Frame-lane kernel: when asked for (measured on B200, the ensemble kernel and the 8-frame
    // chunks stay faster on the 200-frame Doppler job; the autotuner times all three).
    if (interp >= 0 && kind == MACH_B200_KERNEL_FRAME_LANE) {
        if (plan_frame_lane(storage, interp, n_vox, n_frames, channel, channel_on_device, o, p)) return p;
        p = Plan{};
    }
    if (kind == MACH_B200_KERNEL_FRAME_LANE) kind = MACH_B200_KERNEL_AUTO;
    // Ensemble kernel: asked for, or automatic for many frames on a known voxel grid.
    if (interp >= 0 && !batch) {
        const bool many = n_frames >= ((storage & 1) ? 32u : 64u);
        if (kind == MACH_B200_KERNEL_ENSEMBLE ||
            (kind == MACH_B200_KERNEL_AUTO && many && grid_matches(o, n_vox))) {
            if (plan_ensemble(storage, interp, n_vox, n_frames, n_tx, channel, channel_on_device, o, p)) return p;
            p = Plan{};
        }
    }
    if (kind == MACH_B200_KERNEL_ENSEMBLE) kind = MACH_B200_KERNEL_AUTO;
    // Host channel data is staged into fresh (aligned) device buffers.
    const bool vec_ok =
        n_frames % static_cast<uint32_t>(vf) == 0 && (!channel_on_device || reinterpret_cast<uintptr_t>(channel) % 8 == 0);
    // 16 frames per sample (32 bytes or more) as 256-bit vectors: 32-byte aligned rows.
    const bool lane16_ok = n_frames == 16 && (16u * esz) % 32u == 0 &&
                           (!channel_on_device || reinterpret_cast<uintptr_t>(channel) % 32 == 0);
    if (kind == MACH_B200_KERNEL_AUTO) {
        kind = (n_frames <= 8 || lane16_ok) ? MACH_B200_KERNEL_LANE_VOXEL
                                            : (vec_ok ? MACH_B200_KERNEL_STAGED : MACH_B200_KERNEL_WARP);
    }
    if (kind == MACH_B200_KERNEL_LANE_VOXEL && n_frames > 8 && !lane16_ok && !lane8_ok) kind = MACH_B200_KERNEL_WARP;
    if (kind == MACH_B200_KERNEL_STAGED && !vec_ok) kind = MACH_B200_KERNEL_WARP;

    if (kind == MACH_B200_KERNEL_LANE_VOXEL) {
        p.lp.kind = n_frames <= 1 ? kKindLaneVoxel1 : (n_frames == 16 ? kKindLaneVoxel16 : kKindLaneVoxelN);
        if (n_frames > 16) p.lp.kind = kKindLaneVoxel8;  // lane8_ok (checked above)
        p.lp.passes = static_cast<int>(n_frames);
        const int chunk = o.tx_chunk > 0 ? o.tx_chunk
                                         : ((o.flags & MACH_B200_FLAG_SPLIT_DELAY) ? kMaxTxChunkSplit : kMaxTxChunk);
        const uint32_t chunks = std::max<uint32_t>(1u, (n_tx + chunk - 1) / chunk);
        p.lp.tx_chunk = static_cast<int>(std::max<uint32_t>(1u, (n_tx + chunks - 1) / chunks));
        p.lp.block = dim3(kLaneVoxelThreads, 1, 1);
        // One-frame jobs split each voxel's elements over 2 or 4 lanes.  Measured on B200: 4
        // for jobs of fewer than 4 CTAs of 128 voxels per SM and for split delays, 2 otherwise.
        int cs = 1;
        if (n_frames <= 1) {
            if (o.lanes_per_voxel == 1 || o.lanes_per_voxel == 2 || o.lanes_per_voxel == 4) {
                cs = o.lanes_per_voxel;
            } else {
                const bool small = (n_vox + kLaneVoxelThreads - 1) / kLaneVoxelThreads < 4u * 148u;
                cs = small || (o.flags & MACH_B200_FLAG_SPLIT_DELAY) ? 4 : 2;
            }
        }
        p.lp.lanes_per_voxel = cs;
        const int vpc = kLaneVoxelThreads / cs;  // voxels per CTA
        p.lp.grid = dim3(static_cast<unsigned>((n_vox + vpc - 1) / vpc), 1, 1);
        // On a known grid: CTA tiles of wf x (128 / wf) voxels, warps of wf x (32 / wf).
        // Automatic: 2 along the contiguous axis for 16 frames (rows of 32+ bytes), else 4.
        const int wf = o.tile_fast == 1 || o.tile_fast == 2 || o.tile_fast == 4 || o.tile_fast == 8 ||
                               o.tile_fast == 16
                           ? o.tile_fast
                           : (n_frames >= 16 ? 2 : 4);
        if (grid_matches(o, n_vox) && o.grid_shape[2] >= wf) {
            const int lw = wf == 1 ? 0 : (wf == 2 ? 1 : (wf == 4 ? 2 : (wf == 8 ? 3 : 4)));
            p.lp.map_fast = o.grid_shape[2];
            p.lp.map_wlog = lw;
            // Heaviest tiles first (measured on B200: compounding 1.90 -> 1.72 ms, Doppler
            // complex64 4.06 -> 3.84 ms, FP16 2.75 -> 2.48 ms; 3-D 16 frames 67.3 -> 67.8 ms,
            // so 16-frame jobs keep the grid order).
            p.lp.tile_rev = o.tile_order == 1 ? 1 : (o.tile_order == 2 ? 0 : (n_frames == 16 ? 0 : 1));
            p.lp.map_outer = static_cast<int64_t>(n_vox / static_cast<uint64_t>(o.grid_shape[2]));
            const int64_t per_outer = vpc >> lw;
            const int64_t tiles = ((p.lp.map_outer + per_outer - 1) / per_outer) * ((p.lp.map_fast + wf - 1) / wf);
            p.lp.grid = dim3(static_cast<unsigned>(tiles), 1, 1);
        }
        if (p.lp.kind == kKindLaneVoxel8) {  // the 8-frame chunks of a tile run on consecutive CTAs
            p.lp.frame_chunks = static_cast<int>(n_frames / 8);
            p.lp.grid.x *= static_cast<unsigned>(p.lp.frame_chunks);
        }
        // Element blocks: one launch per block of elements whose channel data (all transmits)
        // fits in L2 with room to spare.  Automatic for 16-frame jobs above 126 MB of channel
        // data (3-D: every CTA sweeps every (transmit, element) row set, and CTAs that drift apart
        // evict each other's rows; measured DRAM reads were 70x the channel data in one launch).
        {
            const uint64_t per_elem = static_cast<uint64_t>(n_tx) * n_samples * n_frames * esz;
            int eb = o.element_block;
            if (eb == 0 && n_frames == 16 && per_elem > 0 &&
                per_elem * n_rx > (uint64_t{126} << 20) && !batch) {
                eb = static_cast<int>(std::max<uint64_t>(32, ((uint64_t{80} << 20) / per_elem) / 32 * 32));
            }
            p.lp.element_block = eb > 0 ? eb : 0;
        }
        // split mode stages three words per (transmit, voxel): base, fraction, phase cycles
        p.lp.smem = static_cast<size_t>(p.lp.tx_chunk) * kLaneVoxelThreads * sizeof(float) *
                    ((o.flags & MACH_B200_FLAG_SPLIT_DELAY) ? 3 : 1);
        return p;
    }
    if (kind == MACH_B200_KERNEL_STAGED) {
        const int lanes_needed = static_cast<int>((n_frames + vf - 1) / vf);
        int lv = o.lanes_per_voxel > 0 ? o.lanes_per_voxel : std::min(32, std::max(4, next_pow2(lanes_needed)));
        if (lv != 4 && lv != 8 && lv != 16 && lv != 32) lv = 32;
        // two float2 pairs per lane vector (16-bit real, any 16-bit or half complex): at most 16 lanes
        if (storage != kC64 && storage != kF32) lv = std::min(lv, 16);
        const int fc = lv * vf;
        int w = o.window_rows > 0 ? o.window_rows : (fc * esz >= 256 ? 64 : 128);
        w = std::min(256, std::max(4, (w + 3) & ~3));  // multiple of 4 keeps both windows 128-byte aligned
        p.staged = true;
        p.lp.kind = kKindStaged;
        p.lp.lanes_per_voxel = lv;
        p.lp.block = dim3(kStagedThreads, 1, 1);
        p.lp.tx_chunk = 1;
        p.lp.passes = 1;
        if (grid_matches(o, n_vox)) {
            choose_tile(o, p.st);
            const int64_t tiles = static_cast<int64_t>(p.st.tiles_fast) * p.st.tiles_mid *
                                  ((o.grid_shape[0] + p.st.tile_slow - 1) / p.st.tile_slow);
            p.lp.grid = dim3(static_cast<unsigned>(tiles), (n_frames + fc - 1) / fc, 1);
        } else {
            p.st.grid_fast = 0;
            p.lp.grid =
                dim3(static_cast<unsigned>((n_vox + kTileVoxels - 1) / kTileVoxels), (n_frames + fc - 1) / fc, 1);
        }
        p.st.window_rows = w;
        // TMA needs a 16-byte aligned base and a row pitch that is a multiple of 16 bytes.
        p.st.use_tma = ((!channel_on_device || reinterpret_cast<uintptr_t>(channel) % 16 == 0) &&
                        (static_cast<uint64_t>(n_frames) * esz) % 16 == 0 && tensor_map_encoder() != nullptr)
                           ? 1
                           : 0;
        p.lp.smem = staged_smem_bytes(w, fc, esz, static_cast<int>(n_tx));
        return p;
    }
    // warp-per-voxel multi-frame kernel (any frame count)
    int lpv;
    if (n_frames <= 16) {
        p.lp.kind = kKindWarpHalf;
        lpv = 16;
        p.lp.passes = 1;
    } else {
        p.lp.kind = kKindWarp;
        lpv = 32;
        p.lp.passes = static_cast<int>(std::min<uint32_t>(8, (n_frames + 31) / 32));
    }
    const uint64_t vox_per_cta = static_cast<uint64_t>(kThreadsPerBlock / 32) * (32 / lpv);
    p.lp.block = dim3(kThreadsPerBlock, 1, 1);
    p.lp.grid.x = static_cast<unsigned>((n_vox + vox_per_cta - 1) / vox_per_cta);
    const uint32_t frames_per_cta = static_cast<uint32_t>(lpv * p.lp.passes);
    p.lp.grid.y = (n_frames + frames_per_cta - 1) / frames_per_cta;
    p.lp.grid.z = 1;
    p.lp.smem = 0;
    p.lp.tx_chunk = 1;
    return p;
}

// 2-D TMA view of one launch's channel data: inner dim = frames, outer = (tx, element, sample) rows.
int encode_channel_map(CUtensorMap* map, int storage, const void* channel, uint64_t rows, uint32_t n_frames,
                       int frame_chunk, int window_rows) {
    const int esz = static_cast<int>(storage_bytes(storage));
    const CUtensorMapDataType dt =
        esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : (esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16);
    const cuuint64_t dims[2] = {n_frames, rows};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(n_frames) * esz};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(frame_chunk), static_cast<cuuint32_t>(window_rows)};
    const cuuint32_t elem_strides[2] = {1, 1};
    const CUresult r = tensor_map_encoder()(map, dt, 2, const_cast<void*>(channel), dims, strides, box, elem_strides,
                                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MACH_B200_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", static_cast<int>(r));
    return MACH_B200_OK;
}

cudaError_t dispatch(int storage, const DasArgs& a, int interp, const Plan& plan, const CUtensorMap& map,
                     cudaStream_t st) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
#define MACH_B200_CASE(S)                                                              \
    case S:                                                                             \
        return plan.staged ? launch_das_staged<S>(a, plan.st, map, interp, plan.lp, st) \
                           : launch_das<S>(a, interp, plan.lp, st);
    if (plan.frame_lane) {
#define MACH_B200_FCASE(S) \
    case S: return launch_das_frame_lane<S>(a, plan.fl, interp, plan.lp, st);
        switch (storage) {
            MACH_B200_FCASE(kF32)
            MACH_B200_FCASE(kC64)
            MACH_B200_FCASE(kF16)
            MACH_B200_FCASE(kCF16)
            MACH_B200_FCASE(kBF16)
            MACH_B200_FCASE(kCBF16)
            MACH_B200_FCASE(kI16)
            default: return launch_das_frame_lane<kCI16>(a, plan.fl, interp, plan.lp, st);
        }
#undef MACH_B200_FCASE
    }
    if (plan.ensemble) {
#define MACH_B200_ECASE(S) \
    case S: return launch_das_ensemble<S>(a, plan.st, plan.ea, map, interp, plan.lp.smem, st);
        switch (storage) {
            MACH_B200_ECASE(kF32)
            MACH_B200_ECASE(kC64)
            MACH_B200_ECASE(kF16)
            MACH_B200_ECASE(kCF16)
            MACH_B200_ECASE(kBF16)
            MACH_B200_ECASE(kCBF16)
            MACH_B200_ECASE(kI16)
            default: return launch_das_ensemble<kCI16>(a, plan.st, plan.ea, map, interp, plan.lp.smem, st);
        }
#undef MACH_B200_ECASE
    }
    switch (storage) {
        MACH_B200_CASE(kF32)
        MACH_B200_CASE(kC64)
        MACH_B200_CASE(kF16)
        MACH_B200_CASE(kCF16)
        MACH_B200_CASE(kBF16)
        MACH_B200_CASE(kCBF16)
        MACH_B200_CASE(kI16)
        default:
            return plan.staged ? launch_das_staged<kCI16>(a, plan.st, map, interp, plan.lp, st)
                               : launch_das<kCI16>(a, interp, plan.lp, st);
    }
#undef MACH_B200_CASE
}

// Stream-ordered device buffer released at scope exit (on the stream it was allocated on).
struct DeviceBuffer {
    void* ptr = nullptr;
    cudaStream_t stream = nullptr;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    cudaError_t alloc(size_t bytes, cudaStream_t st) {
        stream = st;
        int device = 0;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaGetDevice(&device);
        if (e == cudaSuccess) e = library_pool(device, &pool);
        if (e != cudaSuccess) return e;
        return cudaMallocFromPoolAsync(&ptr, bytes ? bytes : 1, pool, st);
    }
    ~DeviceBuffer() {
        if (ptr) cudaFreeAsync(ptr, stream);
    }
};

// Launch transmits [0, a.n_tx) so that every launch's channel span stays below 2^31 samples
// (32-bit offsets inside the kernels).  Later launches always accumulate.
// Lane-voxel launches (which may run the elements in blocks, one launch each).
bool lane_voxel_plan(const Plan& plan) {
    return !plan.staged && !plan.ensemble && !plan.frame_lane &&
           (plan.lp.kind == kKindLaneVoxel1 || plan.lp.kind == kKindLaneVoxelN || plan.lp.kind == kKindLaneVoxel16 ||
            plan.lp.kind == kKindLaneVoxel8);
}

// Whether a staging buffer of `bytes` leaves at least as much device memory free (else the
// transmit-chunk staging, whose buffers are bounded, is used).
bool fits_on_device(size_t bytes) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return bytes <= free_b / 2;
}

// Host channel data of a job that runs in element blocks is staged block by block.
bool element_block_staging(const Plan& plan, uint32_t n_rx) {
    return lane_voxel_plan(plan) && plan.lp.element_block > 0 && static_cast<uint32_t>(plan.lp.element_block) < n_rx;
}

int dispatch_split(int storage, DasArgs a, int interp, const Plan& plan, cudaStream_t st) {
    const size_t esz = storage_bytes(storage);
    const int64_t per_tx = static_cast<int64_t>(a.n_rx) * a.row_stride;
    const char* ch = static_cast<const char*>(a.channel);
    const int total = a.n_tx;
    const TransmitSplit split = split_transmits(per_tx, total);
    // Ensemble launches take work items from a zeroed device counter (one per launch).
    DeviceBuffer counters;
    Plan pl = plan;
    if (plan.ensemble) {
        MACH_B200_CUDA_TRY(counters.alloc(sizeof(int) * static_cast<size_t>(split.n_launch), st));
        MACH_B200_CUDA_TRY(cudaMemsetAsync(counters.ptr, 0, sizeof(int) * static_cast<size_t>(split.n_launch), st));
    }
    // Lane-voxel kernels may run the elements in blocks, one launch each, so that a launch's
    // channel data stays in L2 while every CTA sweeps it.
    const bool lane_voxel = lane_voxel_plan(plan);
    const int eblk = lane_voxel && plan.lp.element_block > 0 ? plan.lp.element_block : std::max(a.n_rx, 1);
    for (int64_t k = 0; k < split.n_launch; ++k) {
        const int64_t t0 = launch_first_tx(split, k);
        DasArgs b = a;
        b.n_tx = static_cast<int32_t>(launch_tx_count(split, total, k));
        b.channel = ch + static_cast<size_t>(t0) * static_cast<size_t>(per_tx) * esz;
        b.arrivals = a.arrivals + t0 * a.n_vox;
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if ((plan.staged || plan.ensemble) && plan.st.use_tma && b.n_tx > 0) {
            const int fc = plan.ensemble ? plan.ea.box_x : plan.lp.lanes_per_voxel * static_cast<int>(8 / esz);
            const int rc = encode_channel_map(&map, storage, b.channel,
                                              static_cast<uint64_t>(b.n_tx) * a.n_rx * a.n_samples, a.n_frames, fc,
                                              plan.st.window_rows);
            if (rc) return rc;
        }
        if (plan.ensemble) pl.ea.counter = static_cast<int*>(counters.ptr) + k;
        int e0 = 0;
        do {
            b.e_begin = e0;
            b.e_end = std::min(a.n_rx, e0 + eblk);
            b.accumulate = (t0 == 0 && e0 == 0) ? a.accumulate : 1;
            MACH_B200_CUDA_TRY(dispatch(storage, b, interp, pl, map, st));
            e0 += eblk;
        } while (e0 < a.n_rx);
    }
    return MACH_B200_OK;
}

struct EventPair {
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~EventPair() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    cudaError_t create() {
        for (auto& e : ev) {
            const cudaError_t err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (err != cudaSuccess) return err;
        }
        return cudaSuccess;
    }
};

struct StreamHolder {
    cudaStream_t s = nullptr;
    ~StreamHolder() {
        if (s) cudaStreamDestroy(s);
    }
};

// After a synchronous call that ran a kernel with bounded waits: report (and clear) a timeout.
int check_status(DeviceState* dev, cudaStream_t stream) {
    int status = 0;
    MACH_B200_CUDA_TRY(cudaMemcpyAsync(&status, dev->status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    if (status != 0) {
        const int zero = 0;
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(dev->status, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
        MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
        return fail(MACH_B200_ERR_CUDA, "a kernel wait timed out (status %d); the output is incomplete", status);
    }
    return MACH_B200_OK;
}

// Launch arguments shared by every kernel family (FP32 constants rounded on the host the
// way mach's launcher rounds them, split-delay FP64 constants).
DasArgs make_args(const float* rx_coords_m, const float* scan_coords_m, uint64_t n_scan, uint32_t n_rx,
                  uint32_t n_samples, uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                  float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha, float channel_scale, bool cplx,
                  uint32_t flags) {
    DasArgs a{};
    a.rx = rx_coords_m;
    a.scan = scan_coords_m;
    a.n_vox = static_cast<int64_t>(n_scan);
    a.n_rx = static_cast<int32_t>(n_rx);
    a.e_begin = 0;
    a.e_end = a.n_rx;
    a.n_samples = static_cast<int32_t>(n_samples);
    a.n_frames = static_cast<int32_t>(n_frames);
    a.row_stride = static_cast<int64_t>(n_samples) * n_frames;
    a.inv_c = 1.0f / sound_speed_m_s;  // kernel.cu:750, FP32 on the host
    a.fs = sampling_freq_hz;
    a.t0 = rx_start_s;
    a.two_f_number = 2.0f * f_number;
    a.alpha = tukey_alpha;
    a.one_minus_alpha = 1.0f - tukey_alpha;
    a.mod_rad = (2.0f * kPi) * modulation_freq_hz;  // kernel.cu:571
    a.scale = channel_scale;
    a.hi_nearest = static_cast<float>(n_samples) - 0.5f;
    a.hi_linear = static_cast<float>(n_samples - 1u);
    a.hi_quadratic = static_cast<float>(n_samples) - 2.0f;
    a.apod = tukey_alpha > 0.0f;
    a.rotate = cplx && modulation_freq_hz != 0.0f;
    a.split = (flags & MACH_B200_FLAG_SPLIT_DELAY) != 0u ? 1 : 0;
    a.fs_d = sampling_freq_hz;
    a.t0_d = rx_start_s;
    a.fmod_d = modulation_freq_hz;
    a.fs_over_c = static_cast<double>(sampling_freq_hz) / static_cast<double>(sound_speed_m_s);
    a.fmod_over_c = static_cast<double>(modulation_freq_hz) / static_cast<double>(sound_speed_m_s);
    const double start = -static_cast<double>(rx_start_s) * static_cast<double>(sampling_freq_hz);
    const double b = std::floor(start);
    a.start_base = static_cast<int32_t>(std::max(-2.0e9, std::min(2.0e9, b)));
    a.start_frac = static_cast<float>(start - b);
    return a;
}

// Argument checks shared by every entry point (messages follow mach where it has one).
int check_args(int32_t storage, int32_t interp_type, float tukey_alpha, uint32_t n_tx, uint32_t n_rx,
               uint32_t n_samples, uint64_t n_scan, uint32_t n_frames) {
    if (storage < kF32 || storage > kCI16) return fail(MACH_B200_ERR_VALUE, "unknown storage code %d", storage);
    if (interp_type < kNearest || interp_type > kQuadratic) {
        return fail(MACH_B200_ERR_VALUE,
                    "interp_type must be 0 (NearestNeighbor), 1 (Linear) or 2 (Quadratic), got %d", interp_type);
    }
    // Same range check and message as mach (src/mach/kernel.cu:745-748).
    if (!(tukey_alpha >= 0.0f && tukey_alpha <= 1.0f)) {
        return fail(MACH_B200_ERR_VALUE, "Error: tukey_alpha must be in range [0, 1], but got %f", tukey_alpha);
    }
    if (n_frames > 1000000u) return fail(MACH_B200_ERR_VALUE, "n_frames %u is too large (at most 1000000)", n_frames);
    // Sample positions are rounded with FP32 adds that are exact below 2^22.
    if (n_samples > (1u << 22)) return fail(MACH_B200_ERR_VALUE, "n_samples %u exceeds 2^22", n_samples);
    // One transmit's channel data is addressed with 32-bit offsets.
    if (static_cast<uint64_t>(n_rx) * n_samples * n_frames >= (uint64_t{1} << 31)) {
        return fail(MACH_B200_ERR_VALUE, "one transmit holds %llu samples; at most 2^31 - 1 are supported",
                    static_cast<unsigned long long>(static_cast<uint64_t>(n_rx) * n_samples * n_frames));
    }
    if (n_rx > 0x7fffffffu || n_tx > 0x7fffffffu) return fail(MACH_B200_ERR_VALUE, "n_rx / n_tx too large");
    if (n_scan > 0x7fffffffull * 4ull) {
        return fail(MACH_B200_ERR_VALUE, "n_scan %llu is too large", static_cast<unsigned long long>(n_scan));
    }
    return MACH_B200_OK;
}

int power_impl(int32_t storage, const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
               const float* tx_wave_arrivals_s, void* out, uint32_t n_tx, uint32_t n_rx, uint32_t n_samples,
               uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
               float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha, int32_t interp_type,
               float channel_scale, cudaStream_t stream, const mach_b200_options& opt);

int compound_impl(int32_t storage, const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                  const float* tx_wave_arrivals_s, void* out, uint32_t n_tx, uint32_t n_rx, uint32_t n_samples,
                  uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                  float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha, int32_t interp_type,
                  float channel_scale, cudaStream_t stream, const mach_b200_options& opt) {
    if (opt.flags & MACH_B200_FLAG_POWER_DOPPLER) {
        return power_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                          n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                          modulation_freq_hz, tukey_alpha, interp_type, channel_scale, stream, opt);
    }
    g_error.clear();
    const uint32_t flags = opt.flags;
    int rc0 = check_args(storage, interp_type, tukey_alpha, n_tx, n_rx, n_samples, n_scan, n_frames);
    if (rc0) return rc0;
    if (n_scan == 0 || n_frames == 0) return MACH_B200_OK;  // empty output: nothing to write
    if (!out || !scan_coords_m) return fail(MACH_B200_ERR_VALUE, "out and scan_coords_m must not be NULL");
    const bool need_channel = n_tx > 0 && n_rx > 0 && n_samples > 0;
    if (need_channel && (!channel_data || !rx_coords_m || !tx_wave_arrivals_s)) {
        return fail(MACH_B200_ERR_VALUE, "channel_data, rx_coords_m and tx_wave_arrivals_s must not be NULL");
    }

    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    DeviceState* dev = nullptr;
    int rc;
    if ((rc = device_state(device, &dev))) return rc;
    Residency r_ch = kOnDevice, r_rx = kOnDevice, r_scan = kOnDevice, r_arr = kOnDevice, r_out = kOnDevice;
    if (need_channel) {
        if ((rc = residency(channel_data, device, &r_ch, "channel_data"))) return rc;
        if ((rc = residency(rx_coords_m, device, &r_rx, "rx_coords_m"))) return rc;
        if ((rc = residency(tx_wave_arrivals_s, device, &r_arr, "tx_wave_arrivals_s"))) return rc;
    }
    if ((rc = residency(scan_coords_m, device, &r_scan, "scan_coords_m"))) return rc;
    if ((rc = residency(out, device, &r_out, "out"))) return rc;

    const bool cplx = (storage & 1) != 0;
    const size_t esz = storage_bytes(storage);
    const size_t out_bytes = static_cast<size_t>(n_scan) * n_frames * (cplx ? 8 : 4);

    DasArgs a = make_args(rx_coords_m, scan_coords_m, n_scan, need_channel ? n_rx : 0, n_samples, n_frames, f_number,
                          rx_start_s, sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha,
                          channel_scale, cplx, flags);
    const bool overwrite = (flags & MACH_B200_FLAG_OVERWRITE) != 0u || r_out != kOnDevice;
    Plan plan = plan_launch(storage, n_scan, n_frames, n_tx, channel_data, r_ch == kOnDevice, opt, interp_type, false,
                            n_rx, n_samples);
    plan.st.status = dev->status;
    a.frame_passes = plan.lp.passes;
    a.tx_chunk = plan.lp.tx_chunk;
    a.map_fast = plan.lp.map_fast;
    a.map_wlog = plan.lp.map_wlog;
    a.tile_rev = plan.lp.tile_rev;
    a.map_outer = plan.lp.map_outer;
    a.frame_chunks = plan.lp.frame_chunks;

    const bool all_device = r_ch == kOnDevice && r_rx == kOnDevice && r_scan == kOnDevice && r_arr == kOnDevice &&
                            r_out == kOnDevice;
    if (all_device) {
        a.channel = channel_data;
        a.arrivals = tx_wave_arrivals_s;
        a.out = out;
        a.n_tx = static_cast<int32_t>(need_channel ? n_tx : 0);
        a.accumulate = overwrite ? 0 : 1;
        if ((rc = dispatch_split(storage, a, interp_type, plan, stream))) return rc;
        if (!(flags & MACH_B200_FLAG_ASYNC)) {
            MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
            if (plan.staged || plan.ensemble) return check_status(dev, stream);
        }
        return MACH_B200_OK;
    }

    // ---- staging path: some buffers live in host memory ----
    DeviceBuffer d_rx, d_scan, d_out, d_ch[2], d_arr[2];
    if (need_channel && r_rx != kOnDevice) {
        MACH_B200_CUDA_TRY(d_rx.alloc(static_cast<size_t>(n_rx) * 12, stream));
        MACH_B200_CUDA_TRY(
            cudaMemcpyAsync(d_rx.ptr, rx_coords_m, static_cast<size_t>(n_rx) * 12, cudaMemcpyHostToDevice, stream));
        a.rx = static_cast<const float*>(d_rx.ptr);
    }
    if (r_scan != kOnDevice) {
        MACH_B200_CUDA_TRY(d_scan.alloc(static_cast<size_t>(n_scan) * 12, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_scan.ptr, scan_coords_m, static_cast<size_t>(n_scan) * 12,
                                           cudaMemcpyHostToDevice, stream));
        a.scan = static_cast<const float*>(d_scan.ptr);
    }
    void* dev_out = out;
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(d_out.alloc(out_bytes, stream));
        dev_out = d_out.ptr;
    }
    a.out = dev_out;

    const size_t tx_bytes = static_cast<size_t>(n_rx) * n_samples * n_frames * esz;
    const size_t arr_bytes = static_cast<size_t>(n_scan) * 4;
    if (!need_channel) {
        // No samples to gather: the result is zero.
        MACH_B200_CUDA_TRY(cudaMemsetAsync(dev_out, 0, out_bytes, stream));
    } else if (r_ch == kOnDevice && r_arr == kOnDevice) {
        a.channel = channel_data;
        a.arrivals = tx_wave_arrivals_s;
        a.n_tx = static_cast<int32_t>(n_tx);
        a.accumulate = overwrite ? 0 : 1;
        if ((rc = dispatch_split(storage, a, interp_type, plan, stream))) return rc;
    } else if (r_ch != kOnDevice && element_block_staging(plan, n_rx) &&
               split_transmits(static_cast<int64_t>(n_rx) * a.row_stride, n_tx).n_launch == 1 &&
               fits_on_device(tx_bytes * n_tx)) {
        // Element blocks (the lane-voxel launches of a job far larger than L2): the channel
        // data gets one device buffer, filled block by block on a side stream (one 2-D copy of
        // the block's rows of every transmit), and each block's launch waits only for its own
        // rows, so the copy of block b + 1 overlaps the gather of block b.
        const int eblk = plan.lp.element_block;
        const size_t row_bytes = static_cast<size_t>(n_samples) * n_frames * esz;
        const int n_blk = static_cast<int>((n_rx + eblk - 1) / eblk);
        StreamHolder copy;
        std::vector<cudaEvent_t> block_ready(static_cast<size_t>(n_blk), nullptr);
        struct EventList {
            std::vector<cudaEvent_t>& ev;
            ~EventList() {
                for (auto e : ev)
                    if (e) cudaEventDestroy(e);
            }
        } events{block_ready};
        MACH_B200_CUDA_TRY(cudaStreamCreateWithFlags(&copy.s, cudaStreamNonBlocking));
        for (auto& e : block_ready) MACH_B200_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        MACH_B200_CUDA_TRY(d_ch[0].alloc(tx_bytes * n_tx, stream));
        if (r_arr != kOnDevice) MACH_B200_CUDA_TRY(d_arr[0].alloc(arr_bytes * n_tx, stream));
        cudaEvent_t ready;  // the copy stream must not start before the buffers exist
        MACH_B200_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        cudaEventRecord(ready, stream);
        cudaStreamWaitEvent(copy.s, ready, 0);
        cudaEventDestroy(ready);
        if (r_arr != kOnDevice) {
            MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_arr[0].ptr, tx_wave_arrivals_s, arr_bytes * n_tx,
                                               cudaMemcpyHostToDevice, copy.s));
            a.arrivals = static_cast<const float*>(d_arr[0].ptr);
        } else {
            a.arrivals = tx_wave_arrivals_s;
        }
        a.channel = d_ch[0].ptr;
        a.n_tx = static_cast<int32_t>(n_tx);
        const char* h_ch = static_cast<const char*>(channel_data);
        char* d_base = static_cast<char*>(d_ch[0].ptr);
        for (int k = 0; k < n_blk; ++k) {
            const int e0 = k * eblk;
            const int e1 = std::min<int>(static_cast<int>(n_rx), e0 + eblk);
            MACH_B200_CUDA_TRY(cudaMemcpy2DAsync(d_base + row_bytes * e0, tx_bytes, h_ch + row_bytes * e0, tx_bytes,
                                                 row_bytes * static_cast<size_t>(e1 - e0), n_tx,
                                                 cudaMemcpyHostToDevice, copy.s));
            MACH_B200_CUDA_TRY(cudaEventRecord(block_ready[k], copy.s));
            MACH_B200_CUDA_TRY(cudaStreamWaitEvent(stream, block_ready[k], 0));
            DasArgs b = a;
            b.e_begin = e0;
            b.e_end = e1;
            b.accumulate = (k > 0 || !overwrite) ? 1 : 0;
            CUtensorMap map;
            std::memset(&map, 0, sizeof(map));
            MACH_B200_CUDA_TRY(dispatch(storage, b, interp_type, plan, map, stream));
        }
    } else {
        // Transmit chunks (>= 64 MB, at most 8 of them) copied on a side stream while the
        // previous chunk is gathered.
        const size_t target = size_t{64} << 20;
        const uint32_t by_bytes = static_cast<uint32_t>(std::max<size_t>(1, target / std::max<size_t>(tx_bytes, 1)));
        const uint32_t chunk =
            std::max<uint32_t>(1u, std::min<uint32_t>(n_tx, std::max<uint32_t>(by_bytes, (n_tx + 7u) / 8u)));
        StreamHolder copy;
        EventPair copied, consumed;
        MACH_B200_CUDA_TRY(cudaStreamCreateWithFlags(&copy.s, cudaStreamNonBlocking));
        MACH_B200_CUDA_TRY(copied.create());
        MACH_B200_CUDA_TRY(consumed.create());
        // The copy stream must not start before buffers allocated on `stream` exist.
        cudaEvent_t ready;
        MACH_B200_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        for (int b = 0; b < 2; ++b) {
            if (r_ch != kOnDevice) MACH_B200_CUDA_TRY(d_ch[b].alloc(tx_bytes * chunk, stream));
            if (r_arr != kOnDevice) MACH_B200_CUDA_TRY(d_arr[b].alloc(arr_bytes * chunk, stream));
        }
        cudaEventRecord(ready, stream);
        cudaStreamWaitEvent(copy.s, ready, 0);
        cudaEventDestroy(ready);
        const char* h_ch = static_cast<const char*>(channel_data);
        const char* h_arr = reinterpret_cast<const char*>(tx_wave_arrivals_s);
        uint32_t k = 0;
        for (uint32_t t0 = 0; t0 < n_tx; t0 += chunk, ++k) {
            const uint32_t nt = std::min(chunk, n_tx - t0);
            const int b = static_cast<int>(k & 1u);
            if (k >= 2) MACH_B200_CUDA_TRY(cudaStreamWaitEvent(copy.s, consumed.ev[b], 0));
            if (r_ch != kOnDevice) {
                MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_ch[b].ptr, h_ch + tx_bytes * t0, tx_bytes * nt,
                                                   cudaMemcpyHostToDevice, copy.s));
                a.channel = d_ch[b].ptr;
            } else {
                a.channel = h_ch + tx_bytes * t0;
            }
            if (r_arr != kOnDevice) {
                MACH_B200_CUDA_TRY(cudaMemcpyAsync(d_arr[b].ptr, h_arr + arr_bytes * t0, arr_bytes * nt,
                                                   cudaMemcpyHostToDevice, copy.s));
                a.arrivals = static_cast<const float*>(d_arr[b].ptr);
            } else {
                a.arrivals = reinterpret_cast<const float*>(h_arr + arr_bytes * t0);
            }
            MACH_B200_CUDA_TRY(cudaEventRecord(copied.ev[b], copy.s));
            MACH_B200_CUDA_TRY(cudaStreamWaitEvent(stream, copied.ev[b], 0));
            a.n_tx = static_cast<int32_t>(nt);
            a.accumulate = (k > 0 || !overwrite) ? 1 : 0;
            if ((rc = dispatch_split(storage, a, interp_type, plan, stream))) return rc;
            MACH_B200_CUDA_TRY(cudaEventRecord(consumed.ev[b], stream));
        }
    }
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(out, dev_out, out_bytes, cudaMemcpyDeviceToHost, stream));
    }
    // Host buffers are in use until the stream drains: always synchronous here.
    MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    if (plan.staged || plan.ensemble) return check_status(dev, stream);
    return MACH_B200_OK;
}

// ---------------------------------------------------------------- transmit models
//
// mach_b200_options.tx_model != 0: the [n_tx][n_scan] arrivals are formed on the device by one
// kernel (das_transmit.cu) from the FP64 table tx_params, and the call then runs as with an
// arrivals array.  Only the table and, for host scan points, the points cross the host link.

struct TxArrivals {
    DeviceBuffer params, scan, arr;
    const float* ptr = nullptr;
};

int form_tx_arrivals(const mach_b200_options& o, const float* scan_coords_m, uint32_t n_tx, uint64_t n_scan,
                     float sound_speed_m_s, cudaStream_t stream, TxArrivals& t) {
    if (o.tx_model != MACH_B200_TX_PLANE && o.tx_model != MACH_B200_TX_SPHERICAL) {
        return fail(MACH_B200_ERR_VALUE, "tx_model must be 0 (arrays), 1 (plane) or 2 (spherical), got %d", o.tx_model);
    }
    if (!o.tx_params) return fail(MACH_B200_ERR_VALUE, "tx_model %d needs tx_params", o.tx_model);
    if (n_tx == 0 || n_scan == 0) return MACH_B200_OK;
    if (!scan_coords_m) return fail(MACH_B200_ERR_VALUE, "out and scan_coords_m must not be NULL");
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    Residency r_p, r_s;
    int rc;
    if ((rc = residency(o.tx_params, device, &r_p, "tx_params"))) return rc;
    if ((rc = residency(scan_coords_m, device, &r_s, "scan_coords_m"))) return rc;
    const double* params = o.tx_params;
    if (r_p != kOnDevice) {
        const size_t bytes = static_cast<size_t>(n_tx) * 8 * sizeof(double);
        MACH_B200_CUDA_TRY(t.params.alloc(bytes, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(t.params.ptr, o.tx_params, bytes, cudaMemcpyHostToDevice, stream));
        params = static_cast<const double*>(t.params.ptr);
    }
    const float* scan = scan_coords_m;
    if (r_s != kOnDevice) {
        const size_t bytes = static_cast<size_t>(n_scan) * 12;
        MACH_B200_CUDA_TRY(t.scan.alloc(bytes, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(t.scan.ptr, scan_coords_m, bytes, cudaMemcpyHostToDevice, stream));
        scan = static_cast<const float*>(t.scan.ptr);
    }
    MACH_B200_CUDA_TRY(t.arr.alloc(static_cast<size_t>(n_tx) * n_scan * sizeof(float), stream));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    MACH_B200_CUDA_TRY(launch_tx_arrivals(o.tx_model, params, scan, static_cast<int64_t>(n_scan),
                                          static_cast<int>(n_tx), static_cast<double>(sound_speed_m_s),
                                          static_cast<float*>(t.arr.ptr), stream));
    t.ptr = static_cast<const float*>(t.arr.ptr);
    return MACH_B200_OK;
}

mach_b200_options default_options(uint32_t flags) {
    mach_b200_options o;
    std::memset(&o, 0, sizeof(o));
    o.struct_size = sizeof(o);
    o.flags = flags;
    return o;
}


// ---------------------------------------------------------------- power-Doppler epilogue
//
// out (float32 [n_scan]) (+)= sum over frames of |beamformed value|^2.  All-device jobs that
// the ensemble kernel takes in one launch get the epilogue fused into the kernel (each frame
// block adds its part atomically); every other job is beamformed into a temporary
// [n_scan][n_frames] image that one reduction kernel turns into the power image.

int power_impl(int32_t storage, const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
               const float* tx_wave_arrivals_s, void* out, uint32_t n_tx, uint32_t n_rx, uint32_t n_samples,
               uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
               float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha, int32_t interp_type,
               float channel_scale, cudaStream_t stream, const mach_b200_options& opt) {
    g_error.clear();
    const uint32_t flags = opt.flags;
    int rc = check_args(storage, interp_type, tukey_alpha, n_tx, n_rx, n_samples, n_scan, n_frames);
    if (rc) return rc;
    if (n_scan == 0) return MACH_B200_OK;
    if (!out || !scan_coords_m) return fail(MACH_B200_ERR_VALUE, "out and scan_coords_m must not be NULL");
    const bool need_channel = n_tx > 0 && n_rx > 0 && n_samples > 0 && n_frames > 0;
    if (need_channel && (!channel_data || !rx_coords_m || !tx_wave_arrivals_s)) {
        return fail(MACH_B200_ERR_VALUE, "channel_data, rx_coords_m and tx_wave_arrivals_s must not be NULL");
    }
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    DeviceState* dev = nullptr;
    if ((rc = device_state(device, &dev))) return rc;
    Residency r_out;
    if ((rc = residency(out, device, &r_out, "out"))) return rc;
    bool all_device = r_out == kOnDevice;
    if (need_channel) {
        const void* ptrs[4] = {channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s};
        const char* names[4] = {"channel_data", "rx_coords_m", "scan_coords_m", "tx_wave_arrivals_s"};
        for (int i = 0; i < 4; ++i) {
            Residency r;
            if ((rc = residency(ptrs[i], device, &r, names[i]))) return rc;
            all_device = all_device && r == kOnDevice;
        }
    }
    const bool overwrite = (flags & MACH_B200_FLAG_OVERWRITE) != 0u || r_out != kOnDevice;
    const bool cplx = (storage & 1) != 0;
    const size_t power_bytes = static_cast<size_t>(n_scan) * sizeof(float);

    // ---- fused: the ensemble / frame-lane kernel adds |x|^2 of each frame block into out
    if (all_device && need_channel) {
        Plan plan = plan_launch(storage, n_scan, n_frames, n_tx, channel_data, true, opt, interp_type);
        const int64_t per_tx = static_cast<int64_t>(n_rx) * n_samples * n_frames;
        if ((plan.ensemble || plan.frame_lane) && per_tx * n_tx < (int64_t{1} << 31)) {
            plan.st.status = dev->status;
            DasArgs a = make_args(rx_coords_m, scan_coords_m, n_scan, n_rx, n_samples, n_frames, f_number, rx_start_s,
                                  sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha, channel_scale,
                                  cplx, flags);
            a.frame_passes = plan.lp.passes;
            a.tx_chunk = plan.lp.tx_chunk;
            a.channel = channel_data;
            a.arrivals = tx_wave_arrivals_s;
            a.out = out;
            a.n_tx = static_cast<int32_t>(n_tx);
            a.accumulate = 1;
            a.power = 1;
            if (overwrite) MACH_B200_CUDA_TRY(cudaMemsetAsync(out, 0, power_bytes, stream));
            if ((rc = dispatch_split(storage, a, interp_type, plan, stream))) return rc;
            if (!(flags & MACH_B200_FLAG_ASYNC)) {
                MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
                return check_status(dev, stream);
            }
            return MACH_B200_OK;
        }
    }

    // ---- general: full image into a temporary buffer, then the reduction kernel
    const size_t image_bytes = static_cast<size_t>(n_scan) * n_frames * (cplx ? 8 : 4);
    DeviceBuffer image, power;
    MACH_B200_CUDA_TRY(image.alloc(image_bytes, stream));
    mach_b200_options o = opt;
    o.flags = (flags & ~(MACH_B200_FLAG_POWER_DOPPLER | MACH_B200_FLAG_ASYNC)) | MACH_B200_FLAG_OVERWRITE;
    if (all_device && (flags & MACH_B200_FLAG_ASYNC)) o.flags |= MACH_B200_FLAG_ASYNC;
    if ((rc = compound_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, image.ptr, n_tx,
                            n_rx, n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz,
                            sound_speed_m_s, modulation_freq_hz, tukey_alpha, interp_type, channel_scale, stream,
                            o))) {
        return rc;
    }
    float* dst = static_cast<float*>(out);
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(power.alloc(power_bytes, stream));
        dst = static_cast<float*>(power.ptr);
    }
    MACH_B200_CUDA_TRY(launch_power_epilogue(image.ptr, dst, static_cast<int64_t>(n_scan), static_cast<int>(n_frames),
                                             cplx, !overwrite, stream));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (r_out != kOnDevice) {
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(out, dst, power_bytes, cudaMemcpyDeviceToHost, stream));
    }
    if (!all_device || !(flags & MACH_B200_FLAG_ASYNC)) MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    return MACH_B200_OK;
}

// ---------------------------------------------------------------- channel-data ingest

int ingest_impl(int32_t src_storage, const void* src, int32_t dst_storage, void* dst, uint32_t n_samples,
                uint32_t n_elements, uint32_t n_waves, uint32_t n_frames, float scale, cudaStream_t stream,
                uint32_t flags) {
    g_error.clear();
    if (src_storage < kF32 || src_storage > kCI16 || dst_storage < kF32 || dst_storage > kCI16) {
        return fail(MACH_B200_ERR_VALUE, "unknown storage code (%d -> %d)", src_storage, dst_storage);
    }
    if ((src_storage & 1) != (dst_storage & 1)) {
        return fail(MACH_B200_ERR_VALUE, "source and destination must both be real or both be complex");
    }
    const uint64_t count = static_cast<uint64_t>(n_samples) * n_elements * n_waves * n_frames;
    if (count == 0) return MACH_B200_OK;
    if (!src || !dst) return fail(MACH_B200_ERR_VALUE, "src and dst must not be NULL");
    if (n_samples > 0x7fffffffu || n_elements > 65535u || n_waves > 0x7fffffffu || n_frames > 0x7fffffffu) {
        return fail(MACH_B200_ERR_VALUE, "dimensions out of range (at most 65535 elements)");
    }
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    Residency r_src, r_dst;
    int rc;
    if ((rc = residency(src, device, &r_src, "src"))) return rc;
    if ((rc = residency(dst, device, &r_dst, "dst"))) return rc;
    if (r_dst != kOnDevice) return fail(MACH_B200_ERR_VALUE, "dst must be device memory");
    DeviceBuffer staged;
    const void* dsrc = src;
    if (r_src != kOnDevice) {
        const size_t bytes = count * storage_bytes(src_storage);
        MACH_B200_CUDA_TRY(staged.alloc(bytes, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(staged.ptr, src, bytes, cudaMemcpyHostToDevice, stream));
        dsrc = staged.ptr;
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    MACH_B200_CUDA_TRY(launch_ingest(src_storage, dsrc, dst_storage, dst, static_cast<int>(n_samples),
                                     static_cast<int>(n_elements), static_cast<int>(n_waves),
                                     static_cast<int>(n_frames), scale, stream));
    if (r_src != kOnDevice || !(flags & MACH_B200_FLAG_ASYNC)) MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    return MACH_B200_OK;
}

// ---------------------------------------------------------------- analytic signal (RF -> IQ)
//
// scipy.signal.hilbert along the sample axis (src/mach/io/uff.py:88), from the channel layout
// or fused with the acquisition-order rearrange of src/mach/io/uff.py:101-102.

int hilbert_impl(int32_t src_storage, const void* src, int32_t src_layout, int32_t dst_storage, void* dst,
                 uint32_t n_samples, uint32_t n_elements, uint32_t n_waves, uint32_t n_frames, float scale,
                 cudaStream_t stream, uint32_t flags) {
    g_error.clear();
    if (src_storage < kF32 || src_storage > kCI16 || dst_storage < kF32 || dst_storage > kCI16) {
        return fail(MACH_B200_ERR_VALUE, "unknown storage code (%d -> %d)", src_storage, dst_storage);
    }
    if ((src_storage & 1) || !(dst_storage & 1)) {
        return fail(MACH_B200_ERR_VALUE, "the analytic signal takes real channel data to a complex storage");
    }
    if (src_layout != MACH_B200_LAYOUT_CHANNEL && src_layout != MACH_B200_LAYOUT_ACQUISITION) {
        return fail(MACH_B200_ERR_VALUE, "src_layout must be 0 (channel) or 1 (acquisition), got %d", src_layout);
    }
    const uint64_t count = static_cast<uint64_t>(n_samples) * n_elements * n_waves * n_frames;
    if (count == 0) return MACH_B200_OK;
    if (!src || !dst) return fail(MACH_B200_ERR_VALUE, "src and dst must not be NULL");
    HilbertArgs g{};
    g.n = static_cast<int>(std::min<uint32_t>(n_samples, 0x7fffffffu));
    g.n_stages = hilbert_plan(g.n, g.radix, kHilMaxStages);
    if (g.n_stages < 0) return fail(MACH_B200_ERR_VALUE, "n_samples %u has too many factors", n_samples);
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    int max_smem = 0;
    MACH_B200_CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    // Shared memory: stage twiddles + odd-radix roots + two padded buffers per column pair.
    g.pair_stride = g.n + (g.n >> 5) + 1;  // one float2 of padding per 32
    const uint64_t col_bytes = 8ull * g.pair_stride;
    const uint64_t fixed = 8ull * (kHilRoots + g.n);
    if (col_bytes * 2 + fixed > static_cast<uint64_t>(max_smem)) {
        return fail(MACH_B200_ERR_VALUE, "n_samples %u is too long for the on-device analytic signal (at most %d)",
                    n_samples, static_cast<int>((max_smem - 8 * kHilRoots) / 24 * 32 / 33));
    }
    int roots = 0;
    for (int s = 0; s < g.n_stages; ++s) roots += (g.radix[s] & 1) && g.radix[s] <= 16 ? g.radix[s] : 0;
    if (roots > kHilRoots) return fail(MACH_B200_ERR_VALUE, "n_samples %u has too many odd factors", n_samples);
    const int64_t n_cols = static_cast<int64_t>(n_elements) * n_waves * n_frames;
    // 2, 4, 8 or 16 columns per CTA: as many as keep two CTAs on an SM (113 KB each) with at
    // most 8192 samples per group (32 per thread, prefetched into registers), plus the group's
    // samples in shared memory (xs) for the output phase when they fit.
    auto bytes_for = [&](int l, bool xs) { return col_bytes * (1ull << l) + fixed + (xs ? 4ull * g.n << l : 0); };
    int lc = 1;
    while (lc < 4 && bytes_for(lc + 1, true) <= (113ull << 10) && (static_cast<int64_t>(g.n) << (lc + 1)) <= 8192 &&
           (int64_t{1} << lc) < n_cols) {
        ++lc;
    }
    g.cols_log2 = lc;
    g.x_in_smem = bytes_for(lc, true) <= static_cast<uint64_t>(max_smem) ? 1 : 0;
    const size_t smem = static_cast<size_t>(bytes_for(lc, g.x_in_smem != 0));
    g.n_cols = n_cols;
    g.inv_n = 1.0f / static_cast<float>(g.n);
    g.scale = scale;
    const int64_t N = g.n, F = n_frames, E = n_elements, W = n_waves;
    g.n0 = F;
    if (src_layout == MACH_B200_LAYOUT_CHANNEL) {  // c = (w, e, f); [W][E][N][F] on both sides
        g.n1 = E;
        g.src_stride[0] = 1;
        g.src_stride[1] = N * F;
        g.src_stride[2] = E * N * F;
        g.src_sample = F;
    } else {  // c = (e, w, f); source [N][E][W][F]
        g.n1 = W;
        g.src_stride[0] = 1;
        g.src_stride[1] = F;
        g.src_stride[2] = W * F;
        g.src_sample = E * W * F;
    }
    g.dst_stride[0] = 1;
    g.dst_stride[1] = src_layout == MACH_B200_LAYOUT_CHANNEL ? N * F : E * N * F;  // e or w
    g.dst_stride[2] = src_layout == MACH_B200_LAYOUT_CHANNEL ? E * N * F : N * F;  // w or e
    g.dst_sample = F;
    g.load_cols_fast = g.src_sample != 1;
    g.store_cols_fast = g.dst_sample != 1;

    Residency r_src, r_dst;
    int rc;
    if ((rc = residency(src, device, &r_src, "src"))) return rc;
    if ((rc = residency(dst, device, &r_dst, "dst"))) return rc;
    if (r_dst != kOnDevice) return fail(MACH_B200_ERR_VALUE, "dst must be device memory");
    DeviceBuffer staged;
    g.src = src;
    if (r_src != kOnDevice) {
        const size_t bytes = count * storage_bytes(src_storage);
        MACH_B200_CUDA_TRY(staged.alloc(bytes, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(staged.ptr, src, bytes, cudaMemcpyHostToDevice, stream));
        g.src = staged.ptr;
    }
    g.dst = dst;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    MACH_B200_CUDA_TRY(launch_hilbert(src_storage, dst_storage, g, smem, stream));
    if (r_src != kOnDevice || !(flags & MACH_B200_FLAG_ASYNC)) MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
    return MACH_B200_OK;
}

// ---------------------------------------------------------------- allocation-free ensemble call
//
// mach_b200_beamform_ensemble_noalloc runs the ensemble kernel without allocating anything.
// The kernel's only scratch is one work-item counter per launch; here those counters live
// in this file's static device array instead of a stream-ordered allocation.

struct NoAllocState {
    std::once_flag once;
    cudaError_t init_error = cudaSuccess;
    int* counters = nullptr;  // device address of g_noalloc_counters
};
NoAllocState g_noalloc[kMaxDevices];

// First call on a device (that device current): the device address of the counters.  In host
// code g_noalloc_counters names a host-side stand-in, never the device memory itself.
int noalloc_counters(int device, int** out) {
    if (device < 0 || device >= kMaxDevices) return fail(MACH_B200_ERR_DEVICE, "device %d out of range", device);
    NoAllocState& d = g_noalloc[device];
    std::call_once(d.once, [&d]() {
        void* p = nullptr;
        d.init_error = cudaGetSymbolAddress(&p, g_noalloc_counters);
        d.counters = static_cast<int*>(p);
    });
    if (d.init_error != cudaSuccess) {
        return fail(MACH_B200_ERR_CUDA, "scratch setup failed: %s", cudaGetErrorString(d.init_error));
    }
    *out = d.counters;
    return MACH_B200_OK;
}

int noalloc_impl(int32_t storage, const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                 const float* tx_wave_arrivals_s, void* out, uint32_t n_tx, uint32_t n_rx, uint32_t n_samples,
                 uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                 float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha, int32_t interp_type,
                 float channel_scale, cudaStream_t stream, const mach_b200_options& opt) {
    g_error.clear();
    const uint32_t flags = opt.flags;
    int rc = check_args(storage, interp_type, tukey_alpha, n_tx, n_rx, n_samples, n_scan, n_frames);
    if (rc) return rc;
    if (flags & MACH_B200_FLAG_POWER_DOPPLER) {
        return fail(MACH_B200_ERR_VALUE, "the allocation-free call writes the beamformed frames, not a power image");
    }
    if (n_scan == 0 || n_frames == 0) return MACH_B200_OK;
    if (!out || !scan_coords_m) return fail(MACH_B200_ERR_VALUE, "out and scan_coords_m must not be NULL");
    const bool need_channel = n_tx > 0 && n_rx > 0 && n_samples > 0;
    if (need_channel && (!channel_data || !rx_coords_m || !tx_wave_arrivals_s)) {
        return fail(MACH_B200_ERR_VALUE, "channel_data, rx_coords_m and tx_wave_arrivals_s must not be NULL");
    }
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    DeviceState* dev = nullptr;
    if ((rc = device_state(device, &dev))) return rc;
    int* counters = nullptr;
    if ((rc = noalloc_counters(device, &counters))) return rc;
    const void* ptrs[5] = {channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out};
    const char* names[5] = {"channel_data", "rx_coords_m", "scan_coords_m", "tx_wave_arrivals_s", "out"};
    for (int i = 0; i < 5; ++i) {
        if (!ptrs[i]) continue;  // only optional inputs can be NULL here (checked above)
        Residency r;
        if ((rc = residency(ptrs[i], device, &r, names[i]))) return rc;
        if (r != kOnDevice) {
            return fail(MACH_B200_ERR_VALUE, "%s must be device memory: this call copies and allocates nothing",
                        names[i]);
        }
    }
    Plan plan;
    if (!plan_ensemble(storage, interp_type, n_scan, n_frames, n_tx, channel_data, true, opt, plan)) {
        return fail(MACH_B200_ERR_VALUE,
                    "this job does not fit the ensemble kernel: it needs nearest or linear interpolation, a "
                    "16-byte aligned channel_data, n_frames x sample bytes a multiple of 16 and fewer than 2^31 "
                    "voxels");
    }
    plan.st.status = dev->status;
    const bool cplx = (storage & 1) != 0;
    DasArgs a = make_args(rx_coords_m, scan_coords_m, n_scan, need_channel ? n_rx : 0, n_samples, n_frames, f_number,
                          rx_start_s, sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha,
                          channel_scale, cplx, flags);
    a.frame_passes = plan.lp.passes;
    a.tx_chunk = plan.lp.tx_chunk;
    a.channel = channel_data;
    a.arrivals = tx_wave_arrivals_s;
    a.out = out;
    a.n_tx = static_cast<int32_t>(need_channel ? n_tx : 0);
    a.accumulate = (flags & MACH_B200_FLAG_OVERWRITE) ? 0 : 1;

    // Launches of fewer than 2^31 channel samples each, one counter per launch.
    const size_t esz = storage_bytes(storage);
    const int64_t per_tx = static_cast<int64_t>(a.n_rx) * a.row_stride;
    const int total = a.n_tx;
    const TransmitSplit split = split_transmits(per_tx, total);
    if (split.n_launch > kNoAllocLaunches) {
        return fail(MACH_B200_ERR_VALUE,
                    "this job needs %lld launches; the allocation-free call holds work counters for %d (at most "
                    "%d x (2^31 - 1) channel samples)",
                    static_cast<long long>(split.n_launch), kNoAllocLaunches, kNoAllocLaunches);
    }
    MACH_B200_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(int) * static_cast<size_t>(split.n_launch), stream));
    const char* ch = static_cast<const char*>(a.channel);
    Plan pl = plan;
    for (int64_t k = 0; k < split.n_launch; ++k) {
        const int64_t t0 = launch_first_tx(split, k);
        DasArgs b = a;
        b.n_tx = static_cast<int32_t>(launch_tx_count(split, total, k));
        b.channel = ch + static_cast<size_t>(t0) * static_cast<size_t>(per_tx) * esz;
        b.arrivals = a.arrivals + t0 * a.n_vox;
        b.accumulate = t0 == 0 ? a.accumulate : 1;
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if (b.n_tx > 0) {
            if ((rc = encode_channel_map(&map, storage, b.channel, static_cast<uint64_t>(b.n_tx) * a.n_rx * a.n_samples,
                                         a.n_frames, plan.ea.box_x, plan.st.window_rows))) {
                return rc;
            }
        }
        pl.ea.counter = counters + k;
        MACH_B200_CUDA_TRY(dispatch(storage, b, interp_type, pl, map, stream));
    }
    if (!(flags & MACH_B200_FLAG_ASYNC)) {
        MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
        return check_status(dev, stream);
    }
    return MACH_B200_OK;
}

// ---------------------------------------------------------------- batches

}  // namespace

struct mach_b200_batch {
    int device = 0;
    uint32_t max_jobs = 0;
    static constexpr int kMaxGroups = 32;
    // pinned host tables (filled on the host, copied by the stream)
    BatchJob* h_jobs = nullptr;
    int64_t* h_begin = nullptr;
    BatchHeader* h_hdr = nullptr;
    // device tables
    BatchJob* d_jobs = nullptr;
    int64_t* d_begin = nullptr;
    BatchHeader* d_hdr = nullptr;
    unsigned long long* d_counters = nullptr;
    cudaEvent_t copied = nullptr;  // host tables may be rewritten once this has passed
    bool pending = false;
};

namespace {

struct GroupKey {
    int family;  // 0 lane-voxel, 1 staged, 2 frame-lane
    int storage;
    int interp;
    int variant;  // lane-voxel frame class (1, 0, 16) or staged lanes per voxel
    int split;
    bool operator==(const GroupKey& o) const {
        return family == o.family && storage == o.storage && interp == o.interp && variant == o.variant &&
               split == o.split;
    }
};

cudaError_t launch_group(const GroupKey& k, const PersistentLaunch& pl, cudaStream_t st) {
#define MACH_B200_GCASE(S)                                                                                   \
    case S:                                                                                                   \
        return k.family == 0   ? launch_lane_voxel_persistent<S>(k.interp, k.variant, k.split != 0, pl, st)   \
               : k.family == 2 ? launch_frame_lane_persistent<S>(k.interp, k.variant, k.split != 0, pl, st)   \
                               : launch_staged_persistent<S>(k.interp, k.variant, pl, st);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    switch (k.storage) {
        MACH_B200_GCASE(kF32)
        MACH_B200_GCASE(kC64)
        MACH_B200_GCASE(kF16)
        MACH_B200_GCASE(kCF16)
        MACH_B200_GCASE(kBF16)
        MACH_B200_GCASE(kCBF16)
        MACH_B200_GCASE(kI16)
        default:
            return k.family == 0   ? launch_lane_voxel_persistent<kCI16>(k.interp, k.variant, k.split != 0, pl, st)
                   : k.family == 2 ? launch_frame_lane_persistent<kCI16>(k.interp, k.variant, k.split != 0, pl, st)
                                   : launch_staged_persistent<kCI16>(k.interp, k.variant, pl, st);
    }
#undef MACH_B200_GCASE
}

void batch_free(mach_b200_batch* b) {
    if (!b) return;
    if (b->copied) {
        cudaEventSynchronize(b->copied);
        cudaEventDestroy(b->copied);
    }
    cudaFreeHost(b->h_jobs);
    cudaFreeHost(b->h_begin);
    cudaFreeHost(b->h_hdr);
    cudaFree(b->d_jobs);
    cudaFree(b->d_begin);
    cudaFree(b->d_hdr);
    cudaFree(b->d_counters);
    delete b;
}

int batch_create(uint32_t max_jobs, mach_b200_batch** out) {
    g_error.clear();
    if (!out) return fail(MACH_B200_ERR_VALUE, "batch pointer must not be NULL");
    *out = nullptr;
    if (max_jobs == 0 || max_jobs > (1u << 20)) return fail(MACH_B200_ERR_VALUE, "max_jobs must be in [1, 2^20]");
    auto* b = new mach_b200_batch();
    b->max_jobs = max_jobs;
    const size_t G = mach_b200_batch::kMaxGroups;
    cudaError_t e = cudaGetDevice(&b->device);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_jobs, sizeof(BatchJob) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_begin, sizeof(int64_t) * max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_hdr, sizeof(BatchHeader) * G);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, sizeof(BatchJob) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_begin, sizeof(int64_t) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_hdr, sizeof(BatchHeader) * G);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, sizeof(unsigned long long) * G);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        batch_free(b);
        return fail(MACH_B200_ERR_CUDA, "batch context allocation failed: %s", cudaGetErrorString(e));
    }
    *out = b;
    return MACH_B200_OK;
}

int batch_run(mach_b200_batch* b, const mach_b200_job* jobs, uint32_t n_jobs, cudaStream_t stream, uint32_t flags) {
    g_error.clear();
    if (!b) return fail(MACH_B200_ERR_VALUE, "batch context is NULL");
    if (n_jobs > b->max_jobs) return fail(MACH_B200_ERR_VALUE, "%u jobs exceed the context's %u", n_jobs, b->max_jobs);
    if (n_jobs && !jobs) return fail(MACH_B200_ERR_VALUE, "jobs must not be NULL");
    int device = 0;
    MACH_B200_CUDA_TRY(cudaGetDevice(&device));
    if (device != b->device) return fail(MACH_B200_ERR_DEVICE, "batch context belongs to device %d", b->device);
    DeviceState* dev = nullptr;
    int rc;
    if ((rc = device_state(device, &dev))) return rc;

    // The previous run's table copies read the pinned tables: wait before rewriting them.
    if (b->pending) {
        MACH_B200_CUDA_TRY(cudaEventSynchronize(b->copied));
        b->pending = false;
    }

    // ---- plan every job, assign it to a group (kernel signature)
    GroupKey keys[mach_b200_batch::kMaxGroups];
    int n_groups = 0;
    std::vector<int> group_of(n_jobs), order;
    std::vector<Plan> plans(n_jobs);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        const mach_b200_job& j = jobs[i];
        if ((rc = check_args(j.storage, j.interp_type, j.tukey_alpha, j.n_tx, j.n_rx, j.n_samples, j.n_scan,
                             j.n_frames))) {
            return fail(MACH_B200_ERR_VALUE, "job %u: %s", i, g_error.c_str());
        }
        if (static_cast<uint64_t>(j.n_tx) * j.n_rx * j.n_samples * j.n_frames >= (uint64_t{1} << 31)) {
            return fail(MACH_B200_ERR_VALUE, "job %u: channel data above 2^31 samples; use mach_b200_beamform_ex", i);
        }
        const void* ptrs[5] = {j.channel_data, j.rx_coords_m, j.scan_coords_m, j.tx_wave_arrivals_s, j.out};
        for (const void* p : ptrs) {
            Residency r;
            if (p && (rc = residency(p, device, &r, "a batch buffer"))) return rc;
            if (!p || r != kOnDevice) return fail(MACH_B200_ERR_VALUE, "job %u: batch buffers must be device memory", i);
        }
        mach_b200_options o = default_options(j.flags);
        std::memcpy(o.grid_shape, j.grid_shape, sizeof(o.grid_shape));
        o.kernel = j.kernel == MACH_B200_KERNEL_WARP ? MACH_B200_KERNEL_AUTO : j.kernel;
        o.tx_chunk = j.tx_chunk;
        o.window_rows = j.window_rows;
        o.lanes_per_voxel = j.lanes_per_voxel;
        plans[i] = plan_launch(j.storage, j.n_scan, j.n_frames, j.n_tx, j.channel_data, true, o, j.interp_type, true);
        const Plan& p = plans[i];
        GroupKey k{};
        if (p.frame_lane) {
            k = {2, j.storage, j.interp_type, p.lp.frame_slots, (j.flags & MACH_B200_FLAG_SPLIT_DELAY) ? 1 : 0};
        } else if (p.staged) {
            k = {1, j.storage, j.interp_type, p.lp.lanes_per_voxel, 0};
        } else if (p.lp.kind == kKindLaneVoxel1 || p.lp.kind == kKindLaneVoxelN || p.lp.kind == kKindLaneVoxel16 ||
                   p.lp.kind == kKindLaneVoxel8) {
            int fc = p.lp.kind == kKindLaneVoxel1 ? 1
                     : (p.lp.kind == kKindLaneVoxel16 ? 16 : (p.lp.kind == kKindLaneVoxel8 ? 8 : 0));
            if (fc == 1 && p.lp.lanes_per_voxel > 1) fc = 10 + p.lp.lanes_per_voxel;  // 12 / 14
            k = {0, j.storage, j.interp_type, fc, (j.flags & MACH_B200_FLAG_SPLIT_DELAY) ? 1 : 0};
        } else {
            return fail(MACH_B200_ERR_VALUE, "job %u: %u frames not a multiple of the storage's lane vector", i,
                        j.n_frames);
        }
        int gi = 0;
        while (gi < n_groups && !(keys[gi] == k)) ++gi;
        if (gi == n_groups) {
            if (n_groups == mach_b200_batch::kMaxGroups) return fail(MACH_B200_ERR_VALUE, "too many kernel signatures");
            keys[n_groups++] = k;
        }
        group_of[i] = gi;
    }

    // ---- fill the pinned tables, grouped
    std::vector<int> first(n_groups + 1, 0);
    for (uint32_t i = 0; i < n_jobs; ++i) ++first[group_of[i] + 1];
    for (int g = 0; g < n_groups; ++g) first[g + 1] += first[g];
    std::vector<int> fill(first.begin(), first.end() - 1);
    std::vector<size_t> smem(n_groups, 0);
    std::vector<int64_t> items(n_groups, 0);
    std::vector<int> max_items(n_groups, 0);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        const mach_b200_job& j = jobs[i];
        const int g = group_of[i];
        const int slot = fill[g]++;
        BatchJob& bj = b->h_jobs[slot];
        std::memset(&bj, 0, sizeof(bj));
        const bool cplx = (j.storage & 1) != 0;
        const bool need_channel = j.n_tx > 0 && j.n_rx > 0 && j.n_samples > 0;
        bj.a = make_args(j.rx_coords_m, j.scan_coords_m, j.n_scan, need_channel ? j.n_rx : 0, j.n_samples, j.n_frames,
                         j.f_number, j.rx_start_s, j.sampling_freq_hz, j.sound_speed_m_s, j.modulation_freq_hz,
                         j.tukey_alpha, j.channel_scale, cplx, j.flags);
        bj.a.channel = j.channel_data;
        bj.a.arrivals = j.tx_wave_arrivals_s;
        bj.a.out = j.out;
        bj.a.n_tx = static_cast<int32_t>(need_channel ? j.n_tx : 0);
        bj.a.accumulate = (j.flags & MACH_B200_FLAG_OVERWRITE) ? 0 : 1;
        const Plan& p = plans[i];
        bj.a.frame_passes = p.lp.passes;
        bj.a.tx_chunk = p.lp.tx_chunk;
        bj.a.map_fast = p.lp.map_fast;
        bj.a.map_wlog = p.lp.map_wlog;
        bj.a.tile_rev = p.lp.tile_rev;
        bj.a.map_outer = p.lp.map_outer;
        bj.a.frame_chunks = p.lp.frame_chunks;
        bj.st = p.st;
        bj.st.status = dev->status;
        bj.fl = p.fl;
        bj.tiles = static_cast<int32_t>(p.lp.grid.x);
        bj.chunks = static_cast<int32_t>(p.staged ? p.lp.grid.y : 1);
        if (p.staged && p.st.use_tma && bj.a.n_tx > 0) {
            const int fc = p.lp.lanes_per_voxel * static_cast<int>(8 / storage_bytes(j.storage));
            if ((rc = encode_channel_map(&bj.map, j.storage, j.channel_data,
                                         static_cast<uint64_t>(j.n_tx) * j.n_rx * j.n_samples, j.n_frames, fc,
                                         p.st.window_rows))) {
                return rc;
            }
        }
        const int64_t job_items = static_cast<int64_t>(bj.tiles) * bj.chunks;
        b->h_begin[slot] = items[g];
        items[g] += job_items;
        smem[g] = std::max(smem[g], p.lp.smem);
    }
    for (int g = 0; g < n_groups; ++g) {
        b->h_hdr[g].n_items = items[g];
        b->h_hdr[g].n_jobs = first[g + 1] - first[g];
        max_items[g] = static_cast<int>(std::min<int64_t>(items[g], 1 << 30));
    }

    // ---- copies, counters, one persistent launch per group
    if (n_jobs) {
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(BatchJob) * n_jobs, cudaMemcpyHostToDevice, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(b->d_begin, b->h_begin, sizeof(int64_t) * n_jobs, cudaMemcpyHostToDevice, stream));
        MACH_B200_CUDA_TRY(cudaMemcpyAsync(b->d_hdr, b->h_hdr, sizeof(BatchHeader) * n_groups, cudaMemcpyHostToDevice, stream));
        MACH_B200_CUDA_TRY(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned long long) * n_groups, stream));
        // While capturing a graph the copies run at replay time, from the tables as they are then.
        cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
        MACH_B200_CUDA_TRY(cudaStreamIsCapturing(stream, &capturing));
        if (capturing == cudaStreamCaptureStatusNone) {
            MACH_B200_CUDA_TRY(cudaEventRecord(b->copied, stream));
            b->pending = true;
        }
    }
    bool any_waits = false;  // staged kernels have bounded waits
    for (int g = 0; g < n_groups; ++g) {
        if (items[g] == 0) continue;
        PersistentLaunch pl{b->d_hdr + g, b->d_jobs + first[g], b->d_begin + first[g], b->d_counters + g, smem[g],
                            max_items[g]};
        any_waits |= keys[g].family == 1;
        MACH_B200_CUDA_TRY(launch_group(keys[g], pl, stream));
    }
    if (!(flags & MACH_B200_FLAG_ASYNC)) {
        MACH_B200_CUDA_TRY(cudaStreamSynchronize(stream));
        b->pending = false;
        if (any_waits) return check_status(dev, stream);
    }
    return MACH_B200_OK;
}
}  // namespace

extern "C" {

int mach_b200_beamform_f32(const float* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                           const float* tx_wave_arrivals_s, float* out, uint32_t n_rx, uint32_t n_samples,
                           uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                           float tukey_alpha, int32_t interp_type) {
    return compound_impl(kF32, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, 1u, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, 1.0f, nullptr, default_options(0u));
}

int mach_b200_beamform_c64(const void* channel_data, const float* rx_coords_m, const float* scan_coords_m,
                           const float* tx_wave_arrivals_s, void* out, uint32_t n_rx, uint32_t n_samples,
                           uint64_t n_scan, uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                           float tukey_alpha, int32_t interp_type) {
    return compound_impl(kC64, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, 1u, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, 1.0f, nullptr, default_options(0u));
}

int mach_b200_beamform_compound(int32_t storage, const void* channel_data, const float* rx_coords_m,
                                const float* scan_coords_m, const float* tx_wave_arrivals_s, void* out,
                                uint32_t n_tx, uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                                float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha,
                                int32_t interp_type, float channel_scale, void* cuda_stream, uint32_t flags) {
    return compound_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, channel_scale,
                         static_cast<cudaStream_t>(cuda_stream), default_options(flags));
}

int mach_b200_beamform_ex(int32_t storage, const void* channel_data, const float* rx_coords_m,
                          const float* scan_coords_m, const float* tx_wave_arrivals_s, void* out, uint32_t n_tx,
                          uint32_t n_rx, uint32_t n_samples, uint64_t n_scan, uint32_t n_frames, float f_number,
                          float rx_start_s, float sampling_freq_hz, float sound_speed_m_s, float modulation_freq_hz,
                          float tukey_alpha, int32_t interp_type, float channel_scale, void* cuda_stream,
                          const mach_b200_options* options) {
    mach_b200_options o = default_options(0u);
    if (options) {
        if (options->struct_size < offsetof(mach_b200_options, tx_model)) {
            g_error = "mach_b200_options.struct_size is too small";
            return MACH_B200_ERR_VALUE;
        }
        std::memcpy(&o, options, std::min<size_t>(sizeof(o), options->struct_size));
    }
    if (o.tx_model != MACH_B200_TX_ARRAYS) {
        g_error.clear();
        const int rc0 = check_args(storage, interp_type, tukey_alpha, n_tx, n_rx, n_samples, n_scan, n_frames);
        if (rc0) return rc0;
        TxArrivals t;  // freed in stream order when the call returns
        const int rc = form_tx_arrivals(o, scan_coords_m, n_tx, n_scan, sound_speed_m_s,
                                        static_cast<cudaStream_t>(cuda_stream), t);
        if (rc) return rc;
        o.tx_model = MACH_B200_TX_ARRAYS;
        tx_wave_arrivals_s = t.ptr;
        return compound_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                             n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                             modulation_freq_hz, tukey_alpha, interp_type, channel_scale,
                             static_cast<cudaStream_t>(cuda_stream), o);
    }
    return compound_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                         n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                         modulation_freq_hz, tukey_alpha, interp_type, channel_scale,
                         static_cast<cudaStream_t>(cuda_stream), o);
}

int mach_b200_beamform_ensemble_noalloc(int32_t storage, const void* channel_data, const float* rx_coords_m,
                                        const float* scan_coords_m, const float* tx_wave_arrivals_s, void* out,
                                        uint32_t n_tx, uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                        uint32_t n_frames, float f_number, float rx_start_s, float sampling_freq_hz,
                                        float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha,
                                        int32_t interp_type, float channel_scale, void* cuda_stream,
                                        const mach_b200_options* options) {
    mach_b200_options o = default_options(0u);
    if (options) {
        if (options->struct_size < offsetof(mach_b200_options, tx_model)) {
            g_error = "mach_b200_options.struct_size is too small";
            return MACH_B200_ERR_VALUE;
        }
        std::memcpy(&o, options, std::min<size_t>(sizeof(o), options->struct_size));
    }
    if (o.tx_model != MACH_B200_TX_ARRAYS) {
        g_error = "mach_b200_beamform_ensemble_noalloc takes an arrivals array (tx_model 0): a wave model would "
                  "need a device buffer for the arrivals";
        return MACH_B200_ERR_VALUE;
    }
    return noalloc_impl(storage, channel_data, rx_coords_m, scan_coords_m, tx_wave_arrivals_s, out, n_tx, n_rx,
                        n_samples, n_scan, n_frames, f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                        modulation_freq_hz, tukey_alpha, interp_type, channel_scale,
                        static_cast<cudaStream_t>(cuda_stream), o);
}

int mach_b200_ingest(int32_t src_storage, const void* src, int32_t dst_storage, void* dst, uint32_t n_samples,
                     uint32_t n_elements, uint32_t n_waves, uint32_t n_frames, float scale, void* cuda_stream,
                     uint32_t flags) {
    return ingest_impl(src_storage, src, dst_storage, dst, n_samples, n_elements, n_waves, n_frames, scale,
                       static_cast<cudaStream_t>(cuda_stream), flags);
}

int mach_b200_hilbert(int32_t src_storage, const void* src, int32_t src_layout, int32_t dst_storage, void* dst,
                      uint32_t n_samples, uint32_t n_elements, uint32_t n_waves, uint32_t n_frames, float scale,
                      void* cuda_stream, uint32_t flags) {
    return hilbert_impl(src_storage, src, src_layout, dst_storage, dst, n_samples, n_elements, n_waves, n_frames,
                        scale, static_cast<cudaStream_t>(cuda_stream), flags);
}

int mach_b200_batch_create(uint32_t max_jobs, mach_b200_batch** batch) { return batch_create(max_jobs, batch); }

int mach_b200_batch_run(mach_b200_batch* batch, const mach_b200_job* jobs, uint32_t n_jobs, void* cuda_stream,
                        uint32_t flags) {
    return batch_run(batch, jobs, n_jobs, static_cast<cudaStream_t>(cuda_stream), flags);
}

void mach_b200_batch_destroy(mach_b200_batch* batch) { batch_free(batch); }

int mach_b200_pool_stats(int32_t device, int32_t reset_high, uint64_t* used_high, uint64_t* reserved) {
    if (!used_high || !reserved) return fail(MACH_B200_ERR_VALUE, "used_high and reserved must not be NULL");
    if (device < 0 || device >= kMaxDevices) return fail(MACH_B200_ERR_DEVICE, "device %d out of range", device);
    *used_high = 0;
    *reserved = 0;
    cudaMemPool_t pool = g_devices[device].pool.load();
    if (pool == nullptr) return MACH_B200_OK;  // nothing allocated on this device yet
    if (reset_high) {
        uint64_t zero = 0;
        MACH_B200_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
    }
    MACH_B200_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, used_high));
    MACH_B200_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, reserved));
    return MACH_B200_OK;
}

const char* mach_b200_last_error(void) { return g_error.c_str(); }

const char* mach_b200_nvcc_version(void) { return MACH_B200_NVCC_VERSION; }

const char* mach_b200_version(void) { return MACH_B200_VERSION; }

uint64_t mach_b200_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
