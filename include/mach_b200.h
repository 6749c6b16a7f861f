/*
 * mach_b200 -- C ABI of the B200 delay-and-sum beamformer.
 *
 * Plain pointers, sizes and scalars only.  Every pointer may be device memory
 * (cudaMalloc / managed) or host memory (pinned or pageable); host buffers are
 * staged through the GPU the way mach's binding stages CPU arrays
 * (src/mach/kernel.cu:1090-1208): host inputs are copied in, and a host `out`
 * is OVERWRITTEN with the result, while a device `out` is ACCUMULATED into
 * (src/mach/kernel.cu:675-680, 1135-1139, 1203-1205).
 *
 * Every function returns MACH_B200_OK (0) or an error code; the message of the
 * last failure on the calling thread is available from mach_b200_last_error().
 * No function terminates the process (mach's helper_cuda.h exits on CUDA errors).
 *
 * Kernels that wait on shared-memory barriers (staged and ensemble families) give up after
 * a bounded time and set one status word per device; a synchronous call reads and clears it
 * and fails with MACH_B200_ERR_CUDA.  The word is shared by all calls on a device, so a
 * timeout in an asynchronous call can be reported by the next synchronous call on any
 * stream of that device.  Temporary device buffers (host staging, work counters) come from
 * a memory pool of the library's own (at most 2 GiB of freed memory kept per device); the
 * process's default memory pool is never reconfigured.
 *
 * Layouts (C order):
 *   channel_data        [n_tx][n_rx][n_samples][n_frames] samples of `storage`
 *   rx_coords_m         [n_rx][3]   float32, metres
 *   scan_coords_m       [n_scan][3] float32, metres
 *   tx_wave_arrivals_s  [n_tx][n_scan] float32, seconds
 *   out                 [n_scan][n_frames] float32 (real storage) or complex64 (complex storage)
 */
#ifndef MACH_B200_H_
#define MACH_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MACH_B200_API __attribute__((visibility("default")))
#else
#define MACH_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MACH_B200_OK 0
#define MACH_B200_ERR_VALUE 1 /* bad argument: shape, range, dtype (mach raises RuntimeError) */
#define MACH_B200_ERR_CUDA 2  /* a CUDA runtime call failed */
#define MACH_B200_ERR_DEVICE 3 /* pointer on another device than the current one */

/* Interpolation (mach InterpolationType, src/mach/kernel.cu:25-29). */
#define MACH_B200_NEAREST 0
#define MACH_B200_LINEAR 1
#define MACH_B200_QUADRATIC 2

/* Channel-data storage.  Odd codes are complex (I, Q) pairs.  All arithmetic is FP32. */
#define MACH_B200_STORAGE_F32 0   /* float32 RF (mach's float overload) */
#define MACH_B200_STORAGE_C64 1   /* complex64 IQ (mach's complex64 overload) */
#define MACH_B200_STORAGE_F16 2   /* binary16 RF */
#define MACH_B200_STORAGE_CF16 3  /* binary16 IQ pairs */
#define MACH_B200_STORAGE_BF16 4  /* bfloat16 RF */
#define MACH_B200_STORAGE_CBF16 5 /* bfloat16 IQ pairs */
#define MACH_B200_STORAGE_I16 6   /* int16 RF, value = sample * channel_scale */
#define MACH_B200_STORAGE_CI16 7  /* int16 IQ pairs, value = sample * channel_scale */

/* Flags for mach_b200_beamform_compound / mach_b200_beamform_ex. */
#define MACH_B200_FLAG_ASYNC 1u     /* return without synchronising `cuda_stream` (device buffers only) */
#define MACH_B200_FLAG_OVERWRITE 2u /* out = result instead of out += result */
#define MACH_B200_FLAG_SPLIT_DELAY 4u /* sample positions and phases formed in FP64 per receive path and
                                         per transmit, combined as integer base + FP32 fraction (more
                                         accurate than mach's FP32 delay; not bit-identical to mach) */
#define MACH_B200_FLAG_POWER_DOPPLER 8u /* out is float32 [n_scan]: the power-Doppler image, the sum over
                                           frames of |beamformed value|^2 (the step after the beamformer
                                           in mach's examples/doppler.py:252), fused into the kernel where
                                           it can be; only the compound / _ex entry points take it */

/* Kernel families (mach_b200_options.kernel). */
#define MACH_B200_KERNEL_AUTO 0
#define MACH_B200_KERNEL_LANE_VOXEL 1 /* one lane per voxel, all frames in registers (1..8 frames) */
#define MACH_B200_KERNEL_STAGED 2     /* voxel tiles, sample windows staged in shared memory by TMA */
#define MACH_B200_KERNEL_WARP 3       /* a warp per voxel over frames, taps read from global memory */
#define MACH_B200_KERNEL_ENSEMBLE 4   /* lanes = frames of a 32-lane block, voxel-tile sample windows in
                                         tensor memory (many frames; nearest or linear taps) */
#define MACH_B200_KERNEL_FRAME_LANE 5 /* lanes = frames, a warp walks a run of neighbouring voxels
                                         and loads each element's sample rows once for all of them
                                         (many frames; nearest or linear taps) */

/*
 * Optional launch options.  Zero-initialise, set struct_size = sizeof(mach_b200_options),
 * then set what you need.  The launch fields only affect speed, never the result; tx_model
 * and tx_params replace the arrivals array by its plane / spherical wave model.
 */
typedef struct mach_b200_options {
    uint32_t struct_size;   /* sizeof(mach_b200_options) */
    uint32_t flags;         /* MACH_B200_FLAG_* */
    int32_t grid_shape[3];  /* scan_coords_m as a C-order grid (slow, mid, fast), fast = contiguous
                               axis (e.g. (nx, 1, nz) for a meshgrid(x, [y0], z, indexing="ij")
                               flattened); zeros = no grid: tiles are runs of consecutive voxels */
    int32_t kernel;          /* MACH_B200_KERNEL_*, 0 = automatic */
    int32_t tx_chunk;        /* lane-voxel kernel: transmits per shared-memory pass, 0 = automatic */
    int32_t window_rows;     /* staged / ensemble kernels: sample rows per window, 0 = automatic */
    int32_t lanes_per_voxel; /* staged kernel: 4, 8, 16 or 32; one-frame voxel-per-lane kernel: 1, 2
                                or 4 lanes per voxel, each summing every 2nd / 4th element;
                                0 = automatic */
    int32_t tx_model;        /* MACH_B200_TX_ARRAYS: read tx_wave_arrivals_s; MACH_B200_TX_PLANE /
                                MACH_B200_TX_SPHERICAL: every (point, transmit) arrival is formed on the
                                device from tx_params, by one kernel into a temporary [n_tx][n_scan]
                                device array (tx_wave_arrivals_s may then be NULL) */
    int32_t tile_fast;       /* lane-voxel kernels on a known grid: voxels a warp takes along the
                                contiguous axis (1, 2, 4, 8 or 16; the rest of its 32 along the next
                                axis), 0 = automatic */
    const double* tx_params; /* [n_tx][8]: origin xyz (m), unit direction (plane) or focus xyz (m)
                                (spherical), time offset (s), unused.  The arrival is the distance of
                                src/mach/wavefront.py:8-116 divided by the sound speed, plus the
                                offset, formed in FP64 and rounded to FP32.  Device or host memory. */
    int32_t frame_slots;     /* frame-lane kernel: columns of 32 lane words (frames) a warp holds, 1, 2
                                or 4, with runs of 16, 8 or 4 voxels; 0 = automatic */
    int32_t element_block;   /* voxel-per-lane kernels: elements per launch (the job runs as one launch
                                per block of elements, accumulating), so that a launch's channel data
                                stays in L2; 0 = automatic (blocks of about 80 MB of channel data for
                                16-frame jobs above 126 MB), -1 or >= n_rx = one launch */
    int32_t tile_order;      /* voxel-per-lane kernels on a known grid: 1 = CTAs take the tiles at the far
                                end of the contiguous axis first (the deepest first for a depth-fastest
                                scan: widest aperture, most work, so a launch ends on light tiles),
                                2 = grid order; 0 = automatic (1, except 16-frame jobs) */
} mach_b200_options;

/* Transmit models (mach_b200_options.tx_model). */
#define MACH_B200_TX_ARRAYS 0
#define MACH_B200_TX_PLANE 1
#define MACH_B200_TX_SPHERICAL 2

/*
 * Single-transmit DAS on float32 RF, synchronous on the legacy default stream.
 * Replaces the float32 overload of mach._cuda_impl.beamform
 * (src/mach/kernel.cu:1242-1255, body 1032-1209; stub src/mach/_cuda_impl.pyi:39-53).
 */
MACH_B200_API int mach_b200_beamform_f32(const float* channel_data, const float* rx_coords_m,
                           const float* scan_coords_m, const float* tx_wave_arrivals_s,
                           float* out, uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                           uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s,
                           float modulation_freq_hz, float tukey_alpha, int32_t interp_type);

/*
 * Single-transmit DAS on complex64 IQ (interleaved float pairs), synchronous on the
 * legacy default stream.  Replaces the complex64 overload of mach._cuda_impl.beamform
 * (src/mach/kernel.cu:1229-1241, body 1032-1209; stub src/mach/_cuda_impl.pyi:24-38).
 */
MACH_B200_API int mach_b200_beamform_c64(const void* channel_data, const float* rx_coords_m,
                           const float* scan_coords_m, const float* tx_wave_arrivals_s,
                           void* out, uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                           uint32_t n_frames, float f_number, float rx_start_s,
                           float sampling_freq_hz, float sound_speed_m_s,
                           float modulation_freq_hz, float tukey_alpha, int32_t interp_type);

/*
 * Coherent compounding over n_tx transmits in ONE launch, any storage type, on
 * `cuda_stream` (a cudaStream_t; NULL = legacy default stream).  Replaces the
 * per-transmit loop of mach.experimental.beamform (src/mach/experimental.py:23-108,
 * loop 80-97), which launches and synchronises once per transmit.  With host
 * inputs the transmits are copied in chunks on a second stream while earlier
 * chunks compute.  Synchronous unless MACH_B200_FLAG_ASYNC is set and every
 * buffer is device memory.
 */
MACH_B200_API int mach_b200_beamform_compound(int32_t storage, const void* channel_data,
                                const float* rx_coords_m, const float* scan_coords_m,
                                const float* tx_wave_arrivals_s, void* out, uint32_t n_tx,
                                uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                uint32_t n_frames, float f_number, float rx_start_s,
                                float sampling_freq_hz, float sound_speed_m_s,
                                float modulation_freq_hz, float tukey_alpha,
                                int32_t interp_type, float channel_scale, void* cuda_stream,
                                uint32_t flags);

/*
 * mach_b200_beamform_compound with launch options (grid hint and tuning knobs chosen by
 * the autotuner).  `options` may be NULL.  Same semantics and errors as the compound call.
 */
MACH_B200_API int mach_b200_beamform_ex(int32_t storage, const void* channel_data,
                                const float* rx_coords_m, const float* scan_coords_m,
                                const float* tx_wave_arrivals_s, void* out, uint32_t n_tx,
                                uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                uint32_t n_frames, float f_number, float rx_start_s,
                                float sampling_freq_hz, float sound_speed_m_s,
                                float modulation_freq_hz, float tukey_alpha,
                                int32_t interp_type, float channel_scale, void* cuda_stream,
                                const mach_b200_options* options);

/*
 * mach_b200_beamform_ex restricted to the ensemble kernel (MACH_B200_KERNEL_ENSEMBLE), for
 * callers that must not allocate GPU memory: a host that pre-reserves all of HBM for its own
 * allocator, or a real-time acquisition loop that cannot risk a pool growing (and stalling)
 * inside a call.  The ensemble kernel's only scratch, one work-item counter per launch, lives
 * in a static device array of the library (64 counters, 256 bytes on every device that loads
 * it) instead of a stream-ordered allocation: the call allocates no device memory, creates no
 * memory pool and changes no pool setting.  Its only copy is the read-back of the library's
 * 4-byte timeout status word on synchronous calls (and its reset after a timeout).
 * No counterpart in the reference (mach allocates staging buffers and runs one fixed kernel).
 *
 * - Every buffer must be device memory of the current device (host buffers are rejected, as
 *   they would need staging buffers).  The job must fit the ensemble kernel (nearest or linear
 *   interpolation, 16-byte aligned channel_data, n_frames x sample bytes a multiple of 16,
 *   fewer than 2^31 voxels) and need at most 64 launches, i.e. at most 64 x (2^31 - 1)
 *   channel samples; anything else is rejected with MACH_B200_ERR_VALUE.
 *   It takes an arrivals array only: options->tx_model must be MACH_B200_TX_ARRAYS, since a
 *   wave model is turned into arrivals in a device buffer.
 * - The first call on a device looks up the counters' device address; make that first call
 *   before any stream capture.
 * - All calls share the counters (each call zeroes the ones it uses on `cuda_stream`), so two
 *   calls whose work overlaps on the GPU (different streams, or MACH_B200_FLAG_ASYNC calls not
 *   yet finished on other streams) race and give wrong images.  Serialise them.
 * - Arguments and result as mach_b200_beamform_ex with the ensemble kernel, except that
 *   MACH_B200_FLAG_POWER_DOPPLER is rejected (this call writes the frames).
 */
MACH_B200_API int mach_b200_beamform_ensemble_noalloc(int32_t storage, const void* channel_data,
                                const float* rx_coords_m, const float* scan_coords_m,
                                const float* tx_wave_arrivals_s, void* out, uint32_t n_tx,
                                uint32_t n_rx, uint32_t n_samples, uint64_t n_scan,
                                uint32_t n_frames, float f_number, float rx_start_s,
                                float sampling_freq_hz, float sound_speed_m_s,
                                float modulation_freq_hz, float tukey_alpha,
                                int32_t interp_type, float channel_scale, void* cuda_stream,
                                const mach_b200_options* options);

/*
 * Channel-data ingest: acquisition order [n_samples][n_elements][n_waves][n_frames] (UFF and
 * PyMUST order) to the beamformer's [n_waves][n_elements][n_samples][n_frames], converted from
 * storage `src_storage` to `dst_storage` in the same pass (value x `scale`, rounded to the
 * destination type; int16 destinations saturate).  Both storages must be real or both
 * complex (complex: interleaved (I, Q)).  Replaces the einops rearrange and dtype cast of
 * src/mach/io/uff.py:70-105 and examples/doppler.py:193-195.  `dst` must be device memory;
 * a host `src` is copied to the device first.  Synchronous unless MACH_B200_FLAG_ASYNC is set
 * and both buffers are device memory.
 */
MACH_B200_API int mach_b200_ingest(int32_t src_storage, const void* src, int32_t dst_storage, void* dst,
                                   uint32_t n_samples, uint32_t n_elements, uint32_t n_waves,
                                   uint32_t n_frames, float scale, void* cuda_stream, uint32_t flags);

/* Layouts of the real channel data given to mach_b200_hilbert. */
#define MACH_B200_LAYOUT_CHANNEL 0     /* [n_waves][n_elements][n_samples][n_frames] */
#define MACH_B200_LAYOUT_ACQUISITION 1 /* [n_samples][n_elements][n_waves][n_frames] (UFF, PyMUST) */

/*
 * RF -> IQ by the analytic signal: dst = x + i H{x} along the sample axis of real channel data,
 * the result of scipy.signal.hilbert(x, axis=samples) (src/mach/io/uff.py:88, mach's front end
 * for modulation frequency 0; beamform the result with modulation_freq_hz = 0).  `src` is real
 * storage (F32, F16, BF16, I16) in `src_layout`; `dst` is complex storage (C64, CF16, CBF16,
 * CI16; interleaved (I, Q)) in the channel layout [n_waves][n_elements][n_samples][n_frames],
 * so MACH_B200_LAYOUT_ACQUISITION also does the rearrange of src/mach/io/uff.py:101-102.  Both
 * parts are multiplied by `scale` before rounding (int16 saturates).  Transforms are computed
 * in FP32 with exact twiddles; n_samples is at most (227 KB / 24 bytes) on B200.  `dst` must be
 * device memory and must not overlap `src`; a host `src` is copied to the device first.
 * Synchronous unless MACH_B200_FLAG_ASYNC is set and `src` is device memory.
 */
MACH_B200_API int mach_b200_hilbert(int32_t src_storage, const void* src, int32_t src_layout,
                                    int32_t dst_storage, void* dst, uint32_t n_samples,
                                    uint32_t n_elements, uint32_t n_waves, uint32_t n_frames,
                                    float scale, void* cuda_stream, uint32_t flags);

/* One job of a batch: every pointer must be device memory of the current device. */
typedef struct mach_b200_job {
    int32_t storage;             /* MACH_B200_STORAGE_* */
    int32_t interp_type;         /* MACH_B200_NEAREST / LINEAR / QUADRATIC */
    const void* channel_data;    /* [n_tx][n_rx][n_samples][n_frames] */
    const float* rx_coords_m;    /* [n_rx][3] */
    const float* scan_coords_m;  /* [n_scan][3] */
    const float* tx_wave_arrivals_s; /* [n_tx][n_scan] */
    void* out;                   /* [n_scan][n_frames] */
    uint32_t n_tx, n_rx, n_samples, n_frames;
    uint64_t n_scan;
    float f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha;
    float channel_scale;
    uint32_t flags;              /* MACH_B200_FLAG_OVERWRITE, MACH_B200_FLAG_SPLIT_DELAY */
    int32_t grid_shape[3];       /* as in mach_b200_options */
    int32_t kernel;              /* tuning knobs as in mach_b200_options (0 = automatic);      */
    int32_t tx_chunk;            /* MACH_B200_KERNEL_WARP is not available in batches          */
    int32_t window_rows;
    int32_t lanes_per_voxel;
} mach_b200_job;

/* Reusable batch context: pinned host and device job tables, work counters. */
typedef struct mach_b200_batch mach_b200_batch;

/* Create a context for batches of up to max_jobs jobs on the current device. */
MACH_B200_API int mach_b200_batch_create(uint32_t max_jobs, mach_b200_batch** batch);

/*
 * Beamform a batch of device-resident jobs with one persistent launch per kernel
 * signature (storage, interpolation, kernel family): the resident CTAs pull (job, tile)
 * work items from a device counter until every tile of every job is done, so jobs of
 * different grid sizes, transmit and frame counts share the GPU.  Only asynchronous
 * copies (job table, from the context's pinned buffer), memsets and launches are
 * enqueued on `cuda_stream`, so the call can be captured in a CUDA graph and replayed
 * (replays reuse the captured job table).  mach has no batch interface (its call
 * beamforms one transmit of one job), so this entry point has no counterpart there.
 * `flags`: MACH_B200_FLAG_ASYNC to return without synchronising.
 */
MACH_B200_API int mach_b200_batch_run(mach_b200_batch* batch, const mach_b200_job* jobs, uint32_t n_jobs,
                                      void* cuda_stream, uint32_t flags);

/* Release a batch context (waits for its device work to finish). */
MACH_B200_API void mach_b200_batch_destroy(mach_b200_batch* batch);

/*
 * Measurement helper with no counterpart in the reference: launch, on `cuda_stream`, one
 * kernel that reads `bytes` of the device buffer `buffer` (16-byte aligned, a multiple of 16
 * bytes) `passes` times with L2-cached, L1-bypassing 16-byte loads, spread over every SM.
 * Timed with CUDA events around the launch (after one untimed launch), bytes x passes /
 * time is the L2 read bandwidth when the buffer is smaller than L2: the peak that the gather
 * kernels' L2 traffic is reported against.  Returns MACH_B200_ERR_VALUE for a host, foreign-
 * device or misaligned buffer.
 */
MACH_B200_API int mach_b200_probe_l2_read(const void* buffer, uint64_t bytes, uint32_t passes, void* cuda_stream);

/*
 * Diagnostic with no counterpart in the reference: the library's own memory pool on CUDA
 * device `device` (zeros while the library has not allocated anything there).  *used_high is
 * the most pool memory in use at once since the last reset, *reserved the memory the pool
 * holds now.  reset_high != 0 first resets the high-water mark to the memory in use now.
 */
MACH_B200_API int mach_b200_pool_stats(int32_t device, int32_t reset_high, uint64_t* used_high, uint64_t* reserved);

/* Message of the last failed call on this thread ("" if none). */
MACH_B200_API const char* mach_b200_last_error(void);

/* nvcc version the library was built with, "X.Y.Z" (mach's __nvcc_version__,
 * src/mach/kernel.cu:1215). */
MACH_B200_API const char* mach_b200_nvcc_version(void);

/* Library version string. */
MACH_B200_API const char* mach_b200_version(void);

/* Number of kernels this library has launched since it was loaded. */
MACH_B200_API uint64_t mach_b200_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* MACH_B200_H_ */
