// Persistent batch kernels: one launch runs every tile of every job of one kernel signature.
//
// A batch is a table of jobs in device memory (copied from pinned host memory by the
// batch context, so a whole batch can be captured once in a CUDA graph and replayed).
// Work items are (job, tile[, frame chunk]) in job order; each resident CTA takes the next
// item from a device counter, looks up its job with a forward-only cursor (items grow
// monotonically per CTA), copies the job's arguments into shared memory and runs the same
// tile function as the per-job kernels.  Jobs of different sizes, frame counts and
// transmit counts share the launch; the GPU stays full until the last item.
#pragma once

#include "das_frame_lane.cuh"
#include "das_lane_voxel.cuh"
#include "das_staged.cuh"

namespace mach_b200 {

struct alignas(64) BatchJob {
    CUtensorMap map;  // staged family: TMA view of this job's channel data (64-byte aligned)
    DasArgs a;
    StagedArgs st;
    FrameLaneArgs fl;  // frame-lane family: run mapping and frame chunks
    int32_t tiles;   // spatial tiles (frame-lane family: CTA blocks)
    int32_t chunks;  // frame chunks per tile (staged family), 1 otherwise
};

struct BatchHeader {
    int64_t n_items;  // total work items of the group
    int32_t n_jobs;
    int32_t pad;
};

// Next work item for this CTA: thread 0 takes it from the counter and resolves the job.
// Returns false when the group is exhausted.
__device__ __forceinline__ bool next_item(const BatchHeader* hdr, const int64_t* item_begin,
                                          unsigned long long* counter, int& cursor, int* s_job, int64_t* s_local) {
    __syncthreads();  // everyone is done with the previous item's shared state
    if (threadIdx.x == 0) {
        const long long item = static_cast<long long>(atomicAdd(counter, 1ull));
        if (item >= hdr->n_items) {
            *s_job = -1;
        } else {
            while (cursor + 1 < hdr->n_jobs && item >= item_begin[cursor + 1]) ++cursor;
            *s_job = cursor;
            *s_local = item - item_begin[cursor];
        }
    }
    __syncthreads();
    return *s_job >= 0;
}

template <typename T>
__device__ __forceinline__ void copy_words(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(T) / 4); i += blockDim.x) d[i] = s[i];
}

template <int S, int INTERP, int NF, bool SPLIT, int CS = 1>
__global__ void __launch_bounds__(kLaneVoxelThreads, NF == 16 ? 4 : 8)
    das_lane_voxel_persistent(const BatchHeader* __restrict__ hdr, const BatchJob* __restrict__ jobs,
                              const int64_t* __restrict__ item_begin, unsigned long long* counter) {
    extern __shared__ float smem_words[];
    __shared__ DasArgs s_args;
    __shared__ int s_job;
    __shared__ int64_t s_local;
    int cursor = 0;
    while (next_item(hdr, item_begin, counter, cursor, &s_job, &s_local)) {
        copy_words(&s_args, &jobs[s_job].a);
        __syncthreads();
        if (NF >= 2 && s_args.frame_chunks > 1) {  // items: the 8-frame chunks of each tile
            const int64_t tile = s_local / s_args.frame_chunks;
            lane_voxel_tile<S, INTERP, NF, SPLIT, CS>(s_args, tile, smem_words,
                                                      static_cast<int>(s_local - tile * s_args.frame_chunks));
        } else {
            lane_voxel_tile<S, INTERP, NF, SPLIT, CS>(s_args, s_local, smem_words);
        }
    }
}

template <int S, int INTERP, int LV>
__global__ void __launch_bounds__(kStagedThreads, 3)
    das_staged_persistent(const BatchHeader* __restrict__ hdr, const BatchJob* __restrict__ jobs,
                          const int64_t* __restrict__ item_begin, unsigned long long* counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ DasArgs s_args;
    __shared__ StagedArgs s_st;
    __shared__ int s_job;
    __shared__ int64_t s_local;
    int cursor = 0;
    while (next_item(hdr, item_begin, counter, cursor, &s_job, &s_local)) {
        copy_words(&s_args, &jobs[s_job].a);
        copy_words(&s_st, &jobs[s_job].st);
        __syncthreads();
        const int chunks = jobs[s_job].chunks;
        const int tile = static_cast<int>(s_local / chunks);
        const int chunk = static_cast<int>(s_local - static_cast<int64_t>(tile) * chunks);
        if (!staged_tile<S, INTERP, LV>(s_args, s_st, &jobs[s_job].map, tile, chunk, smem)) return;
    }
}

template <int S, int INTERP, int J, bool SPLIT>
__global__ void __launch_bounds__(kFrameLaneThreads, 4)
    das_frame_lane_persistent(const BatchHeader* __restrict__ hdr, const BatchJob* __restrict__ jobs,
                              const int64_t* __restrict__ item_begin, unsigned long long* counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DasArgs s_args;
    __shared__ FrameLaneArgs s_fl;
    __shared__ int s_job;
    __shared__ int64_t s_local;
    int cursor = 0;
    while (next_item(hdr, item_begin, counter, cursor, &s_job, &s_local)) {
        copy_words(&s_args, &jobs[s_job].a);
        copy_words(&s_fl, &jobs[s_job].fl);
        __syncthreads();
        frame_lane_block<S, INTERP, J, 16 / J, SPLIT>(s_args, s_fl, s_local, smem_raw);
    }
}

}  // namespace mach_b200
