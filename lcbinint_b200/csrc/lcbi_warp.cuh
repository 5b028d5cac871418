// Warp-cooperative helpers.
//
// The finite-source kernels run one warp per work item.  Control flow that the
// reference executes serially (seed bookkeeping, row-scan state machine, BFS
// queue) is executed redundantly and uniformly by all 32 lanes; the expensive
// independent pieces (root solves, lens-map evaluations of consecutive cells)
// are spread across lanes and their results broadcast with shuffles.  Writes
// to shared state are done by lane 0 and published with __syncwarp().
#pragma once

#include <cuda_runtime.h>

namespace lcbi {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ int shfl_i(int v, int src) { return __shfl_sync(kFull, v, src); }

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(kFull, v, o);
        v = (w < v) ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(kFull, v, o);
        v = (v < w) ? w : v;
    }
    return v;
}

__device__ __forceinline__ int warp_sum_i(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Exclusive prefix count of a predicate across the warp.
__device__ __forceinline__ int prefix_count(unsigned ballot) { return __popc(ballot & ((1u << lane_id()) - 1u)); }

} // namespace lcbi
