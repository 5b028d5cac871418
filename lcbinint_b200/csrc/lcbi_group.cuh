// Cooperative groups of W warps for the finite-source scans.
//
// W = 1: every warp of the block is its own group (ordinary points, one warp
// each).  W > 1: the whole block (W warps) is one group and works on one point
// at a time (the few points with millions of cells).  Control flow is uniform
// across a group; per-lane results are combined into W-word ballot masks that
// every thread holds in registers.
#pragma once

#include "lcbi_warp.cuh"

namespace lcbi {

template <int W>
struct Grp {
    static constexpr int N = 32 * W;  // lanes of the group
    __device__ static int rank() { return W == 1 ? lane_id() : (int)threadIdx.x; }
    __device__ static int warp() { return W == 1 ? 0 : warp_in_block(); }
    __device__ static void sync()
    {
        if (W == 1) __syncwarp();
        else __syncthreads();
    }
    __device__ static bool any(bool p)
    {
        if (W == 1) return __any_sync(kFull, p);
        return __syncthreads_or(p) != 0;
    }
};

// Shared words a group uses to exchange masks and scalars.  Masks go through a
// double buffer: every thread reads a mask right after the barrier that
// publishes it, so by the time a buffer is written again (two publications
// later) every reader has passed the barrier in between.
template <int W>
struct GroupShared {
    unsigned mask[2][2][W];
    long long i64[4];
    double f64[4];
    unsigned long long u64[W];
    long long s64[W];
};

// Ballots of p (and of q) over the group, as W words each, in every thread.
template <int W>
__device__ __forceinline__ void group_ballot2(GroupShared<W>& S, int& phase, bool p, bool q, unsigned* pw, unsigned* qw)
{
    const unsigned bp = __ballot_sync(kFull, p);
    const unsigned bq = __ballot_sync(kFull, q);
    if (W == 1) {
        pw[0] = bp;
        qw[0] = bq;
        return;
    }
    if (lane_id() == 0) {
        S.mask[phase][0][warp_in_block()] = bp;
        S.mask[phase][1][warp_in_block()] = bq;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < W; ++w) {
        pw[w] = S.mask[phase][0][w];
        qw[w] = S.mask[phase][1][w];
    }
    phase ^= 1;
}

template <int W>
__device__ __forceinline__ void group_ballot(GroupShared<W>& S, int& phase, bool p, unsigned* pw)
{
    const unsigned bp = __ballot_sync(kFull, p);
    if (W == 1) {
        pw[0] = bp;
        return;
    }
    if (lane_id() == 0) S.mask[phase][0][warp_in_block()] = bp;
    __syncthreads();
#pragma unroll
    for (int w = 0; w < W; ++w) pw[w] = S.mask[phase][0][w];
    phase ^= 1;
}

// Index of the first set bit at or after `from` in the W-word mask m, or 32 W.
template <int W>
__device__ __forceinline__ int first_set(const unsigned* m, int from)
{
    const int fw = from >> 5;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        if (w < fw) continue;
        const unsigned x = m[w] & ((w == fw) ? (kFull << (from & 31)) : kFull);
        if (x) return (w << 5) + __ffs(x) - 1;
    }
    return 32 * W;
}

// Value of rank 0 in every thread of the group.
// Also orders the global-memory writes rank 0 made before the call ahead of
// every later read by the group.
template <int W>
__device__ __forceinline__ long long group_bcast(GroupShared<W>& S, long long v)
{
    if (W == 1) {
        __syncwarp();
        return __shfl_sync(kFull, v, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) S.i64[0] = v;
    __syncthreads();
    return S.i64[0];
}

// Exact fixed-point accumulation of FP64 terms: value = hi + lo * 2^-64 as a
// two's-complement 128-bit integer.  Integer addition is associative, so a
// sum formed lane by lane and then reduced across the group is the same in
// every run and for every group width; the only rounding is that of each
// term below 2^-64 and the final conversion back to FP64.
struct Fixed128 {
    unsigned long long lo;
    long long hi;
};

__device__ __forceinline__ void fx_add(Fixed128& a, unsigned long long lo, long long hi)
{
    const unsigned long long s = a.lo + lo;
    a.hi += hi + (s < lo ? 1 : 0);
    a.lo = s;
}

__device__ __forceinline__ void fx_add_double(Fixed128& a, double v)
{
    const double f = floor(v);
    const double frac = v - f;  // exact, in [0, 1)
    fx_add(a, __double2ull_rn(frac * 18446744073709551616.0), static_cast<long long>(f));
}

__device__ __forceinline__ double fx_to_double(const Fixed128& a)
{
    return static_cast<double>(a.hi) + static_cast<double>(a.lo) * (1.0 / 18446744073709551616.0);
}

// Sum of every thread's accumulator, in every thread of the group.
template <int W>
__device__ __forceinline__ Fixed128 group_fx_sum(GroupShared<W>& S, Fixed128 a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long lo = __shfl_xor_sync(kFull, a.lo, o);
        const long long hi = __shfl_xor_sync(kFull, a.hi, o);
        fx_add(a, lo, hi);
    }
    if (W == 1) return a;
    __syncthreads();
    if (lane_id() == 0) {
        S.u64[warp_in_block()] = a.lo;
        S.s64[warp_in_block()] = a.hi;
    }
    __syncthreads();
    Fixed128 t{0ull, 0ll};
    for (int w = 0; w < W; ++w) fx_add(t, S.u64[w], S.s64[w]);
    __syncthreads();
    return t;
}

} // namespace lcbi
