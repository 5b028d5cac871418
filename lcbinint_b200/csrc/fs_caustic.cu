// Caustic sampling and limb-darkening tables.
//
// caustic_roots_kernel   one thread per (model, phase): the quartic critical-curve
//                        roots and their source-plane images (ensure_binary_caustic_cache,
//                        finite_source_magnifier.cpp:4030-4041).
// caustic_track_kernel   one warp per model: bounding box, branch tracking by the
//                        minimum-cost permutation over 4! assignments
//                        (append_tracked_caustic_points, :569-611) and the longest
//                        non-wrapping segment (:4072-4098).
// ld_table_kernel        the 20,001-entry nearest-neighbour table of I(r^2) (:3979-3999).
#include "lcbi_fs.cuh"
#include "lcbi_fs_kernels.h"
#include "lcbi_warp.cuh"

namespace lcbi {

__global__ void ld_table_kernel(const double2* __restrict__ coeffs, int n_tables, double* tables)
{
    const int total = n_tables * (kLdTable + 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int k = t / (kLdTable + 1);
        const int i = t - k * (kLdTable + 1);
        const double2 cd = coeffs[k];
        tables[t] = surface_brightness(static_cast<double>(i) / static_cast<double>(kLdTable), cd.x, cd.y);
    }
}

__global__ void __launch_bounds__(128) caustic_roots_kernel(const CausticModel* __restrict__ models, int n_models,
                                                           const double2* __restrict__ phases,
                                                           const long long* __restrict__ raw_offset, P2* raw,
                                                           const unsigned char* __restrict__ needed,
                                                           int critical_points)
{
    // Flattened (model, phase) index; models are laid out back to back.
    const int m = blockIdx.y;
    if (m >= n_models || (needed && !needed[m])) return;
    const CausticModel md = models[m];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < md.bins; i += gridDim.x * blockDim.x) {
        const double2 ph = phases[md.phase_offset + i];
        dc roots[4];
        critical_roots(md.s, md.q, dc{ph.x, ph.y}, roots);
        P2* out = raw + raw_offset[m] + 4ll * i;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            out[k] = critical_points ? P2{roots[k].re, roots[k].im} : lens_equation_complex(md.s, md.q, roots[k]);
    }
}

// Lexicographic rank -> permutation of {0,1,2,3} (the order std::next_permutation
// visits starting from the identity).
__device__ __forceinline__ void perm_of_rank(int r, int* p)
{
    int avail[4] = {0, 1, 2, 3};
    int fact[4] = {6, 2, 1, 1};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int k = r / fact[i];
        r -= k * fact[i];
        p[i] = avail[k];
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (j >= k) avail[j] = avail[j + 1];
    }
}

__device__ __forceinline__ bool angle_less(P2 l, P2 r) { return atan2(l.y, l.x) < atan2(r.y, r.x); }

// The 24 permutations of {0, 1, 2, 3} in lexicographic order (the order
// std::next_permutation visits from the identity), packed two bits per entry:
// entry b of permutation r is (kPermCode[r] >> 2b) & 3.
__constant__ unsigned char kPermCode[24] = {228, 180, 216, 120, 156, 108, 225, 177, 201, 57, 141, 45,
                                            210, 114, 198, 54,  78,  30,  147, 99,  135, 39, 75,  27};

// Branch tracking of four models per warp, eight lanes per model: each lane
// costs three of the 24 permutations (ranks 3g .. 3g + 2), the first least
// cost over the model's eight lanes comes from a three-step butterfly on
// (cost, rank), and the group's lanes share their own shuffles and barriers,
// so the four models of a warp run independently.
constexpr int kTrackLanes = 8;
constexpr int kTrackPerLane = 24 / kTrackLanes;
constexpr int kTrackGroups = 32 / kTrackLanes;
constexpr int kTrackWarps = 4;                                  // warps per block
constexpr int kTrackBatch = 16;                                 // steps staged per batch
constexpr int kTrackLoads = 4 * kTrackBatch / kTrackLanes;      // points each lane loads per batch

__global__ void __launch_bounds__(32 * kTrackWarps) caustic_track_kernel(CausticModel* models, int n_models,
                                                                         const long long* __restrict__ raw_offset,
                                                                         const P2* __restrict__ raw,
                                                                         P2* __restrict__ branches,
                                                                         const unsigned char* __restrict__ needed)
{
    const int lane = lane_id();
    const int grp = lane / kTrackLanes;
    const int g = lane % kTrackLanes;
    const unsigned gmask = ((1u << kTrackLanes) - 1u) << (grp * kTrackLanes);
    const int m = (blockIdx.x * kTrackWarps + warp_in_block()) * kTrackGroups + grp;
    if (m >= n_models || (needed && !needed[m])) return;
    CausticModel md = models[m];
    const int bins = md.bins;
    const P2* pts = raw + raw_offset[m];
    P2* br = branches + md.branch_offset;

    // The permutations this lane costs.
    int perm[kTrackPerLane][4];
    unsigned code_of[kTrackPerLane];
#pragma unroll
    for (int j = 0; j < kTrackPerLane; ++j) {
        perm_of_rank(g * kTrackPerLane + j, perm[j]);
        code_of[j] = kPermCode[g * kTrackPerLane + j];
    }

    // Branch tracking: sample 0 sorted by polar angle, then each sample assigned
    // by the first minimum-cost permutation in lexicographic order.
    P2 end[4];
    double mnx, mxx, mny, mxy;
    {
        P2 v[4] = {pts[0], pts[1], pts[2], pts[3]};
        mnx = dmin_(dmin_(v[0].x, v[1].x), dmin_(v[2].x, v[3].x));
        mxx = dmax_(dmax_(v[0].x, v[1].x), dmax_(v[2].x, v[3].x));
        mny = dmin_(dmin_(v[0].y, v[1].y), dmin_(v[2].y, v[3].y));
        mxy = dmax_(dmax_(v[0].y, v[1].y), dmax_(v[2].y, v[3].y));
        for (int i = 1; i < 4; ++i) {
            const P2 x = v[i];
            int k = i;
            while (k > 0 && angle_less(x, v[k - 1])) {
                v[k] = v[k - 1];
                --k;
            }
            v[k] = x;
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) end[b] = v[b];
        if (g < 4) br[(long long)g * bins] = v[g];
    }
    // The samples are consumed strictly in order, one step (4 points) at a
    // time, and each step's assignment depends on the previous one; so the
    // points are staged in shared memory kTrackBatch steps at a time, the
    // next batch being loaded into registers while the current one is
    // consumed.  The loads also give the bounding box over every sampled
    // point (exact min/max, independent of the order).
    __shared__ P2 stage_all[kTrackWarps][kTrackGroups][4 * kTrackBatch];
    P2* stage = stage_all[warp_in_block()][grp];
    P2 nxt[kTrackLoads];
    auto load_batch = [&](int s0) {
        const long long first = 4ll * s0, last = 4ll * bins;
#pragma unroll
        for (int u = 0; u < kTrackLoads; ++u) {
            const long long j = first + g + kTrackLanes * u;
            if (j < last) {
                nxt[u] = pts[j];
                mnx = dmin_(mnx, nxt[u].x);
                mxx = dmax_(mxx, nxt[u].x);
                mny = dmin_(mny, nxt[u].y);
                mxy = dmax_(mxy, nxt[u].y);
            }
        }
    };
    double max_seg2 = 0.0;
    load_batch(1);
    for (int s0 = 1; s0 < bins; s0 += kTrackBatch) {
        const int s1 = min(bins, s0 + kTrackBatch);
        __syncwarp(gmask);
#pragma unroll
        for (int u = 0; u < kTrackLoads; ++u) {
            const int j = g + kTrackLanes * u;
            if (j < 4 * (s1 - s0)) stage[j] = nxt[u];
        }
        __syncwarp(gmask);
        if (s1 < bins) load_batch(s1);
        for (int i = s0; i < s1; ++i) {
            const P2* cur = stage + 4 * (i - s0);
            // This lane's first least cost; a cost that is not below +inf (NaN
            // included) competes as +inf, so with none below +inf rank 0 wins,
            // as in a serial scan with a strict comparison.
            double best = dinf();
            int bp = 64;
#pragma unroll
            for (int j = 0; j < kTrackPerLane; ++j) {
                double cost = 0.0;
#pragma unroll
                for (int b = 0; b < 4; ++b) cost += dist2(end[b], cur[perm[j][b]]);
                const double c = cost < dinf() ? cost : dinf();
                const int r = g * kTrackPerLane + j;
                if (c < best || (c == best && r < bp)) {
                    best = c;
                    bp = r;
                }
            }
#pragma unroll
            for (int off = kTrackLanes / 2; off > 0; off >>= 1) {
                const double ob = __shfl_xor_sync(gmask, best, off);
                const int op = __shfl_xor_sync(gmask, bp, off);
                if (ob < best || (ob == best && op < bp)) {
                    best = ob;
                    bp = op;
                }
            }
            const unsigned code = kPermCode[bp];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const P2 sel = cur[(code >> (2 * b)) & 3u];
                const double seg2 = dist2(end[b], sel);
                if (seg2 > max_seg2) max_seg2 = seg2;
                end[b] = sel;
            }
            if (g < 4) br[(long long)g * bins + i] = cur[(code >> (2 * g)) & 3u];
        }
    }
#pragma unroll
    for (int off = kTrackLanes / 2; off > 0; off >>= 1) {
        mnx = dmin_(mnx, __shfl_xor_sync(gmask, mnx, off));
        mxx = dmax_(mxx, __shfl_xor_sync(gmask, mxx, off));
        mny = dmin_(mny, __shfl_xor_sync(gmask, mny, off));
        mxy = dmax_(mxy, __shfl_xor_sync(gmask, mxy, off));
    }
    if (g == 0) {
        md.min_x = mnx;
        md.max_x = mxx;
        md.min_y = mny;
        md.max_y = mxy;
        const double width = dmax_(mxx - mnx, 1.0e-12);
        const double height = dmax_(mxy - mny, 1.0e-12);
        md.step_x = width / static_cast<double>(kCausticGrid);
        md.step_y = height / static_cast<double>(kCausticGrid);
        md.max_seg_len = sqrt(max_seg2);
        models[m] = md;
    }
}

cudaError_t launch_ld_tables(const double2* coeffs, int n_tables, double* tables, cudaStream_t stream)
{
    if (n_tables <= 0) return cudaSuccess;
    const int total = n_tables * (kLdTable + 1);
    ld_table_kernel<<<(total + 255) / 256, 256, 0, stream>>>(coeffs, n_tables, tables);
    return cudaGetLastError();
}

cudaError_t launch_caustics(CausticModel* models, int n_models, int max_bins, const double2* phases,
                            const long long* raw_offset, P2* raw, P2* branches, cudaStream_t stream,
                            const unsigned char* needed, bool critical_points)
{
    if (n_models <= 0) return cudaSuccess;
    dim3 grid((max_bins + 127) / 128, n_models);
    caustic_roots_kernel<<<grid, 128, 0, stream>>>(models, n_models, phases, raw_offset, raw, needed,
                                                   critical_points ? 1 : 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int per_block = kTrackWarps * kTrackGroups;
    caustic_track_kernel<<<(n_models + per_block - 1) / per_block, 32 * kTrackWarps, 0, stream>>>(
        models, n_models, raw_offset, raw, branches, needed);
    return cudaGetLastError();
}

} // namespace lcbi
