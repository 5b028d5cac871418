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
                                                           const long long* __restrict__ raw_offset, P2* raw)
{
    // Flattened (model, phase) index; models are laid out back to back.
    const int m = blockIdx.y;
    if (m >= n_models) return;
    const CausticModel md = models[m];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < md.bins; i += gridDim.x * blockDim.x) {
        const double2 ph = phases[md.phase_offset + i];
        dc roots[4];
        critical_roots(md.s, md.q, dc{ph.x, ph.y}, roots);
        P2* out = raw + raw_offset[m] + 4ll * i;
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = lens_equation_complex(md.s, md.q, roots[k]);
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

__global__ void __launch_bounds__(32) caustic_track_kernel(CausticModel* models, int n_models,
                                                          const long long* __restrict__ raw_offset,
                                                          const P2* __restrict__ raw, P2* branches)
{
    const int m = blockIdx.x;
    if (m >= n_models) return;
    const int lane = lane_id();
    CausticModel md = models[m];
    const int bins = md.bins;
    const P2* pts = raw + raw_offset[m];
    P2* br = branches + md.branch_offset;

    // Bounding box over every sampled point (order-independent exact min/max).
    double mnx = dinf(), mxx = -dinf(), mny = dinf(), mxy = -dinf();
    for (int t = lane; t < 4 * bins; t += 32) {
        const P2 p = pts[t];
        mnx = dmin_(mnx, p.x);
        mxx = dmax_(mxx, p.x);
        mny = dmin_(mny, p.y);
        mxy = dmax_(mxy, p.y);
    }
    mnx = warp_min(mnx);
    mxx = warp_max(mxx);
    mny = warp_min(mny);
    mxy = warp_max(mxy);

    // Branch tracking: sample 0 sorted by polar angle, then each sample assigned
    // by the first minimum-cost permutation in lexicographic order.
    int perm[4];
    perm_of_rank(lane < 24 ? lane : 0, perm);
    P2 end[4];
    {
        P2 v[4] = {pts[0], pts[1], pts[2], pts[3]};
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
        if (lane < 4) br[(long long)lane * bins] = v[lane];
    }
    double max_seg2 = 0.0;
    for (int i = 1; i < bins; ++i) {
        const P2* cur = pts + 4ll * i;
        P2 c[4] = {cur[0], cur[1], cur[2], cur[3]};
        double cost = 0.0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            P2 sel = c[0];
#pragma unroll
            for (int k = 1; k < 4; ++k)
                if (perm[b] == k) sel = c[k];
            cost += dist2(end[b], sel);
        }
        double best = dinf();
        int bp = 0;
        for (int r = 0; r < 24; ++r) {
            const double cr = shfl_d(cost, r);
            if (cr < best) {
                best = cr;
                bp = r;
            }
        }
        int pb[4];
        perm_of_rank(bp, pb);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            P2 sel = c[0];
#pragma unroll
            for (int k = 1; k < 4; ++k)
                if (pb[b] == k) sel = c[k];
            const double seg2 = dist2(end[b], sel);
            if (seg2 > max_seg2) max_seg2 = seg2;
            end[b] = sel;
        }
        if (lane < 4) {
            P2 sel = c[0];
            for (int k = 1; k < 4; ++k)
                if (pb[lane] == k) sel = c[k];
            br[(long long)lane * bins + i] = sel;
        }
    }
    if (lane == 0) {
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
                            const long long* raw_offset, P2* raw, P2* branches, cudaStream_t stream)
{
    if (n_models <= 0) return cudaSuccess;
    dim3 grid((max_bins + 127) / 128, n_models);
    caustic_roots_kernel<<<grid, 128, 0, stream>>>(models, n_models, phases, raw_offset, raw);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    caustic_track_kernel<<<n_models, 32, 0, stream>>>(models, n_models, raw_offset, raw, branches);
    return cudaGetLastError();
}

} // namespace lcbi
