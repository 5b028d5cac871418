// Finite-source decision tree, one warp per evaluation
// (FiniteSourceMagnifier::binary_mag, finite_source_magnifier.cpp:4633-4843):
// caustic bounding-box exit, sampled and segment caustic distances, the
// point-source derivative check, the 13-solve hexadecapole (12 ring samples
// solved by 12 lanes at once) and the inverse-ray method choice.  Items that
// need inverse-ray integration are appended to the Cartesian or polar list.
#include "lcbi_caustic.cuh"
#include "lcbi_fs_kernels.h"

namespace lcbi {

namespace {

constexpr double kSqrtHalf = 0.70710678118654752440;

__device__ __forceinline__ void ring_sample(int k, double x, double y, double rho, double* px, double* py)
{
    // hexadecapole_binary sample order (FSM:807-820): for i in 0..3: +rho, +rho/2, x-rho.
    const double sineta[8] = {0.0, 1.0, 0.0, -1.0, kSqrtHalf, kSqrtHalf, -kSqrtHalf, -kSqrtHalf};
    const double coseta[8] = {1.0, 0.0, -1.0, 0.0, kSqrtHalf, -kSqrtHalf, -kSqrtHalf, kSqrtHalf};
    const int i = k / 3;
    const int j = k - 3 * i;
    if (j == 0) {
        *px = x + rho * coseta[i];
        *py = y + rho * sineta[i];
    } else if (j == 1) {
        *px = x + 0.5 * rho * coseta[i];
        *py = y + 0.5 * rho * sineta[i];
    } else {
        *px = x + rho * coseta[i + 4];
        *py = y + rho * sineta[i + 4];
    }
}

} // namespace

__global__ void __launch_bounds__(128) decide_kernel(FsWork w)
{
    const int lane = lane_id();
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int it = gw; it < w.n_items; it += nw) {
        const FsItem item = w.items[it];
        const FsSettingsDev st = w.settings[item.settings];
        const double s = item.s, q = item.q, x = item.x, y = item.y, rho = item.rho;
        double a_ps = item.a_ps;
        if (item.flags & kItemPsOnDevice) {
            double a = 0.0;
            if (lane == 0) a = point_source(s, q, x, y).magnification;
            a_ps = shfl_d(a, 0);
        }
        FsOut o{0.0, 0.0, 0, 1, 0, 0};
        bool done = true;
        if (rho <= 0.0) {
            double a = 0.0;
            if (lane == 0) a = point_source(s, q, x, y).magnification;
            o.A = shfl_d(a, 0);
        } else if (st.finite_mode <= 0) {
            o.A = a_ps;
        } else if (item.flags & kItemOutsideBox) {
            // Outside the outer caustic box by the margin, hence outside the
            // sampled caustic's bounding box by it: the bounding-box exit.
            o.A = a_ps;
        } else {
            const CausticModel md = w.models[item.model];
            const P2* raw = w.raw + w.raw_offset[item.model];
            const P2* br = w.branches + md.branch_offset;
            const double margin = st.kinji_threshold * rho;
            const bool adaptive = st.adaptive_source_bins != 0 && (st.tol > 0.0 || st.reltol > 0.0);
            const double amargin = adaptive ? dmax_(margin, 60.0 * rho) : margin;
            const double sampled = sampled_caustic_distance(md, raw, x, y, amargin);
            if (x < md.min_x - amargin || x > md.max_x + amargin || y < md.min_y - amargin ||
                y > md.max_y + amargin) {
                o.A = a_ps;
            } else {
                const double refined = caustic_distance(md, raw, br, x, y, sampled);
                const bool near = refined < st.hex_threshold * rho;
                done = false;
                if (!near) {
                    double safety = 1.0;
                    if (rho >= 1.0e-3 && isfinite(refined) && rho > 0.0) {
                        const double ratio = refined / rho;
                        const double t = st.hex_threshold / dmax_(ratio, st.hex_threshold);
                        safety = dmax_(1.0, 30.0 * t * t * t);
                    }
                    double req = st.adaptive_hex_threshold > 0.0 ? st.adaptive_hex_threshold : 1.0e-3;
                    if (adaptive) req = st.reltol + st.tol / dmax_(fabs(a_ps), 1.0);
                    if (st.hex_threshold > 0.0) {
                        // binary_mag0_with_derivatives on a fresh magnifier (cold roots).
                        double ad = 0.0, ind = 0.0;
                        int cnt = 0;
                        if (lane == 0 && s != 0.0 && q > 0.0) {
                            const BinaryGeom g = make_geom(s, q, x, y);
                            dc roots[5];
                            if (solve_images(g, roots)) {
                                const unsigned mask = physical_mask(g, roots);
                                ad = sum_inverse_jacobians(g, roots, mask, &cnt);
                                ind = derivative_indicator(g, roots, mask);
                            } else {
                                ad = dnan();
                            }
                        }
                        ad = shfl_d(ad, 0);
                        ind = shfl_d(ind, 0);
                        const double rel = ind * rho * rho / dmax_(fabs(ad), 1.0e-10);
                        if (isfinite(rel) && rel <= req / safety) {
                            o.A = ad;
                            o.err = rel * dmax_(fabs(ad), 1.0);
                            done = true;
                        }
                    }
                    if (!done) {
                        // hexadecapole_binary (FSM:792-847): lanes 0..11 solve the ring,
                        // lane 12 the centre when the caller's value is not exact.
                        double v = 0.0;
                        if (lane < 12) {
                            double px, py;
                            ring_sample(lane, x, y, rho, &px, &py);
                            v = point_source(s, q, px, py).magnification;
                        } else if (lane == 12) {
                            v = (item.flags & kItemPsExact) ? a_ps : point_source(s, q, x, y).magnification;
                        }
                        const double a0 = shfl_d(v, 12);
                        double a1p = 0.0, a2p = 0.0, a1c = 0.0;
                        for (int i = 0; i < 4; ++i) {
                            a1p += shfl_d(v, 3 * i);
                            a2p += shfl_d(v, 3 * i + 1);
                            a1c += shfl_d(v, 3 * i + 2);
                        }
                        a1p = a1p / 4.0 - a0;
                        a2p = a2p / 4.0 - a0;
                        a1c = a1c / 4.0 - a0;
                        const double a2rho2 = (16.0 * a2p - a1p) / 3.0;
                        const double a4rho4 = (a1p + a1c) / 2.0 - a2rho2;
                        const double gm = ld_gamma(st.ld_c, st.ld_d);
                        const double lm = ld_lambda(st.ld_c, st.ld_d);
                        const double quad = 0.5 * a2rho2 * (1.0 - 0.2 * gm - lm / 9.0);
                        const double hexc = a4rho4 / 3.0 * (1.0 - 11.0 * gm / 35.0 - 7.0 * lm / 39.0);
                        const double mag = a0 + quad + hexc;
                        const double rel = fabs(hexc) / dmax_(fabs(mag), 1.0e-10);
                        double thr = st.adaptive_hex_threshold;
                        if (adaptive) {
                            const double req2 = st.reltol + st.tol / dmax_(fabs(mag), 1.0);
                            const double cap = req2 / safety;
                            thr = (cap < thr) ? cap : thr;
                        }
                        if (rel <= thr) {
                            o.A = mag;
                            o.err = rel * dmax_(fabs(mag), 1.0);
                            o.method = 1;
                            done = true;
                        }
                    }
                }
                if (!done) {
                    const bool auto_polar = st.finite_mode == 4 && fabs(a_ps) >= 100.0;
                    const bool polar = st.finite_mode == 2 || auto_polar;
                    o.method = polar ? 3 : 2;
                    o.converged = 0;
                    if (lane == 0) {
                        const int slot = atomicAdd(&w.ir_count[polar ? 1 : 0], 1);
                        (polar ? w.ir_polar : w.ir_cart)[slot] = it;
                    }
                }
            }
        }
        if (lane == 0) {
            if (done && !isfinite(o.A)) o.status = kFsNumerical;
            w.out[it] = o;
        }
    }
}

__global__ void __launch_bounds__(128) certify_kernel(FsItem* __restrict__ items, long long n,
                                                     const FsSettingsDev* __restrict__ settings,
                                                     const int* __restrict__ model_base, int pass,
                                                     unsigned char* __restrict__ needed)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const FsItem item = items[i];
        const FsSettingsDev st = settings[item.settings];
        if (!(item.rho > 0.0) || st.finite_mode <= 0) continue;
        // The decision's margin (finite_source_magnifier.cpp:4679-4698).
        const double margin = st.kinji_threshold * item.rho;
        const bool adaptive = st.adaptive_source_bins != 0 && (st.tol > 0.0 || st.reltol > 0.0);
        const double amargin = adaptive ? dmax_(margin, 60.0 * item.rho) : margin;
        const CausticBox b = caustic_outer_box(item.s, item.q);
        if (b.ok && (item.x < b.lo_x - amargin || item.x > b.hi_x + amargin || item.y < -b.half_y - amargin ||
                     item.y > b.half_y + amargin))
            items[i].flags = item.flags | kItemOutsideBox;
        else
            needed[model_base[i / pass] + item.model] = 1;
    }
}

cudaError_t launch_certify(FsItem* items, long long n, const FsSettingsDev* settings, const int* model_base, int pass,
                           unsigned char* needed, int sm_count, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    long long blocks = (n + 127) / 128;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    certify_kernel<<<(unsigned)blocks, 128, 0, stream>>>(items, n, settings, model_base, pass, needed);
    return cudaGetLastError();
}

cudaError_t launch_decide(const FsWork& w, int sm_count, cudaStream_t stream)
{
    if (w.n_items <= 0) return cudaSuccess;
    const int warps = w.n_items;
    int blocks = (warps + 3) / 4;
    const int cap = sm_count * 16;
    if (blocks > cap) blocks = cap;
    decide_kernel<<<blocks, 128, 0, stream>>>(w);
    return cudaGetLastError();
}

// ----- early block routing of large Cartesian points -----
//
// A Cartesian point's in-source cell count is about pi nbin^2 |A| (image area
// A pi rho^2 over cells of (rho / nbin)^2); with the point-source A in place
// of the finite-source one this ranked the largest point of the 4,096-point
// fs_batch first, at its exact count.  The prediction only decides where a
// point runs (the block pass gives the first pass's results bit for bit),
// never what it returns.

struct RouteCand {
    int k;
    int pad;
    double est;
};

__global__ void __launch_bounds__(128) route_estimate_kernel(FsWork w, double min_cells, RouteCand* cand, int* ncand)
{
    const int n = w.ir_count[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int it = w.ir_cart[k];
        const FsOut o = w.out[it];
        const FsItem item = w.items[it];
        if (o.status != kFsOk || !(item.rho > 0.0)) continue;
        const FsSettingsDev st = w.settings[item.settings];
        const double nbin = static_cast<double>(max(st.source_bins, 1));
        const double a = point_source(item.s, item.q, item.x, item.y).magnification;
        const double est = kPi * nbin * nbin * dmax_(fabs(a), 1.0);
        if (est > min_cells) {
            const int c = atomicAdd(ncand, 1);
            if (c < kRouteCands) cand[c] = RouteCand{k, 0, est};
        }
    }
}

// The kEarlyMax largest candidates, largest first (ties by list position).
__global__ void __launch_bounds__(256) route_select_kernel(FsWork w, const RouteCand* cand, const int* ncand)
{
    const int m = min(*ncand, kRouteCands);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const RouteCand c = cand[i];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const RouteCand o = cand[j];
            rank += (o.est > c.est || (o.est == c.est && o.k < c.k)) ? 1 : 0;
        }
        if (rank < kEarlyMax) w.early_cart[rank] = c.k;
    }
    if (threadIdx.x == 0) w.ir_count[5] = min(m, kEarlyMax);
}

size_t route_bytes() { return (size_t)kRouteCands * sizeof(RouteCand); }

cudaError_t launch_route_early(const FsWork& w, double min_cells, void* cand, int max_points, int sm_count,
                               cudaStream_t stream)
{
    if (max_points <= 0) return cudaSuccess;
    int blocks = (max_points + 127) / 128;
    if (blocks > 4 * sm_count) blocks = 4 * sm_count;
    int* ncand = w.ir_count + 48;
    route_estimate_kernel<<<blocks, 128, 0, stream>>>(w, min_cells, static_cast<RouteCand*>(cand), ncand);
    route_select_kernel<<<1, 256, 0, stream>>>(w, static_cast<const RouteCand*>(cand), ncand);
    return cudaGetLastError();
}

} // namespace lcbi
