// Warp-cooperative caustic-distance queries over a sampled caustic model.
//
// The reference buckets caustic points into a 128x128 grid and scans the
// buckets a query window covers (finite_source_magnifier.cpp:4107-4246).  A
// minimum does not depend on visiting order, so a warp instead scans every
// sampled point (5,600 at the default 1,400 phases) and keeps the ones whose
// bucket lies in the window: the same set, the same minimum, no bucket lists.
#pragma once

#include "lcbi_fs.cuh"
#include "lcbi_warp.cuh"

namespace lcbi {

// binary_sampled_caustic_distance (FSM:4183-4246).
__device__ __forceinline__ double sampled_caustic_distance(const CausticModel& md, const P2* __restrict__ raw,
                                                           double x, double y, double R)
{
    if (R > 0.0 && (x < md.min_x - R || x > md.max_x + R || y < md.min_y - R || y > md.max_y + R)) return dinf();
    double d2 = dinf();
    const int n = 4 * md.bins;
    if (R > 0.0) {
        const int ix0 = grid_cell(x - R, md.min_x, md.step_x), ix1 = grid_cell(x + R, md.min_x, md.step_x);
        const int iy0 = grid_cell(y - R, md.min_y, md.step_y), iy1 = grid_cell(y + R, md.min_y, md.step_y);
        for (int t = lane_id(); t < n; t += 32) {
            const P2 p = raw[t];
            const int ix = grid_cell(p.x, md.min_x, md.step_x);
            const int iy = grid_cell(p.y, md.min_y, md.step_y);
            if (ix < ix0 || ix > ix1 || iy < iy0 || iy > iy1) continue;
            const double dx = x - p.x;
            const double dy = y - p.y;
            const double c = dx * dx + dy * dy;
            if (c < d2) d2 = c;
        }
        d2 = warp_min(d2);
        if (d2 == dinf()) return d2;
    } else {
        for (int t = lane_id(); t < n; t += 32) {
            const P2 p = raw[t];
            const double dx = x - p.x;
            const double dy = y - p.y;
            const double c = dx * dx + dy * dy;
            if (c < d2) d2 = c;
        }
        d2 = warp_min(d2);
    }
    return sqrt(d2);
}

// binary_caustic_distance (FSM:4107-4181): segment distance refined from a hint.
__device__ __forceinline__ double caustic_distance(const CausticModel& md, const P2* __restrict__ raw,
                                                   const P2* __restrict__ br, double x, double y, double hint)
{
    double nearest = hint;
    const int bins = md.bins;
    if (!isfinite(nearest)) {
        double n2 = dinf();
        for (int t = lane_id(); t < 4 * bins; t += 32) {
            const P2 p = raw[t];
            const double dx = x - p.x;
            const double dy = y - p.y;
            const double d2 = dx * dx + dy * dy;
            if (d2 < n2) n2 = d2;
        }
        nearest = sqrt(warp_min(n2));
    }
    const double R = nearest + md.max_seg_len;
    const int ix0 = grid_cell(x - R, md.min_x, md.step_x), ix1 = grid_cell(x + R, md.min_x, md.step_x);
    const int iy0 = grid_cell(y - R, md.min_y, md.step_y), iy1 = grid_cell(y + R, md.min_y, md.step_y);
    double d = nearest;
    const P2 src{x, y};
    for (int t = lane_id(); t < 4 * bins; t += 32) {
        const int b = t / bins;
        const int pos = t - b * bins;
        const P2* bb = br + (long long)b * bins;
        const P2 p = bb[pos];
        const int ix = grid_cell(p.x, md.min_x, md.step_x);
        const int iy = grid_cell(p.y, md.min_y, md.step_y);
        if (ix < ix0 || ix > ix1 || iy < iy0 || iy > iy1) continue;
        if (bins < 2) continue;
        const int prev = pos > 0 ? pos - 1 : bins - 1;
        const int next = (pos + 1) % bins;
        d = dmin_(d, seg_dist(src, bb[prev], p));
        d = dmin_(d, seg_dist(src, p, bb[next]));
    }
    return warp_min(d);
}

} // namespace lcbi
