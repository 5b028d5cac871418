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

// A box that holds every point of a binary lens's caustic, from the lens
// equation alone (no sampling), so that a source outside it by the decision's
// margin is outside the sampled caustic's bounding box by that margin too
// (the sampled points lie on the caustic).
//
// Lens frame of the sampled caustic: mass m1 (the heavier) at z = a, mass m2
// at 0, a = -s or s; a critical point z has |m1/(z-a)^2 + m2/z^2| = 1 and maps
// to w = z - m1/conj(z-a) - m2/conj(z).  Split the critical points by which
// lens dominates, mn/dn^2 >= mf/df^2 (dn, df their distances to the near and
// far lens).  Then
//   dn <= sqrt(2 mn)                              (1 <= mn/dn^2 + mf/df^2),
//   df >= max(s - sqrt(2 mn), s / (1 + sqrt(mn/mf)))   (dn + df >= s, dominance),
//   mn/dn^2 <= 1 + e,  e = mf / df_min^2          (reverse triangle inequality),
//   mn/dn^2 >= 1 - e   when e < 1,
// and |w - zn| <= |dn - mn/dn| + mf/df, with |d - mn/d| increasing away from
// sqrt(mn) so that its maximum over [dn_min, dn_max] is at an end.  When
// dn_max < s the far lens's deflection is nearly constant near zn:
// |w - (zn - mf/conj(zn - zf))| <= |dn - mn/dn| + mf dn_max / (s (s - dn_max)).
// The smaller of the two discs about each lens is kept.
struct CausticBox {
    double lo_x, hi_x, half_y;  // source frame of the decision (the lens frame shifted by -a m1)
    bool ok;
};

__device__ __forceinline__ void dominated_disc(double mn, double mf, double s, double zn, double shift, double* c,
                                               double* r)
{
    double dmax = sqrt(2.0 * mn);
    const double dfmin = fmax(s - dmax, s / (1.0 + sqrt(mn / mf)));
    const double e = mf / (dfmin * dfmin);
    const double dmin = sqrt(mn / (1.0 + e));
    if (e < 1.0) dmax = fmin(dmax, sqrt(mn / (1.0 - e)));
    const double core = fmax(fabs(dmin - mn / dmin), fabs(dmax - mn / dmax));
    *c = zn;
    *r = core + mf / dfmin;
    if (dmax < s) {
        const double r2 = core + mf * dmax / (s * (s - dmax));
        if (r2 < *r) {
            *c = zn - shift;
            *r = r2;
        }
    }
}

__device__ __forceinline__ CausticBox caustic_outer_box(double separation, double mass_ratio)
{
    CausticBox b{0.0, 0.0, 0.0, false};
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    if (!(s > 0.0) || !(q_in > 0.0) || !isfinite(s) || !isfinite(q_in)) return b;
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const double a = q_in < 1.0 ? -s : s;
    const double m1 = 1.0 / (1.0 + q);
    const double m2 = q * m1;
    double c1, r1, c2, r2;
    dominated_disc(m1, m2, s, a, m2 / a, &c1, &r1);     // near m1: far-lens deflection m2/conj(a - 0)
    dominated_disc(m2, m1, s, 0.0, -m1 / a, &c2, &r2);  // near m2: far-lens deflection m1/conj(0 - a)
    // Generous slack for the rounding of the sampled points and of this bound.
    r1 = r1 * (1.0 + 1.0e-6) + 1.0e-9;
    r2 = r2 * (1.0 + 1.0e-6) + 1.0e-9;
    const double sh = a * m1;
    b.lo_x = fmin(c1 - r1, c2 - r2) - sh;
    b.hi_x = fmax(c1 + r1, c2 + r2) - sh;
    const double pad = 1.0e-9 + 1.0e-9 * (fabs(b.lo_x) + fabs(b.hi_x));
    b.lo_x -= pad;
    b.hi_x += pad;
    b.half_y = fmax(r1, r2);
    b.ok = isfinite(b.lo_x) && isfinite(b.hi_x) && isfinite(b.half_y);
    return b;
}

} // namespace lcbi
