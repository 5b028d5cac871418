// Binary-lens point-source magnification on the device.
//
// Follows PointSourceMagnifier::binary_mag0 (point_source_magnifier.cpp:652-693):
// lens geometry (make_fast_vbm_geometry, :105-117), the six coefficients of
// the lens quintic (binary_polynomial_coefficients, :152-185), its five roots
// (lcbi_roots.cuh), residual-ranked image selection (select_physical_roots,
// :225-279) and the sum of 1/|det J| (point_source_result_from_roots, :281-297).
// Operation order is the reference's, so results are bit-identical under
// --fmad=false.
#pragma once

#include "lcbi_roots.cuh"

namespace lcbi {

// Lens frame: the heavier mass m1 at z = a, the lighter m2 at the origin,
// a = -s when q < 1 (else +s, with q inverted).  y is the source shifted from
// the centre-of-mass frame into this frame.
struct BinaryGeom {
    double a, m1, m2, a2, a3, m2_2;
    dc y;
};

__device__ __forceinline__ BinaryGeom make_geom(double separation, double mass_ratio, double y1, double y2)
{
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const double a = q_in < 1.0 ? -s : s;
    const double m1 = 1.0 / (1.0 + q);
    const double m2 = q * m1;
    const double a2 = a * a;
    BinaryGeom g;
    g.a = a;
    g.m1 = m1;
    g.m2 = m2;
    g.a2 = a2;
    g.a3 = a2 * a;
    g.m2_2 = m2 * m2;
    g.y = dc{y1 + a * m1, y2};
    return g;
}

__device__ __forceinline__ void quintic_coefficients(const BinaryGeom& g, dc* c)
{
    const double a = g.a;
    const dc y = g.y;
    const dc yc{y.re, -y.im};
    const double c9 = g.a2 * g.m2_2;
    const double c10 = a * g.m2;
    const dc c12{a - yc.re, 0.0 - yc.im};
    const dc c13{a + y.re, 0.0 + y.im};
    const dc c14 = cadd(c13, y);
    const dc c15{c14.re, -c14.im};
    const dc c16 = cscale(a, y);
    const dc c17{c16.re, -c16.im};
    const dc c18{c12.re, -c12.im};

    c[0] = cscale(c9, y);
    {
        const dc t1 = cscale(2.0, c17);
        const dc t2{t1.re - (2.0 + g.a2), t1.im - 0.0};
        const dc t3 = cmul(t2, y);
        const dc t5 = cscale(c10, dc{a + t3.re, 0.0 + t3.im});
        c[1] = dc{-c9 + t5.re, 0.0 + t5.im};
    }
    {
        const dc u1{1.0 + c16.re, 0.0 + c16.im};
        const dc u3 = cmul(cscale(2.0, yc), c13);
        const dc u5 = cscale(c10, csub(u1, u3));
        const dc v1{c17.re - 1.0, c17.im - 0.0};
        const dc v3 = csub(cmul(c16, c12), c18);
        c[2] = csub(u5, cmul(v1, v3));
    }
    {
        const dc w1 = cscale(c10, c15);
        const dc w3 = cscale(2.0 * (1.0 + g.a2), y);
        const dc w4{g.a3 + w3.re, 0.0 + w3.im};
        const dc w6 = csub(w4, cmul(c17, c14));
        const dc w8 = cadd(w1, cmul(w6, yc));
        c[3] = csub(w8, cscale(a, c13));
    }
    {
        const dc x2 = cmul(yc, dc{c13.re + a, c13.im + 0.0});
        const dc x4 = cmul(c12, dc{x2.re - 1.0, x2.im - 0.0});
        c[4] = dc{-c10 - x4.re, 0.0 - x4.im};
    }
    c[5] = cmul(yc, c12);
}

// Squared lens-equation residual of image z (residual_squared, :187-203).
__device__ __forceinline__ double image_residual2(const BinaryGeom& g, dc z)
{
    const double u1 = z.re - g.a;
    const double v1 = -z.im;
    const double d1 = u1 * u1 + v1 * v1;
    const double u2 = z.re;
    const double v2 = -z.im;
    const double d2 = u2 * u2 + v2 * v2;
    const double r_re = g.y.re - z.re + g.m1 * u1 / d1 + g.m2 * u2 / d2;
    const double r_im = g.y.im - z.im - g.m1 * v1 / d1 - g.m2 * v2 / d2;
    return r_re * r_re + r_im * r_im;
}

// det J of image z (jacobian_determinant, :205-223).
__device__ __forceinline__ double image_jacobian(const BinaryGeom& g, dc z)
{
    const double u1 = z.re - g.a;
    const double v1 = z.im;
    const double d1 = u1 * u1 + v1 * v1;
    const double d1_2 = d1 * d1;
    const double u2 = z.re;
    const double v2 = z.im;
    const double d2 = u2 * u2 + v2 * v2;
    const double d2_2 = d2 * d2;
    const double dre = g.m1 * (u1 * u1 - v1 * v1) / d1_2 + g.m2 * (u2 * u2 - v2 * v2) / d2_2;
    const double dim = -2.0 * g.m1 * u1 * v1 / d1_2 - 2.0 * g.m2 * u2 * v2 / d2_2;
    return 1.0 - (dre * dre + dim * dim);
}

// Bit mask of physical roots: the two worst residuals are dropped when the
// third worst is 1e8 times smaller (plus 1e-24) (select_physical_roots).
__device__ __forceinline__ unsigned physical_mask(const BinaryGeom& g, const dc* roots)
{
    int w1 = 0, w2 = 0, w3 = 0;
    double v1 = 0.0, v2 = 0.0, v3 = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const double r = image_residual2(g, roots[i]);
        if (i == 0) {
            w1 = 0; v1 = r;
        } else if (i == 1) {
            if (r > v1) { w2 = w1; v2 = v1; w1 = 1; v1 = r; }
            else { w2 = 1; v2 = r; }
        } else if (i == 2) {
            if (r > v1) { w3 = w2; v3 = v2; w2 = w1; v2 = v1; w1 = 2; v1 = r; }
            else if (r > v2) { w3 = w2; v3 = v2; w2 = 2; v2 = r; }
            else { w3 = 2; v3 = r; }
        } else if (r > v1) {
            w3 = w2; v3 = v2; w2 = w1; v2 = v1; w1 = i; v1 = r;
        } else if (r > v2) {
            w3 = w2; v3 = v2; w2 = i; v2 = r;
        } else if (r > v3) {
            w3 = i; v3 = r;
        }
    }
    (void)w3;
    const bool three = v2 * 1.0e-8 > v3 + 1.0e-24;
    unsigned mask = 0x1fu;
    if (three) mask &= ~((1u << w1) | (1u << w2));
    return mask;
}

struct PsResult {
    double magnification;
    int image_count;
    int status;  // 0 ok, 2 = numerical error (degenerate quintic)
};

__device__ __forceinline__ double sum_inverse_jacobians(const BinaryGeom& g, const dc* roots, unsigned mask,
                                                        int* count)
{
    double A = 0.0;
    int n = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        if (!(mask & (1u << i))) continue;
        A += 1.0 / fabs(image_jacobian(g, roots[i]));
        ++n;
    }
    *count = n;
    return A;
}

// Solves the lens quintic; false when its leading coefficient vanishes (the
// source sits exactly on the lighter lens), a case on which the reference's
// polish step never terminates.
__device__ __forceinline__ bool solve_images(const BinaryGeom& g, dc* roots)
{
    dc c[6];
    quintic_coefficients(g, c);
    if (czero(c[5])) return false;
    roots5(c, roots);
    return true;
}

// binary_mag0 for one source position (cold start).
__device__ __forceinline__ PsResult point_source(double separation, double mass_ratio, double y1, double y2)
{
    PsResult r{0.0, 0, 0};
    if (separation == 0.0 || mass_ratio <= 0.0) return r;
    const BinaryGeom g = make_geom(separation, mass_ratio, y1, y2);
    dc roots[5];
    if (!solve_images(g, roots)) {
        r.magnification = __longlong_as_double(0x7ff8000000000000ll);
        r.status = 2;
        return r;
    }
    const unsigned mask = physical_mask(g, roots);
    r.magnification = sum_inverse_jacobians(g, roots, mask, &r.image_count);
    return r;
}

// VBM-style smoothness indicator of the point-source map at the physical
// images (derivative_error_indicator_from_roots, :313-359); +inf on a singular image.
__device__ __forceinline__ double derivative_indicator(const BinaryGeom& g, const dc* roots, unsigned mask)
{
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double indicator = 0.0;
    const dc a{g.a, 0.0};
    const dc m1{g.m1, 0.0};
    const dc m2{g.m2, 0.0};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        if (!(mask & (1u << i))) continue;
        const dc z = roots[i];
        const dc dza = csub(z, a);
        const dc za2 = cmul(dza, dza);
        const dc zb2 = cmul(z, z);
        const dc j1 = cadd(cdiv(m1, za2), cdiv(m2, zb2));
        const dc j1c{j1.re, -j1.im};
        const double det_j = 1.0 - cmul(j1, j1c).re;
        if (det_j == 0.0 || !isfinite(det_j)) return inf;
        dc j2 = cscale(-2.0, cadd(cdiv(m1, cmul(za2, dza)), cdiv(m2, cmul(zb2, z))));
        dc j3 = cscale(6.0, cadd(cdiv(m1, cmul(za2, za2)), cdiv(m2, cmul(zb2, zb2))));
        const double det_j2 = det_j * det_j;
        const dc j1c2 = cmul(j1c, j1c);
        j3 = cmul(j3, j1c2);
        const double ob2 = (j2.re * j2.re + j2.im * j2.im) * (6.0 - 6.0 * det_j + det_j2);
        j2 = cmul(cmul(cmul(j2, j2), j1c2), j1c);
        const double den = fabs(det_j * det_j2 * det_j2);
        if (den == 0.0 || !isfinite(den)) return inf;
        const double cq = 0.5 * (fabs(ob2 - 6.0 * j2.re - 2.0 * j3.re * det_j) + 3.0 * fabs(j2.im)) / den;
        if (!isfinite(cq)) return inf;
        indicator += cq;
    }
    return indicator;
}

// Image candidates sorted by residual (binary_image_candidates, :739-778):
// positions, sqrt-residuals and the 3-image rule with ratio 1e-4 and gap 1e-12.
// Returns the number of physical candidates (3 or 5); 0 if degenerate.
__device__ __forceinline__ int image_candidates(const BinaryGeom& g, dc* pos, double* res, double* det)
{
    dc roots[5];
    if (!solve_images(g, roots)) return 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        pos[i] = roots[i];
        res[i] = sqrt(image_residual2(g, roots[i]));
        det[i] = image_jacobian(g, roots[i]);
    }
    // Stable insertion sort by residual.
#pragma unroll
    for (int i = 1; i < 5; ++i) {
#pragma unroll
        for (int k = i; k > 0; --k) {
            if (res[k] < res[k - 1]) {
                const double tr = res[k]; res[k] = res[k - 1]; res[k - 1] = tr;
                const double td = det[k]; det[k] = det[k - 1]; det[k - 1] = td;
                const dc tp = pos[k]; pos[k] = pos[k - 1]; pos[k - 1] = tp;
            }
        }
    }
    return (res[3] * 1.0e-4 > res[2] + 1.0e-12) ? 3 : 5;
}

} // namespace lcbi
