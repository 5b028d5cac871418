// Double-precision complex arithmetic for the lcbinint B200 kernels.
//
// Every operation is written out component by component in the same order as
// the reference (SkowronGould.h operators, the FastComplex helpers of
// point_source_magnifier.cpp:45-96), and the translation units that include
// this header are compiled with --fmad=false, so each result is the IEEE
// double the reference's SSE2 build computes.  Bit-exact parity depends on it.
#pragma once

#include <cuda_runtime.h>

namespace lcbi {

struct dc {
    double re, im;
};

__host__ __device__ __forceinline__ dc mkc(double re, double im) { return dc{re, im}; }
__host__ __device__ __forceinline__ dc cadd(dc a, dc b) { return dc{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ dc csub(dc a, dc b) { return dc{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ dc cmul(dc a, dc b)
{
    return dc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ dc cscale(double s, dc a) { return dc{s * a.re, s * a.im}; }
// Textbook quotient, the formula of SkowronGould.h operator/(complex, complex).
__host__ __device__ __forceinline__ dc cdiv(dc a, dc b)
{
    const double md = b.re * b.re + b.im * b.im;
    return dc{(a.re * b.re + a.im * b.im) / md, (a.im * b.re - a.re * b.im) / md};
}
// Smith (1962) quotient, the algorithm libgcc's __divdc3 applies to
// std::complex<double> division in the reference's lens-equation helpers
// (point_source_magnifier.cpp:780-792).  Only the finite, non-extreme branch
// is needed: operands here are O(1e-12 .. 1e12).
__host__ __device__ __forceinline__ dc cdiv_smith(dc a, dc b)
{
    const double c = b.re, d = b.im;
    if (fabs(c) < fabs(d)) {
        const double ratio = c / d;
        const double denom = (c * ratio) + d;
        return dc{((a.re * ratio) + a.im) / denom, ((a.im * ratio) - a.re) / denom};
    }
    const double ratio = d / c;
    const double denom = (d * ratio) + c;
    return dc{((a.im * ratio) + a.re) / denom, (a.im - (a.re * ratio)) / denom};
}
__host__ __device__ __forceinline__ double cnorm2(dc a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ double cabs_(dc a) { return sqrt(a.re * a.re + a.im * a.im); }
__host__ __device__ __forceinline__ bool czero(dc a) { return a.re == 0.0 && a.im == 0.0; }
__host__ __device__ __forceinline__ bool ceq(dc a, dc b) { return a.re == b.re && a.im == b.im; }
// Square root with the branch convention of SkowronGould.h sqrt(complex).
__host__ __device__ __forceinline__ dc csqrt_sg(dc z)
{
    const double md = sqrt(z.re * z.re + z.im * z.im);
    if (!(md > 0.0)) return dc{0.0, 0.0};
    return dc{sqrt((md + z.re) / 2.0), sqrt((md - z.re) / 2.0) * ((z.im > 0.0) ? 1.0 : -1.0)};
}

// hypot by Borges (2019, "An improved algorithm for hypot(a,b)"), the
// correction step without fused multiply-add.  It returns the same double as
// the host C library's hypot for the magnitudes used here (checked on 5e7
// random pairs), which matters because probe directions in the seed search
// are normalised by it.
__host__ __device__ __forceinline__ double hypot_borges(double x, double y)
{
    x = fabs(x);
    y = fabs(y);
    const double ax = x < y ? y : x;
    const double ay = x < y ? x : y;
    if (ay <= ax * 0x1p-54) return ax + ay;
    double h = sqrt(ax * ax + ay * ay);
    double t1, t2;
    if (h <= 2.0 * ay) {
        const double delta = h - ay;
        t1 = ax * (2.0 * delta - ax);
        t2 = (delta - 2.0 * (ax - ay)) * delta;
    } else {
        const double delta = h - ax;
        t1 = 2.0 * delta * (ax - 2.0 * ay);
        t2 = (4.0 * delta - ay) * ay + delta * delta;
    }
    h -= (t1 + t2) / (2.0 * h);
    return h;
}

} // namespace lcbi
