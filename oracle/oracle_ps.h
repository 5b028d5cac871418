// CPU oracle (test infrastructure only): restatement of the lcbinint
// point-source path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline arm may load the library built from this file (oracle/_build).
//
// Every routine follows the reference's arithmetic operation by operation so
// that, compiled without floating-point contraction (plain x86-64 SSE2, as the
// reference's own Release build is), it reproduces the reference bit for bit.
// Citations are to files of the NunotaKansuke/lcbinint repository:
//   SG  = third_party/skowron_gould/SkowronGould.cpp (Skowron & Gould 2012)
//   PSM = src/lcbinint/magnification/point_source_magnifier.cpp
#pragma once

#include <cmath>

namespace oracle {

struct cplx {
    double re, im;
};

inline cplx mk(double re, double im) { return {re, im}; }
inline cplx add(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx sub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx mul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cplx scl(double s, cplx a) { return {s * a.re, s * a.im}; }
// Division by the textbook formula, the same formula SkowronGould.h uses.
inline cplx dvd(cplx a, cplx b)
{
    const double md = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / md, (a.im * b.re - a.re * b.im) / md};
}
inline double norm2(cplx a) { return a.re * a.re + a.im * a.im; }
inline double cabs(cplx a) { return std::sqrt(a.re * a.re + a.im * a.im); }
inline bool is_zero(cplx a) { return a.re == 0.0 && a.im == 0.0; }
inline bool same(cplx a, cplx b) { return a.re == b.re && a.im == b.im; }
// Principal square root with the sign convention of SkowronGould.h sqrt(complex).
inline cplx csqrt_sg(cplx z)
{
    const double md = std::sqrt(z.re * z.re + z.im * z.im);
    if (!(md > 0.0)) return {0.0, 0.0};
    return {std::sqrt((md + z.re) / 2.0), std::sqrt((md - z.re) / 2.0) * ((z.im > 0.0) ? 1.0 : -1.0)};
}

// Roots of sum_k poly[k] z^k (degree <= 5) by the deflation scheme of
// cmplx_roots_gen (SG:79-168): Laguerre/second-order/Newton per root,
// quadratic tail, then Newton polish of degree-1 roots on the full polynomial.
void roots_gen(cplx* roots, const cplx* poly, int degree, bool polish);

struct PointSource {
    double magnification;
    int image_count;
};

// binary_mag0 (PSM:652-693, cold start).
PointSource binary_mag0(double separation, double mass_ratio, double y1, double y2);

// binary_mag0_with_derivatives (PSM:583-611) -> also returns the indicator.
PointSource binary_mag0_derivatives(double separation, double mass_ratio, double y1, double y2,
                                    double* indicator);

// binary_image_candidates (PSM:739-778): up to 5 rows of x, y, detJ, residual, physical,
// sorted by residual.  Returns the row count.
int binary_image_candidates(double separation, double mass_ratio, double y1, double y2,
                            double* out);

} // namespace oracle
