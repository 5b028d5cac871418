// Complex polynomial roots on the device: the Skowron & Gould (2012) scheme
// (Laguerre / second-order general / Newton regimes, deflation, direct
// quadratic tail, Newton polish on the full polynomial), as the reference
// drives it through cmplx_roots_gen (third_party/skowron_gould/SkowronGould.cpp:79-168)
// with a cold start and polishing on.
//
// One thread solves one polynomial.  The degree is a template parameter so
// every Horner loop unrolls and all coefficients stay in registers.  Each
// iteration loop is bounded (80 steps per regime, as in the method), so a
// solve always terminates.
#pragma once

#include "lcbi_complex.cuh"

namespace lcbi {

namespace sg {

constexpr int kMaxIt = 80;
constexpr double kFracErr = 2.0e-15;
constexpr double kTwoPi = 6.283185307179586476925286766559;

// Cycle-breaking jump fractions published with the method.
__device__ __forceinline__ double jump(int k)
{
    switch (k) {
    case 0: return 0.64109297;
    case 1: return 0.91577881;
    case 2: return 0.25921289;
    case 3: return 0.50487203;
    case 4: return 0.08177045;
    case 5: return 0.13653241;
    case 6: return 0.306162;
    case 7: return 0.37794326;
    case 8: return 0.04618805;
    default: return 0.75132137;
    }
}

// Random-direction escape used only when a derivative is exactly zero.
static __device__ __noinline__ dc escape_dir(double angle)
{
    double s, c;
    sincos(angle, &s, &c);
    return dc{c, s};
}

// p(z), p'(z), p''(z)/2 and the Adams (1967) stopping bound ek.
template <int N, bool D2>
__device__ __forceinline__ void horner(const dc* poly, dc z, dc& p, dc& dp, dc& d2, double& ek,
                                       bool with_ek)
{
    ek = cabs_(poly[N]);
    const double absroot = cabs_(z);
    p = poly[N];
    dp = dc{0.0, 0.0};
    d2 = dc{0.0, 0.0};
#pragma unroll
    for (int k = N; k >= 1; --k) {
        if (D2) d2 = cadd(dp, cmul(d2, z));
        dp = cadd(p, cmul(dp, z));
        p = cadd(poly[k - 1], cmul(p, z));
        if (with_ek) ek = absroot * ek + cabs_(p);
    }
}

__device__ __forceinline__ double crit2(double ek)
{
    const double t = kFracErr * ek;
    return t * t;
}

// A degree-N polynomial passed by value, so that a call that is not inlined
// takes no address of the caller's coefficients (which then stay in registers).
template <int N>
struct PolyN {
    dc c[N + 1];
};

// Plain Laguerre iteration (cmplx_laguerre, SkowronGould.cpp:472-625), the
// fallback when the three-regime solver does not converge in 80 steps; returns
// the root it reaches (its last iterate when it does not converge).  Rarely
// taken, so kept out of line.
template <int N>
__device__ __noinline__ dc laguerre_fallback(const PolyN<N> pn, dc root)
{
    const dc* poly = pn.c;
    const double one_nth = 1.0 / N;
    const double n_1_nth = (N - 1.0) * one_nth;
    const double two_n_div_n_1 = 2.0 / n_1_nth;
    bool good = false;
    for (int i = 1; i <= kMaxIt; ++i) {
        const double absroot = cabs_(root);
        dc p, dp, d2;
        double ek;
        horner<N, true>(poly, root, p, dp, d2, ek, true);
        const double abs2p = cnorm2(p);
        if (abs2p == 0.0) return root;
        const double cr = crit2(ek);
        if (abs2p < cr) {
            if (abs2p < 0.01 * cr) return root;
            good = true;
        } else {
            good = false;
        }
        dc denom{0.0, 0.0}, fn{0.0, 0.0};
        if (!czero(dp)) {
            fn = cdiv(p, dp);
            const dc fe = cdiv(d2, dp);
            const dc fh = cmul(fn, fe);
            const dc t = cscale(two_n_div_n_1, fh);
            const dc ds = csqrt_sg(dc{1.0 - t.re, 0.0 - t.im});
            const dc nd = cscale(n_1_nth, ds);
            denom = (ds.re >= 0.0) ? dc{one_nth + nd.re, 0.0 + nd.im} : dc{one_nth - nd.re, 0.0 - nd.im};
        }
        dc dx;
        if (czero(denom)) dx = cscale(absroot + 1.0, escape_dir(jump(i % 10) * 2 * 3.14159265358979323846));
        else dx = cdiv(fn, denom);
        dc nr = csub(root, dx);
        if (ceq(nr, root)) return root;
        if (good) return nr;
        if (i % 10 == 0) nr = csub(root, cscale(jump((i / 10 - 1) % 10), dx));
        root = nr;
    }
    return root;
}

// Three-regime solver (cmplx_laguerre2newton, SkowronGould.cpp:764-1130),
// starting in Laguerre mode from `root`.  Returns false on non-convergence.
template <int N>
__device__ __forceinline__ bool laguerre2newton(const dc* poly, dc& root)
{
    const double one_nth = 1.0 / N;
    const double n_1_nth = (N - 1) * one_nth;
    const double two_n_div_n_1 = 2.0 / n_1_nth;
    int iter = 0;
    double cr = 0.0;
    int j = 1;
    bool good = false;
    int mode = 2;
    // Each pass of this loop runs at most 80 + 80 + 11 steps and adds at least
    // one to `iter`; the Newton regime leaves with failure once iter >= 80.
    for (int guard = 0; guard < 64; ++guard) {
        if (mode >= 2) {
            int i;
            for (i = 1; i <= kMaxIt; ++i) {
                dc p, dp, d2;
                double ek;
                horner<N, true>(poly, root, p, dp, d2, ek, true);
                const double abs2p = cnorm2(p);
                ++iter;
                if (abs2p == 0.0) return true;
                cr = crit2(ek);
                if (abs2p < cr) {
                    if (abs2p < 0.01 * cr) return true;
                    good = true;
                } else {
                    good = false;
                }
                dc denom{0.0, 0.0}, fn{0.0, 0.0};
                if (!czero(dp)) {
                    fn = cdiv(p, dp);
                    const dc fe = cdiv(d2, dp);
                    const dc fh = cmul(fn, fe);
                    const double a2f = cnorm2(fh);
                    if (a2f <= 0.0625) mode = (a2f <= 0.000625) ? 0 : 1;
                    const dc t = cscale(two_n_div_n_1, fh);
                    const dc ds = csqrt_sg(dc{1.0 - t.re, 0.0 - t.im});
                    const dc nd = cscale(n_1_nth, ds);
                    denom = (ds.re > 0.0) ? dc{one_nth + nd.re, 0.0 + nd.im} : dc{one_nth - nd.re, 0.0 - nd.im};
                }
                dc dx;
                if (czero(denom)) {
                    const dc e = escape_dir(jump(i % 10) * 2 * 3.14159265358979323846);
                    dx = dc{(cabs_(root) + 1.0) + e.re, e.im};
                } else {
                    dx = cdiv(fn, denom);
                }
                dc nr = csub(root, dx);
                if (ceq(nr, root)) return true;
                if (good) { root = nr; return true; }
                if (mode != 2) {
                    root = nr;
                    j = i + 1;
                    break;
                }
                if (i % 10 == 0) nr = csub(root, cscale(jump((i / 10 - 1) % 10), dx));
                root = nr;
            }
            if (i >= kMaxIt) return false;
        }
        if (mode == 1) {
            int i;
            for (i = j; i <= kMaxIt; ++i) {
                const bool fresh = ((i - j) % 10 == 0);
                dc p, dp, d2;
                double ek;
                horner<N, true>(poly, root, p, dp, d2, ek, fresh);
                if (fresh) cr = crit2(ek);
                const double abs2p = cnorm2(p);
                ++iter;
                if (abs2p == 0.0) return true;
                if (abs2p < cr) {
                    if (czero(dp)) return true;
                    if (abs2p < 0.01 * cr) return true;
                    good = true;
                } else {
                    good = false;
                }
                dc dx;
                if (czero(dp)) {
                    dx = cscale(cabs_(root) + 1.0, escape_dir(jump(i % 10) * 2 * 3.14159265358979323846));
                } else {
                    const dc fn = cdiv(p, dp);
                    const dc fe = cdiv(d2, dp);
                    const dc fh = cmul(fn, fe);
                    if (cnorm2(fh) <= 0.000625) mode = 0;
                    dx = cmul(fn, dc{1.0 + fh.re, 0.0 + fh.im});
                }
                dc nr = csub(root, dx);
                if (ceq(nr, root)) return true;
                if (good) { root = nr; return true; }
                if (mode != 1) {
                    root = nr;
                    j = i + 1;
                    break;
                }
                if (i % 10 == 0) nr = csub(root, cscale(jump((i / 10 - 1) % 10), dx));
                root = nr;
            }
            if (i >= kMaxIt) return false;
        }
        if (mode == 0) {
            for (int i = j; i <= j + 10; ++i) {
                const bool fresh = (i == j);
                dc p, dp, d2;
                double ek;
                horner<N, false>(poly, root, p, dp, d2, ek, fresh);
                if (fresh) cr = crit2(ek);
                const double abs2p = cnorm2(p);
                ++iter;
                if (abs2p == 0.0) return true;
                if (abs2p < cr) {
                    if (czero(dp)) return true;
                    if (abs2p < 0.01 * cr) return true;
                    good = true;
                } else {
                    good = false;
                }
                dc dx;
                if (czero(dp)) dx = cscale(cabs_(root) + 1.0, escape_dir(2 * 3.14159265358979323846 * jump(i % 10)));
                else dx = cdiv(p, dp);
                const dc nr = csub(root, dx);
                if (ceq(nr, root)) return true;
                if (good) { root = nr; return true; }
                root = nr;
            }
            if (iter >= kMaxIt) return false;
            mode = 2;
        }
    }
    return false;
}

// Newton polish on the full polynomial (cmplx_newton_spec, SkowronGould.cpp:626-763).
template <int N>
__device__ __forceinline__ void newton_polish(const dc* poly, dc& root)
{
    bool good = false;
    double cr = 0.0;
    for (int i = 1; i <= kMaxIt; ++i) {
        const bool fresh = (i % 10 == 1);
        dc p, dp, d2;
        double ek;
        horner<N, false>(poly, root, p, dp, d2, ek, fresh);
        if (fresh) cr = crit2(ek);
        const double abs2p = cnorm2(p);
        if (abs2p == 0.0) return;
        if (abs2p < cr) {
            if (czero(dp)) return;
            if (abs2p < 0.01 * cr) return;
            good = true;
        } else {
            good = false;
        }
        dc dx;
        if (czero(dp)) dx = cscale(cabs_(root) + 1.0, escape_dir(jump(i % 10) * 2 * 3.14159265358979323846));
        else dx = cdiv(p, dp);
        dc nr = csub(root, dx);
        if (ceq(nr, root)) return;
        if (good) { root = nr; return; }
        if (i % 10 == 0) nr = csub(root, cscale(jump((i / 10 - 1) % 10), dx));
        root = nr;
    }
}

// Find one root of the degree-N leading block of p2 from a cold start, then
// divide it out in place (SkowronGould.cpp:123-155).
template <int N>
__device__ __forceinline__ dc deflate_step(dc* p2)
{
    dc root{0.0, 0.0};
    if (!laguerre2newton<N>(p2, root)) {
        PolyN<N> pn;
#pragma unroll
        for (int i = 0; i <= N; ++i) pn.c[i] = p2[i];
        root = laguerre_fallback<N>(pn, dc{0.0, 0.0});
    }
    dc coef = p2[N];
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        const dc prev = p2[i];
        p2[i] = coef;
        coef = cadd(prev, cmul(root, coef));
    }
    return root;
}

// Direct quadratic tail (solve_quadratic_eq, SkowronGould.cpp:1132-1154).
__device__ __forceinline__ void quadratic(dc& x0, dc& x1, const dc* poly)
{
    const dc a = poly[2];
    const dc b = poly[1];
    const dc c = poly[0];
    const dc b2 = cmul(b, b);
    const dc delta = csqrt_sg(csub(b2, cmul(cscale(4.0, a), c)));
    const double dot = b.re * delta.re + b.im * delta.im;
    dc r0 = (dot >= 0.0) ? cscale(-0.5, cadd(b, delta)) : cscale(-0.5, csub(b, delta));
    dc r1;
    if (czero(r0)) {
        r1 = dc{0.0, 0.0};
    } else {
        r1 = cdiv(c, r0);
        r0 = cdiv(r0, a);
    }
    x0 = r0;
    x1 = r1;
}

} // namespace sg

namespace sg {

// newton_polish as one out-of-line copy: the solvers polish several roots
// with the same code, and inlining it once per root made the point-source
// kernel larger than the instruction cache (its largest stall was waiting
// for instructions).  The polynomial goes by value, so no caller's
// coefficients need an address.
template <int N>
__device__ __noinline__ dc polish_root(const PolyN<N> pn, dc root)
{
    newton_polish<N>(pn.c, root);
    return root;
}

} // namespace sg

// All five roots of the binary-lens quintic, cold start, polished.
__device__ __forceinline__ void roots5(const dc* poly, dc* roots)
{
    dc p2[6];
    sg::PolyN<5> pn;
#pragma unroll
    for (int i = 0; i < 6; ++i) p2[i] = pn.c[i] = poly[i];
    roots[4] = sg::deflate_step<5>(p2);
    roots[3] = sg::deflate_step<4>(p2);
    roots[2] = sg::deflate_step<3>(p2);
    sg::quadratic(roots[1], roots[0], p2);
#pragma unroll
    for (int n = 0; n < 4; ++n) roots[n] = sg::polish_root<5>(pn, roots[n]);
}

// All four roots of a quartic (critical-curve polynomial), cold start, polished.
__device__ __forceinline__ void roots4(const dc* poly, dc* roots)
{
    dc p2[5];
    sg::PolyN<4> pn;
#pragma unroll
    for (int i = 0; i < 5; ++i) p2[i] = pn.c[i] = poly[i];
    roots[3] = sg::deflate_step<4>(p2);
    roots[2] = sg::deflate_step<3>(p2);
    sg::quadratic(roots[1], roots[0], p2);
#pragma unroll
    for (int n = 0; n < 3; ++n) roots[n] = sg::polish_root<4>(pn, roots[n]);
}

} // namespace lcbi
