// Complex polynomial roots on the device: the Skowron & Gould (2012) scheme
// (Laguerre / second-order general / Newton regimes, deflation, direct
// quadratic tail, Newton polish on the full polynomial), as the reference
// drives it through cmplx_roots_gen (third_party/skowron_gould/SkowronGould.cpp:79-168)
// with a cold start and polishing on.
//
// One thread solves one polynomial.  The largest degree is a template
// parameter so every Horner loop unrolls and all coefficients stay in
// registers.  The quintic's solves of the deflation degrees run as one loop
// of evaluations (deflation_chain), so the lanes of a warp share them whatever
// regime or degree each lane is in; the quartic's run as the method's loops,
// one degree after the other (laguerre2newton, deflate_step).  Both forms make
// the same steps.  Each regime is bounded (80 steps, as in the method), so a
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

// Degree-n Horner evaluation over coefficients poly[0..n] held in an array of
// M + 1 registers (n <= M): the steps of horner<n, true> in the same order,
// the steps above n skipped, so lanes of one warp at different degrees share
// one copy of the code.
template <int M>
__device__ __forceinline__ void horner_upto(const dc* poly, int n, dc z, dc& p, dc& dp, dc& d2, double& ek,
                                            bool with_ek)
{
    dc lead = poly[M];
#pragma unroll
    for (int k = 0; k < M; ++k)
        if (n == k) lead = poly[k];
    ek = cabs_(lead);
    const double absroot = cabs_(z);
    p = lead;
    dp = dc{0.0, 0.0};
    d2 = dc{0.0, 0.0};
#pragma unroll
    for (int k = M; k >= 1; --k) {
        if (k <= n) {
            d2 = cadd(dp, cmul(d2, z));
            dp = cadd(p, cmul(dp, z));
            p = cadd(poly[k - 1], cmul(p, z));
            if (with_ek) ek = absroot * ek + cabs_(p);
        }
    }
}

// The Laguerre constants 1/n, (n - 1)/n and 2/((n - 1)/n), as the method
// forms them for degree n (each rounded once, as the compiler folds them).
__device__ __forceinline__ void laguerre_constants(int n, double& one_nth, double& n_1_nth, double& two_n_div_n_1)
{
    constexpr double o5 = 1.0 / 5, o4 = 1.0 / 4, o3 = 1.0 / 3;
    constexpr double m5 = 4 * o5, m4 = 3 * o4, m3 = 2 * o3;
    constexpr double t5 = 2.0 / m5, t4 = 2.0 / m4, t3 = 2.0 / m3;
    one_nth = n == 5 ? o5 : (n == 4 ? o4 : o3);
    n_1_nth = n == 5 ? m5 : (n == 4 ? m4 : m3);
    two_n_div_n_1 = n == 5 ? t5 : (n == 4 ? t4 : t3);
}

// State of one three-regime solve (cmplx_laguerre2newton,
// SkowronGould.cpp:764-1130).  The method runs three loops in turn: Laguerre
// (mode 2, steps i = 1..80), the second-order general step (mode 1,
// i = j..80) and Newton (mode 0, 11 steps from i = j, then back to Laguerre,
// at most 64 times).  Here one trip is one step of whichever loop (mode, i, j)
// names, with that step's decisions and arithmetic.
struct RegimeState {
    dc root;
    double cr;
    int iter, mode, i, j, pass;
};

__device__ __forceinline__ RegimeState regime_start()
{
    return RegimeState{dc{0.0, 0.0}, 0.0, 0, 2, 1, 1, 0};
}

enum : int { kTripGoOn = 0, kTripConverged = 1, kTripFailed = 2 };

template <int M>
__device__ __forceinline__ int regime_trip(const dc* poly, int n, double one_nth, double n_1_nth,
                                           double two_n_div_n_1, RegimeState& st)
{
    // The Adams bound is formed on every Laguerre step, on the first step of
    // each ten of the second-order regime and on the first Newton step.
    const bool fresh = (st.mode == 2) || (st.mode == 1 ? ((st.i - st.j) % 10 == 0) : (st.i == st.j));
    dc p, dp, d2;
    double ek;
    horner_upto<M>(poly, n, st.root, p, dp, d2, ek, fresh);
    if (fresh) st.cr = crit2(ek);
    const double cr = st.cr;
    const int i = st.i;
    const double abs2p = cnorm2(p);
    ++st.iter;
    if (abs2p == 0.0) return kTripConverged;
    bool good = false;
    if (abs2p < cr) {
        if (st.mode != 2 && czero(dp)) return kTripConverged;
        if (abs2p < 0.01 * cr) return kTripConverged;
        good = true;
    }
    const int step_mode = st.mode;
    const dc root = st.root;
    dc dx;
    if (step_mode == 2) {
        dc denom{0.0, 0.0}, fn{0.0, 0.0};
        if (!czero(dp)) {
            fn = cdiv(p, dp);
            const dc fe = cdiv(d2, dp);
            const dc fh = cmul(fn, fe);
            const double a2f = cnorm2(fh);
            if (a2f <= 0.0625) st.mode = (a2f <= 0.000625) ? 0 : 1;
            const dc t = cscale(two_n_div_n_1, fh);
            const dc ds = csqrt_sg(dc{1.0 - t.re, 0.0 - t.im});
            const dc nd = cscale(n_1_nth, ds);
            denom = (ds.re > 0.0) ? dc{one_nth + nd.re, 0.0 + nd.im} : dc{one_nth - nd.re, 0.0 - nd.im};
        }
        if (czero(denom)) {
            const dc e = escape_dir(jump(i % 10) * 2 * 3.14159265358979323846);
            dx = dc{(cabs_(root) + 1.0) + e.re, e.im};
        } else {
            dx = cdiv(fn, denom);
        }
    } else if (step_mode == 1) {
        if (czero(dp)) {
            dx = cscale(cabs_(root) + 1.0, escape_dir(jump(i % 10) * 2 * 3.14159265358979323846));
        } else {
            const dc fn = cdiv(p, dp);
            const dc fe = cdiv(d2, dp);
            const dc fh = cmul(fn, fe);
            if (cnorm2(fh) <= 0.000625) st.mode = 0;
            dx = cmul(fn, dc{1.0 + fh.re, 0.0 + fh.im});
        }
    } else {
        if (czero(dp)) dx = cscale(cabs_(root) + 1.0, escape_dir(2 * 3.14159265358979323846 * jump(i % 10)));
        else dx = cdiv(p, dp);
    }
    dc nr = csub(root, dx);
    if (ceq(nr, root)) return kTripConverged;
    if (good) { st.root = nr; return kTripConverged; }
    if (step_mode == 0) {
        // Newton takes no cycle-breaking jump; after its 11th step the method
        // gives up once 80 evaluations are spent, else returns to Laguerre.
        st.root = nr;
        if (++st.i > st.j + 10) {
            if (st.iter >= kMaxIt) return kTripFailed;
            if (++st.pass >= 64) return kTripFailed;
            st.mode = 2;
            st.i = 1;
        }
        return kTripGoOn;
    }
    if (st.mode != step_mode) {
        // Regime switch: the next regime starts at the following step index,
        // unless this step was the last one.
        st.root = nr;
        if (i >= kMaxIt) return kTripFailed;
        st.j = i + 1;
        st.i = st.j;
        return kTripGoOn;
    }
    if (i % 10 == 0) nr = csub(root, cscale(jump((i / 10 - 1) % 10), dx));
    st.root = nr;
    if (++st.i > kMaxIt) return kTripFailed;
    return kTripGoOn;
}

// The plain-Laguerre fallback for the degree-n leading block of p2.
template <int N, int M>
__device__ __forceinline__ void fallback_if(const dc* p2, int n, dc& root)
{
    if constexpr (N <= M) {
        if (n == N) {
            PolyN<N> pn;
#pragma unroll
            for (int i = 0; i <= N; ++i) pn.c[i] = p2[i];
            root = laguerre_fallback<N>(pn, dc{0.0, 0.0});
        }
    }
}

// Divides the root out of the degree-n leading block of p2 in place
// (SkowronGould.cpp:145-155): the steps of the degree-n deflation, the
// entries above n untouched.
template <int M>
__device__ __forceinline__ void deflate_upto(dc* p2, int n, dc root)
{
    dc coef = p2[M];
#pragma unroll
    for (int k = 0; k < M; ++k)
        if (n == k) coef = p2[k];
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        if (i < n) {
            const dc prev = p2[i];
            p2[i] = coef;
            coef = cadd(prev, cmul(root, coef));
        }
    }
}

// Roots of degrees M, M - 1, ..., 3 of p2 from cold starts, each divided out
// before the next is sought (cmplx_roots_gen, SkowronGould.cpp:123-155);
// the root of degree n goes to roots[n - 1] and p2[0..2] is left holding the
// quadratic.  The solves run as one loop of regime trips, so a lane that has
// found its root deflates and starts the next degree while the others go on,
// and a warp's lanes share the polynomial evaluations.
template <int M>
__device__ __forceinline__ void deflation_chain(dc* p2, dc* roots)
{
    int n = M;
    double one_nth, n_1_nth, two_n_div_n_1;
    laguerre_constants(n, one_nth, n_1_nth, two_n_div_n_1);
    RegimeState st = regime_start();
    // Each degree's solve ends (converged or failed) within a bounded number
    // of trips, and every end lowers n.
    for (;;) {
        const int r = regime_trip<M>(p2, n, one_nth, n_1_nth, two_n_div_n_1, st);
        if (r == kTripGoOn) continue;
        dc root = st.root;
        if (r == kTripFailed) {
            fallback_if<5, M>(p2, n, root);
            fallback_if<4, M>(p2, n, root);
            fallback_if<3, M>(p2, n, root);
        }
        deflate_upto<M>(p2, n, root);
#pragma unroll
        for (int k = 0; k < M; ++k)
            if (k == n - 1) roots[k] = root;
        if (--n < 3) break;
        laguerre_constants(n, one_nth, n_1_nth, two_n_div_n_1);
        st = regime_start();
    }
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

// Three-regime solver (cmplx_laguerre2newton, SkowronGould.cpp:764-1130) for
// one degree, its regimes as three loops run in turn, starting in Laguerre
// mode from `root`.  Returns false on non-convergence.  The quartic solves of
// the caustic sampling use this form: the phases a warp takes lie side by side
// on one critical curve and need about as many steps each, so the fused loop
// of deflation_chain saves them little and costs its predicated steps
// (caustic sampling of the 1,024-model orbital batch: 577 ms with this form,
// 630 ms fused).
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
    sg::deflation_chain<5>(p2, roots);
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
