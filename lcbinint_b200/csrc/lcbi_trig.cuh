// Correctly rounded sine and cosine of one FP64 argument, the same on the
// device and the host.
//
// The polar inverse ray places its cell centres at radius * (cos phi, sin phi)
// and weights each cell by a limb-darkening table entry picked by rounding
// |image - source|^2 / rho^2 to the nearest of 4096 steps; the reference
// evaluates these angles with the host C library
// (finite_source_magnifier.cpp:1198-1203, std::cos / std::sin).  An angle one
// unit in the last place away moves a cell centre by about 1e-16 and can move
// a cell into the next table entry, which changes a polar magnification by
// about 1e-11.  The host library's results are, up to very rare cases,
// correctly rounded, so these functions round correctly too: the argument is
// reduced by pi/2 carried to 185 bits (Cody & Waite splitting, exact products
// for |x| < 2^20 pi/2), the Taylor series of sin and cos about 0 is summed in
// double-double arithmetic (Dekker 1971; its high-order terms, below 2^-50 of
// the sum, in plain FP64), and the double-double result is rounded once.  Its
// error is below about 2^-100 relative, so the rounding is wrong only for
// arguments whose exact value lies that close to a rounding midpoint.
//
// Every operation is a separately rounded IEEE add or multiply or an
// explicit fma(); the file must be compiled without floating-point
// contraction (nvcc --fmad=false, g++ -ffp-contract=off), which the
// two_sum steps rely on.  Constants: gen_trig_constants.py.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define LCBI_TRIG_FN __host__ __device__ __forceinline__
#else
#define LCBI_TRIG_FN inline
#endif

namespace lcbi {
namespace trig {

struct DD {
    double hi, lo;
};

LCBI_TRIG_FN DD two_sum(double a, double b)
{
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

// |a| >= |b| (or a == 0).
LCBI_TRIG_FN DD quick_two_sum(double a, double b)
{
    const double s = a + b;
    return {s, b - (s - a)};
}

LCBI_TRIG_FN DD dd_mul(DD a, DD b)
{
    const double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e = fma(a.hi, b.lo, e);
    e = fma(a.lo, b.hi, e);
    return quick_two_sum(p, e);
}

LCBI_TRIG_FN DD dd_add(DD a, DD b)
{
    DD s = two_sum(a.hi, b.hi);
    const DD t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = quick_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return quick_two_sum(s.hi, s.lo);
}

LCBI_TRIG_FN DD dd_add_d(DD a, double b)
{
    DD s = two_sum(a.hi, b);
    s.lo += a.lo;
    return quick_two_sum(s.hi, s.lo);
}

// pi/2 = kP1 + kP2 + kP3 + kP4 + kP5 (kP1..kP4: 33 significant bits each).
constexpr double kP1 = 0x1.921fb54400000p+0;
constexpr double kP2 = 0x1.0b4611a600000p-34;
constexpr double kP3 = 0x1.3198a2e000000p-69;
constexpr double kP4 = 0x1.b839a25200000p-104;
constexpr double kP5 = 0x1.27044533e63a0p-142;
constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;

// (-1)^n / (2n+1)!: n = 0..7 as double-double, 8..13 as doubles.
#define LCBI_SIN_DD(n) \
    ((n) == 0 ? DD{0x1.0000000000000p+0, 0.0} : \
     (n) == 1 ? DD{-0x1.5555555555555p-3, -0x1.5555555555555p-57} : \
     (n) == 2 ? DD{0x1.1111111111111p-7, 0x1.1111111111111p-63} : \
     (n) == 3 ? DD{-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73} : \
     (n) == 4 ? DD{0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73} : \
     (n) == 5 ? DD{-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80} : \
     (n) == 6 ? DD{0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87} : \
                DD{-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97})
constexpr double kSin8 = 0x1.952c77030ad4ap-49;
constexpr double kSin9 = -0x1.2f49b46814157p-57;
constexpr double kSin10 = 0x1.71b8ef6dcf572p-66;
constexpr double kSin11 = -0x1.761b41316381ap-75;
constexpr double kSin12 = 0x1.3f3ccdd165fa9p-84;
constexpr double kSin13 = -0x1.d1ab1c2dccea3p-94;

// (-1)^n / (2n)!: n = 0..8 as double-double, 9..14 as doubles.
#define LCBI_COS_DD(n) \
    ((n) == 0 ? DD{0x1.0000000000000p+0, 0.0} : \
     (n) == 1 ? DD{-0x1.0000000000000p-1, 0.0} : \
     (n) == 2 ? DD{0x1.5555555555555p-5, 0x1.5555555555555p-59} : \
     (n) == 3 ? DD{-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65} : \
     (n) == 4 ? DD{0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76} : \
     (n) == 5 ? DD{-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76} : \
     (n) == 6 ? DD{0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83} : \
     (n) == 7 ? DD{-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92} : \
                DD{0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101})
constexpr double kCos9 = -0x1.6827863b97d97p-53;
constexpr double kCos10 = 0x1.e542ba4020225p-62;
constexpr double kCos11 = -0x1.0ce396db7f853p-70;
constexpr double kCos12 = 0x1.f2cf01972f578p-80;
constexpr double kCos13 = -0x1.88e85fc6a4e5ap-89;
constexpr double kCos14 = 0x1.0a18a2635085dp-98;

// sin and cos of r (|r| <= pi/4 (1 + 2^-20)) as double-double, r given as one.
// Truncation: the first omitted terms are below 1.3e-34 (sin) and 3.8e-33
// (cos) of the sums.
LCBI_TRIG_FN void sincos_reduced(DD r, DD* s, DD* c)
{
    const DD r2 = dd_mul(r, r);
    const double x = r2.hi;
    // sin r = r (sum_n (-1)^n r^2n / (2n+1)!)
    double ts = kSin13;
    ts = fma(ts, x, kSin12);
    ts = fma(ts, x, kSin11);
    ts = fma(ts, x, kSin10);
    ts = fma(ts, x, kSin9);
    ts = fma(ts, x, kSin8);
    DD as{ts, 0.0};
#pragma unroll
    for (int n = 7; n >= 0; --n) as = dd_add(dd_mul(as, r2), LCBI_SIN_DD(n));
    *s = dd_mul(r, as);
    // cos r = sum_n (-1)^n r^2n / (2n)!
    double tc = kCos14;
    tc = fma(tc, x, kCos13);
    tc = fma(tc, x, kCos12);
    tc = fma(tc, x, kCos11);
    tc = fma(tc, x, kCos10);
    tc = fma(tc, x, kCos9);
    DD ac{tc, 0.0};
#pragma unroll
    for (int n = 8; n >= 0; --n) ac = dd_add(dd_mul(ac, r2), LCBI_COS_DD(n));
    *c = ac;
}

// Correctly rounded (up to cases closer than about 2^-100 relative to a
// rounding midpoint) sin x and cos x for finite |x| < 2^20 pi/2.
LCBI_TRIG_FN void sincos_cr(double x, double* sn, double* cs)
{
    const double k = rint(x * kTwoOverPi);
    // x - k kP1 is exact: k kP1 has at most 53 significant bits and lies
    // within a factor two of x whenever k != 0 (Sterbenz).
    const double r0 = x - k * kP1;
    DD r = two_sum(r0, -(k * kP2));
    r = dd_add_d(r, -(k * kP3));
    r = dd_add_d(r, -(k * kP4));
    r = dd_add_d(r, -(k * kP5));
    DD s, c;
    sincos_reduced(r, &s, &c);
    const double sv = s.hi + s.lo;  // the double-double is normalised: this is s.hi
    const double cv = c.hi + c.lo;
    switch (static_cast<int>(static_cast<long long>(k) & 3)) {
    case 0: *sn = sv; *cs = cv; break;
    case 1: *sn = cv; *cs = -sv; break;
    case 2: *sn = -sv; *cs = -cv; break;
    default: *sn = -cv; *cs = sv; break;
    }
}

} // namespace trig
} // namespace lcbi
