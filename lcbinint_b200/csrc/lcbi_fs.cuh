// Finite-source device helpers: lens map, Jacobian, limb darkening, caustic
// geometry.  Each function names the reference routine it reproduces in
// src/lcbinint/magnification/finite_source_magnifier.cpp (FSM) and keeps its
// operation order (compiled with --fmad=false) so decisions and sums match the
// reference bit for bit.
#pragma once

#include "lcbi_ps.cuh"

#include <climits>

namespace lcbi {

constexpr double kPi = 3.14159265358979323846;
constexpr int kLdTable = 20000;
constexpr int kRowKeyOffset = 2000000;
constexpr int kCausticGrid = 128;

struct P2 {
    double x, y;
};

__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000ll); }
__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000ll); }

// static_cast<int>(double) as the reference's x86-64 build evaluates it
// (cvttsd2si): NaN and out-of-range values give INT_MIN.  Grid queries with
// the 1e18*rho search radius of lcbinint.binary_inverse_ray depend on it.
__device__ __forceinline__ int to_int_x86(double v)
{
    if (!(v > -2147483649.0 && v < 2147483648.0)) return INT_MIN;
    return static_cast<int>(v);
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
__device__ __forceinline__ double clampd(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }

// Lens frame of make_binary_lens_mapper (FSM:43-52): m1 at a, m2 at 0.
struct Mapper {
    double a, m1, m2;
};

__device__ __forceinline__ Mapper make_mapper(double separation, double mass_ratio)
{
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const double m1 = 1.0 / (1.0 + q);
    return Mapper{q_in < 1.0 ? -s : s, m1, q * m1};
}

__device__ __forceinline__ double dist2(P2 a, P2 b)
{
    const double dx = a.x - b.x;
    const double dy = a.y - b.y;
    return dx * dx + dy * dy;
}

// map_binary_lens_real (FSM:278-291): image -> source plane (centre-of-mass frame).
__device__ __forceinline__ P2 map_real(const Mapper& m, double x, double y)
{
    const double xa = x - m.a;
    const double den1 = xa * xa + y * y;
    const double den2 = x * x + y * y;
    return P2{x - m.m1 * xa / den1 - m.m2 * x / den2 - m.a * m.m1, y - m.m1 * y / den1 - m.m2 * y / den2};
}

// mapped_binary_lens_distance2 (FSM:65-80).
__device__ __forceinline__ double mapped_dist2(const Mapper& m, double x, double y, P2 src)
{
    const double xa = x - m.a;
    const double den1 = xa * xa + y * y;
    const double den2 = x * x + y * y;
    const double mx = x - m.m1 * xa / den1 - m.m2 * x / den2 - m.a * m.m1;
    const double my = y - m.m1 * y / den1 - m.m2 * y / den2;
    const double dx = mx - src.x;
    const double dy = my - src.y;
    return dx * dx + dy * dy;
}

// FP32 ray map about an image-centred anchor Z (FP64): the map of a cell
// z = Z + d is the FP64 map at Z plus a difference formed in FP32,
//   w(Z + d) - w(Z) = d + m1 conj(d / (U1 (U1 + d))) + m2 conj(d / (U2 (U2 + d))),
// U1 = Z - a, U2 = Z (from 1/conj(U + d) - 1/conj(U) = -conj(d / (U (U + d)))),
// so the FP32 rounding is relative to the cell's offset from the anchor, not
// to its position, and the squared distance to the source is accumulated
// from the anchor's FP64 offset.  Used only when a context asks for FP32 rays.
struct Anchor32 {
    double zx, zy;           // anchor
    float wx, wy;            // map(anchor) - source
    float u1x, u1y, u2x, u2y;
    float m1, m2;
};

__device__ __forceinline__ Anchor32 make_anchor32(const Mapper& m, double zx, double zy, P2 src)
{
    Anchor32 A;
    A.zx = zx;
    A.zy = zy;
    const P2 w = map_real(m, zx, zy);
    A.wx = static_cast<float>(w.x - src.x);
    A.wy = static_cast<float>(w.y - src.y);
    A.u1x = static_cast<float>(zx - m.a);
    A.u1y = static_cast<float>(zy);
    A.u2x = static_cast<float>(zx);
    A.u2y = static_cast<float>(zy);
    A.m1 = static_cast<float>(m.m1);
    A.m2 = static_cast<float>(m.m2);
    return A;
}

// m conj(d / (U (U + d))) for one lens.
__device__ __forceinline__ void anchor_term(float ux, float uy, float m, float dx, float dy, float* tx, float* ty)
{
    const float vx = ux + dx, vy = uy + dy;
    const float px = ux * vx - uy * vy, py = ux * vy + uy * vx;
    const float f = m / (px * px + py * py);
    *tx = (dx * px + dy * py) * f;
    *ty = (dx * py - dy * px) * f;
}

__device__ __forceinline__ float anchored_dist2(const Anchor32& A, double x, double y)
{
    const float dx = static_cast<float>(x - A.zx), dy = static_cast<float>(y - A.zy);
    float t1x, t1y, t2x, t2y;
    anchor_term(A.u1x, A.u1y, A.m1, dx, dy, &t1x, &t1y);
    anchor_term(A.u2x, A.u2y, A.m2, dx, dy, &t2x, &t2y);
    const float ex = A.wx + (dx + t1x + t2x);
    const float ey = A.wy + (dy + t1y + t2y);
    return ex * ex + ey * ey;
}

// Jacobian determinant 1 - |m1/u1^2 + m2/u2^2|^2 of the cell, in FP32.
__device__ __forceinline__ float anchored_jacobian(const Anchor32& A, double x, double y)
{
    const float dx = static_cast<float>(x - A.zx), dy = static_cast<float>(y - A.zy);
    const float ax = A.u1x + dx, ay = A.u1y + dy, bx = A.u2x + dx, by = A.u2y + dy;
    const float ia = 1.0f / (ax * ax + ay * ay), ib = 1.0f / (bx * bx + by * by);
    // m / u^2 = m conj(u)^2 / |u|^4
    const float re = A.m1 * (ax * ax - ay * ay) * ia * ia + A.m2 * (bx * bx - by * by) * ib * ib;
    const float im = -2.0f * (A.m1 * ax * ay * ia * ia + A.m2 * bx * by * ib * ib);
    return 1.0f - (re * re + im * im);
}

// evaluate_binary_lens_cell (FSM:121-153): distance and Jacobian sharing denominators.
__device__ __forceinline__ double eval_cell(const Mapper& m, double x, double y, P2 src, double* jac)
{
    const double xa = x - m.a;
    const double y2 = y * y;
    const double den1 = xa * xa + y2;
    const double den2 = x * x + y2;
    const double i1 = 1.0 / den1;
    const double i2 = 1.0 / den2;
    const double mx = x - m.m1 * xa * i1 - m.m2 * x * i2 - m.a * m.m1;
    const double my = y - m.m1 * y * i1 - m.m2 * y * i2;
    const double dx = mx - src.x;
    const double dy = my - src.y;
    double j = 0.0;
    if (den1 >= 1.0e-20 && den2 >= 1.0e-20) {
        const double i1s = i1 * i1;
        const double i2s = i2 * i2;
        const double re = m.m1 * (xa * xa - y2) * i1s + m.m2 * (x * x - y2) * i2s;
        const double im = -2.0 * y * (m.m1 * xa * i1s + m.m2 * x * i2s);
        j = 1.0 - re * re - im * im;
    }
    *jac = j;
    return dx * dx + dy * dy;
}

// binary_jacobian (FSM:196-209).
__device__ __forceinline__ double jacobian(const Mapper& m, double x, double y)
{
    const double xa = x - m.a;
    const double den1 = xa * xa + y * y;
    const double den2 = x * x + y * y;
    if (den1 < 1.0e-20 || den2 < 1.0e-20) return 0.0;
    const double d1s = den1 * den1;
    const double d2s = den2 * den2;
    const double re = m.m1 * (xa * xa - y * y) / d1s + m.m2 * (x * x - y * y) / d2s;
    const double im = -2.0 * y * (m.m1 * xa / d1s + m.m2 * x / d2s);
    return 1.0 - re * re - im * im;
}

__device__ __forceinline__ int sign_of(double j) { return j > 0.0 ? 1 : j < 0.0 ? -1 : 0; }

// point_segment_distance (FSM:330-342).
__device__ __forceinline__ double seg_dist(P2 p, P2 a, P2 b)
{
    const double dx = b.x - a.x;
    const double dy = b.y - a.y;
    const double l2 = dx * dx + dy * dy;
    if (l2 == 0.0) return sqrt(dist2(p, a));
    const double t = clampd(((p.x - a.x) * dx + (p.y - a.y) * dy) / l2, 0.0, 1.0);
    return hypot_borges(p.x - (a.x + t * dx), p.y - (a.y + t * dy));
}

// ----- limb darkening (FSM:344-384, 3979-4012) -----
__device__ __forceinline__ double flux_factor(double c, double d) { return 1.0 - c / 3.0 - d / 5.0; }

__device__ __forceinline__ double source_flux(double rho, double c, double d)
{
    const double ff = flux_factor(c, d);
    if (ff <= 0.0 || !isfinite(ff)) return dnan();
    return kPi * rho * rho * ff;
}

__device__ __forceinline__ double ld_gamma(double c, double d)
{
    const double den = 15.0 - 5.0 * c - 3.0 * d;
    return den == 0.0 ? 0.0 : 10.0 * c / den;
}

__device__ __forceinline__ double ld_lambda(double c, double d)
{
    const double den = 15.0 - 5.0 * c - 3.0 * d;
    return den == 0.0 ? 0.0 : 12.0 * d / den;
}

__host__ __device__ __forceinline__ double surface_brightness(double r2, double c, double d)
{
    const double b = (r2 < 0.0) ? 0.0 : (1.0 < r2) ? 1.0 : r2;
    const double t = 1.0 - b;
    const double mu = sqrt((0.0 < t) ? t : 0.0);
    return 1.0 - c * (1.0 - mu) - d * (1.0 - sqrt(mu));
}

// Nearest-entry lookup in the 20,001-entry table of I(r^2) (FSM:4001-4012).
__device__ __forceinline__ double ld_lookup(const double* __restrict__ table, double r2)
{
    if (r2 <= 0.0) return table[0];
    if (r2 >= 1.0) return table[kLdTable];
    return __ldg(table + static_cast<int>(r2 * static_cast<double>(kLdTable) + 0.5));
}

// The same lookup in a copy of the table held in shared memory.
__device__ __forceinline__ double ld_lookup_shared(const double* table, double r2)
{
    if (r2 <= 0.0) return table[0];
    if (r2 >= 1.0) return table[kLdTable];
    return table[static_cast<int>(r2 * static_cast<double>(kLdTable) + 0.5)];
}

// ----- critical curve (FSM:528-567) -----

// critical_curve_polynomial_coefficients with std::complex product semantics.
__device__ __forceinline__ void critical_poly(double separation, double mass_ratio, dc phase, dc* c)
{
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const dc a{q_in < 1.0 ? -s : s, 0.0};
    const dc m1{1.0 / (1.0 + q), 0.0};
    const dc m2{m1.re * q, m1.im * q};
    const dc a2 = cmul(a, a);
    c[0] = cmul(m2, a2);
    c[1] = cmul(dc{m2.re * -2.0, m2.im * -2.0}, a);
    c[2] = csub(cadd(m1, m2), cmul(phase, a2));
    c[3] = cmul(dc{phase.re * 2.0, phase.im * 2.0}, a);
    c[4] = dc{-phase.re, -phase.im};
}

// The four critical-curve roots at one phase e^{i phi} (given as cos, sin).
__device__ __forceinline__ void critical_roots(double s, double q, dc phase, dc* roots)
{
    dc c[5];
    critical_poly(s, q, phase, c);
    roots4(c, roots);
}

// PointSourceMagnifier::binary_lens_equation (point_source_magnifier.cpp:780-792)
// with std::complex division (Smith's algorithm), used by the caustic cache.
__device__ __forceinline__ P2 lens_equation_complex(double separation, double mass_ratio, dc z)
{
    const double s = fabs(separation);
    const double q_in = fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const dc a{q_in < 1.0 ? -s : s, 0.0};
    const dc m1{1.0 / (1.0 + q), 0.0};
    const dc m2{m1.re * q, m1.im * q};
    const dc zc{z.re, -z.im};
    const dc t1 = cdiv_smith(m1, csub(zc, a));
    const dc t2 = cdiv_smith(m2, zc);
    const dc sh = csub(csub(z, t1), t2);
    const dc src = csub(sh, cmul(a, m1));
    return P2{src.re, src.im};
}

// ----- shared tables and per-call descriptors -----

// Host-computed cos/sin tables, so every fixed angle matches the host C
// library bit for bit (the reference evaluates these with std::cos/std::sin).
struct TrigTables {
    const double2* seed_phase;      // 1400: polar(1, (2pi/1400) * k), seeding scan (FSM:1741-1762)
    const double2* boundary;        // 400: (cos, sin)(2pi i/400) (FSM:1578-1586)
    const double2* interior;        // 64: (cos, sin)(2pi i/64) (FSM:1605-1614)
    const double2* angular;         // 16: (cos, sin)(2pi i/16) (FSM:1538-1553)
};

// FiniteSourceSettings (finite_source_magnifier.hpp:22-38) plus the LD table slot.
struct FsSettingsDev {
    int source_bins;
    int caustic_bins;
    double grid_ratio;
    int polar_source_bins;
    double polar_grid_ratio;
    int finite_mode;
    double kinji_threshold;
    double hex_threshold;
    double adaptive_hex_threshold;
    double ld_c;
    double ld_d;
    int adaptive_source_bins;
    int max_source_bins;
    double tol;
    double reltol;
    int ld_table;  // index of this settings' LD table (20001 doubles each)
    int pad;
};

// Sampled caustic of one (s, q, caustic_bins) model (FSM:4014-4105).
struct CausticModel {
    double s, q;
    int bins;
    int phase_offset;   // into the caustic phase table (bins entries of polar(1, 2pi i/bins))
    long long branch_offset;  // 4 * bins points: branch b, sample j at branch_offset + b * bins + j
    double min_x, max_x, min_y, max_y, step_x, step_y, max_seg_len;
};

__device__ __forceinline__ int grid_cell(double v, double lo, double step)
{
    return clampi(to_int_x86((v - lo) / step), 0, kCausticGrid - 1);
}

} // namespace lcbi
