// CPU oracle (test infrastructure only): point-source restatement.  See oracle_ps.h.
#include "oracle_ps.h"

#include <cmath>
#include <limits>

namespace oracle {
namespace {

constexpr int kMaxIt = 80;            // MAXIT = MT*MR (SkowronGould.h:5-7)
constexpr double kFracErr = 2.0e-15;  // SG:500, SG:809
constexpr double kPi = 3.14159265358979323846264338327950288;
// Cycle-breaking jump fractions (SG:502-505, published with the method).
const double kJumps[10] = {0.64109297, 0.91577881, 0.25921289, 0.50487203, 0.08177045,
                           0.13653241, 0.306162, 0.37794326, 0.04618805, 0.75132137};

cplx unit_phase(double t) { return {std::cos(t), std::sin(t)}; }

// One Laguerre-family evaluation: p, p', p''/2 by Horner with the Adams (1967)
// stopping bound ek (SG:549-561).
struct Eval {
    cplx p, dp, d2;
    double ek;
};

Eval horner2(const cplx* poly, int degree, cplx root, bool with_ek)
{
    Eval e;
    e.ek = cabs(poly[degree]);
    const double absroot = cabs(root);
    e.p = poly[degree];
    e.dp = {0.0, 0.0};
    e.d2 = {0.0, 0.0};
    for (int k = degree; k >= 1; --k) {
        e.d2 = add(e.dp, mul(e.d2, root));
        e.dp = add(e.p, mul(e.dp, root));
        e.p = add(poly[k - 1], mul(e.p, root));
        if (with_ek) e.ek = absroot * e.ek + cabs(e.p);
    }
    return e;
}

Eval horner1(const cplx* poly, int degree, cplx root, bool with_ek)
{
    Eval e;
    e.ek = cabs(poly[degree]);
    const double absroot = cabs(root);
    e.p = poly[degree];
    e.dp = {0.0, 0.0};
    for (int k = degree; k >= 1; --k) {
        e.dp = add(e.p, mul(e.dp, root));
        e.p = add(poly[k - 1], mul(e.p, root));
        if (with_ek) e.ek = absroot * e.ek + cabs(e.p);
    }
    return e;
}

inline cplx minus_scaled(cplx root, double faq, cplx dx) { return sub(root, scl(faq, dx)); }

// cmplx_laguerre (SG:472-625): plain Laguerre, used only when the three-regime
// solver runs out of iterations.
void laguerre(const cplx* poly, int degree, cplx* root, bool* success)
{
    if (is_zero(poly[degree])) {
        if (degree == 0) return;
        laguerre(poly, degree - 1, root, success);
    }
    if (degree <= 1) {
        if (degree == 0) {
            *success = false;
            return;
        }
        *root = dvd(scl(-1.0, poly[0]), poly[1]);
        return;
    }
    const double one_nth = 1.0 / degree;
    const double n_1_nth = (degree - 1.0) * one_nth;
    const double two_n_div_n_1 = 2.0 / n_1_nth;
    bool good_to_go = false;
    for (int i = 1; i <= kMaxIt; ++i) {
        const double absroot = cabs(*root);
        const Eval e = horner2(poly, degree, *root, true);
        const double abs2p = norm2(e.p);
        if (abs2p == 0.0) return;
        const double crit = (kFracErr * e.ek) * (kFracErr * e.ek);
        if (abs2p < crit) {
            if (abs2p < 0.01 * crit) return;
            good_to_go = true;
        } else {
            good_to_go = false;
        }
        cplx denom = {0.0, 0.0};
        cplx fac_newton = {0.0, 0.0};
        if (!is_zero(e.dp)) {
            fac_newton = dvd(e.p, e.dp);
            const cplx fac_extra = dvd(e.d2, e.dp);
            const cplx f_half = mul(fac_newton, fac_extra);
            const cplx t = scl(two_n_div_n_1, f_half);
            const cplx ds = csqrt_sg({1.0 - t.re, 0.0 - t.im});
            const cplx nd = scl(n_1_nth, ds);
            denom = (ds.re >= 0.0) ? cplx{one_nth + nd.re, 0.0 + nd.im}
                                   : cplx{one_nth - nd.re, 0.0 - nd.im};
        }
        cplx dx;
        if (is_zero(denom)) {
            dx = scl(absroot + 1.0, unit_phase(kJumps[i % 10] * 2 * kPi));
        } else {
            dx = dvd(fac_newton, denom);
        }
        cplx newroot = sub(*root, dx);
        if (same(newroot, *root)) return;
        if (good_to_go) {
            *root = newroot;
            return;
        }
        if (i % 10 == 0) newroot = minus_scaled(*root, kJumps[(i / 10 - 1) % 10], dx);
        *root = newroot;
    }
    *success = false;
}

// cmplx_laguerre2newton (SG:764-1130): Laguerre -> second-order general -> Newton.
void laguerre2newton(const cplx* poly, int degree, cplx* root, bool* success)
{
    *success = true;
    int iter = 0;
    double crit = 0.0;
    int j = 1;
    bool good_to_go = false;
    int mode = 2;
    for (;;) {
        if (mode >= 2) {
            const double one_nth = 1.0 / degree;
            const double n_1_nth = (degree - 1) * one_nth;
            const double two_n_div_n_1 = 2.0 / n_1_nth;
            int i;
            for (i = 1; i <= kMaxIt; ++i) {
                const Eval e = horner2(poly, degree, *root, true);
                const double abs2p = norm2(e.p);
                ++iter;
                if (abs2p == 0.0) return;
                crit = (kFracErr * e.ek) * (kFracErr * e.ek);
                if (abs2p < crit) {
                    if (abs2p < 0.01 * crit) return;
                    good_to_go = true;
                } else {
                    good_to_go = false;
                }
                cplx denom = {0.0, 0.0};
                cplx fac_newton = {0.0, 0.0};
                if (!is_zero(e.dp)) {
                    fac_newton = dvd(e.p, e.dp);
                    const cplx fac_extra = dvd(e.d2, e.dp);
                    const cplx f_half = mul(fac_newton, fac_extra);
                    const double a2f = norm2(f_half);
                    if (a2f <= 0.0625) mode = (a2f <= 0.000625) ? 0 : 1;
                    const cplx t = scl(two_n_div_n_1, f_half);
                    const cplx ds = csqrt_sg({1.0 - t.re, 0.0 - t.im});
                    const cplx nd = scl(n_1_nth, ds);
                    denom = (ds.re > 0.0) ? cplx{one_nth + nd.re, 0.0 + nd.im}
                                          : cplx{one_nth - nd.re, 0.0 - nd.im};
                }
                cplx dx;
                if (is_zero(denom)) {
                    const cplx j2 = unit_phase(kJumps[i % 10] * 2 * kPi);
                    dx = {(cabs(*root) + 1.0) + j2.re, j2.im};
                } else {
                    dx = dvd(fac_newton, denom);
                }
                cplx newroot = sub(*root, dx);
                if (same(newroot, *root)) return;
                if (good_to_go) {
                    *root = newroot;
                    return;
                }
                if (mode != 2) {
                    *root = newroot;
                    j = i + 1;
                    break;
                }
                if (i % 10 == 0) newroot = minus_scaled(*root, kJumps[(i / 10 - 1) % 10], dx);
                *root = newroot;
            }
            if (i >= kMaxIt) {
                *success = false;
                return;
            }
        }
        if (mode == 1) {
            int i;
            for (i = j; i <= kMaxIt; ++i) {
                const bool fresh = ((i - j) % 10 == 0);
                const Eval e = horner2(poly, degree, *root, fresh);
                if (fresh) crit = (kFracErr * e.ek) * (kFracErr * e.ek);
                const double abs2p = norm2(e.p);
                ++iter;
                if (abs2p == 0.0) return;
                if (abs2p < crit) {
                    if (is_zero(e.dp)) return;
                    if (abs2p < 0.01 * crit) return;
                    good_to_go = true;
                } else {
                    good_to_go = false;
                }
                cplx dx;
                if (is_zero(e.dp)) {
                    dx = scl(cabs(*root) + 1.0, unit_phase(kJumps[i % 10] * 2 * kPi));
                } else {
                    const cplx fac_newton = dvd(e.p, e.dp);
                    const cplx fac_extra = dvd(e.d2, e.dp);
                    const cplx f_half = mul(fac_newton, fac_extra);
                    if (norm2(f_half) <= 0.000625) mode = 0;
                    dx = mul(fac_newton, cplx{1.0 + f_half.re, 0.0 + f_half.im});
                }
                cplx newroot = sub(*root, dx);
                if (same(newroot, *root)) return;
                if (good_to_go) {
                    *root = newroot;
                    return;
                }
                if (mode != 1) {
                    *root = newroot;
                    j = i + 1;
                    break;
                }
                if (i % 10 == 0) newroot = minus_scaled(*root, kJumps[(i / 10 - 1) % 10], dx);
                *root = newroot;
            }
            if (i >= kMaxIt) {
                *success = false;
                return;
            }
        }
        if (mode == 0) {
            for (int i = j; i <= j + 10; ++i) {
                const bool fresh = (i == j);
                const Eval e = horner1(poly, degree, *root, fresh);
                if (fresh) crit = (kFracErr * e.ek) * (kFracErr * e.ek);
                const double abs2p = norm2(e.p);
                ++iter;
                if (abs2p == 0.0) return;
                if (abs2p < crit) {
                    if (is_zero(e.dp)) return;
                    if (abs2p < 0.01 * crit) return;
                    good_to_go = true;
                } else {
                    good_to_go = false;
                }
                cplx dx;
                if (is_zero(e.dp)) {
                    dx = scl(cabs(*root) + 1.0, unit_phase(2 * kPi * kJumps[i % 10]));
                } else {
                    dx = dvd(e.p, e.dp);
                }
                const cplx newroot = sub(*root, dx);
                if (same(newroot, *root)) return;
                if (good_to_go) {
                    *root = newroot;
                    return;
                }
                *root = newroot;
            }
            if (iter >= kMaxIt) {
                *success = false;
                return;
            }
            mode = 2;
        }
    }
}

// cmplx_newton_spec (SG:626-763): Newton polish, stopping bound refreshed every 10 steps.
void newton_polish(const cplx* poly, int degree, cplx* root)
{
    bool good_to_go = false;
    double crit = 0.0;
    for (int i = 1; i <= kMaxIt; ++i) {
        const bool fresh = (i % 10 == 1);
        const Eval e = horner1(poly, degree, *root, fresh);
        if (fresh) crit = (kFracErr * e.ek) * (kFracErr * e.ek);
        const double abs2p = norm2(e.p);
        if (abs2p == 0.0) return;
        if (abs2p < crit) {
            if (is_zero(e.dp)) return;
            if (abs2p < 0.01 * crit) return;
            good_to_go = true;
        } else {
            good_to_go = false;
        }
        cplx dx;
        if (is_zero(e.dp)) {
            dx = scl(cabs(*root) + 1.0, unit_phase(kJumps[i % 10] * 2 * kPi));
        } else {
            dx = dvd(e.p, e.dp);
        }
        cplx newroot = sub(*root, dx);
        if (same(newroot, *root)) return;
        if (good_to_go) {
            *root = newroot;
            return;
        }
        if (i % 10 == 0) newroot = minus_scaled(*root, kJumps[(i / 10 - 1) % 10], dx);
        *root = newroot;
    }
}

// solve_quadratic_eq (SG:1132-1154).
void quadratic(cplx* x0, cplx* x1, const cplx* poly)
{
    const cplx a = poly[2];
    const cplx b = poly[1];
    const cplx c = poly[0];
    const cplx b2 = mul(b, b);
    const cplx delta = csqrt_sg(sub(b2, mul(scl(4.0, a), c)));
    const double dot = b.re * delta.re + b.im * delta.im;
    cplx r0 = (dot >= 0.0) ? scl(-0.5, add(b, delta)) : scl(-0.5, sub(b, delta));
    cplx r1;
    if (is_zero(r0)) {
        r1 = {0.0, 0.0};
    } else {
        r1 = dvd(c, r0);
        r0 = dvd(r0, a);
    }
    *x0 = r0;
    *x1 = r1;
}

struct Geometry {
    double a, m1, m2, a2, a3, m2_2;
    cplx y;
};

// make_fast_vbm_geometry (PSM:105-117).
Geometry make_geometry(double separation, double mass_ratio, double y1, double y2)
{
    const double s = std::fabs(separation);
    const double q_in = std::fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const double a = q_in < 1.0 ? -s : s;
    const double m1 = 1.0 / (1.0 + q);
    const double m2 = q * m1;
    const double a2 = a * a;
    return {a, m1, m2, a2, a2 * a, m2 * m2, {y1 + a * m1, y2}};
}

// binary_polynomial_coefficients (PSM:152-185), operation order preserved.
void coefficients(const Geometry& g, cplx* c)
{
    const double a = g.a;
    const double m2 = g.m2;
    const cplx y = g.y;
    const cplx yc = {y.re, -y.im};
    const double c9 = g.a2 * g.m2_2;
    const double c10 = a * m2;
    const cplx c12 = {a - yc.re, 0.0 - yc.im};
    const cplx c13 = {a + y.re, 0.0 + y.im};
    const cplx c14 = add(c13, y);
    const cplx c15 = {c14.re, -c14.im};
    const cplx c16 = scl(a, y);
    const cplx c17 = {c16.re, -c16.im};
    const cplx c18 = {c12.re, -c12.im};

    c[0] = scl(c9, y);
    {
        const cplx t1 = scl(2.0, c17);
        const cplx t2 = {t1.re - (2.0 + g.a2), t1.im - 0.0};
        const cplx t3 = mul(t2, y);
        const cplx t4 = {a + t3.re, 0.0 + t3.im};
        const cplx t5 = scl(c10, t4);
        c[1] = {-c9 + t5.re, 0.0 + t5.im};
    }
    {
        const cplx u1 = {1.0 + c16.re, 0.0 + c16.im};
        const cplx u3 = mul(scl(2.0, yc), c13);
        const cplx u5 = scl(c10, sub(u1, u3));
        const cplx v1 = {c17.re - 1.0, c17.im - 0.0};
        const cplx v3 = sub(mul(c16, c12), c18);
        c[2] = sub(u5, mul(v1, v3));
    }
    {
        const cplx w1 = scl(c10, c15);
        const cplx w3 = scl(2.0 * (1.0 + g.a2), y);
        const cplx w4 = {g.a3 + w3.re, 0.0 + w3.im};
        const cplx w6 = sub(w4, mul(c17, c14));
        const cplx w8 = add(w1, mul(w6, yc));
        c[3] = sub(w8, scl(a, c13));
    }
    {
        const cplx x1 = {c13.re + a, c13.im + 0.0};
        const cplx x2 = mul(yc, x1);
        const cplx x3 = {x2.re - 1.0, x2.im - 0.0};
        const cplx x4 = mul(c12, x3);
        c[4] = {-c10 - x4.re, 0.0 - x4.im};
    }
    c[5] = mul(yc, c12);
}

// residual_squared (PSM:187-203).
double residual2(const Geometry& g, cplx z)
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

// jacobian_determinant (PSM:205-223).
double jacobian(const Geometry& g, cplx z)
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

// select_physical_roots (PSM:225-279): drop the two worst residuals when the
// third-worst is far better (ratio 1e-8, gap 1e-24).
void select_physical(const Geometry& g, const cplx* roots, bool* physical)
{
    double r[5];
    int w1 = 0, w2 = 0, w3 = 0;
    for (int i = 0; i < 5; ++i) {
        r[i] = residual2(g, roots[i]);
        if (i == 0) {
            w1 = i;
        } else if (i == 1) {
            if (r[i] > r[w1]) {
                w2 = w1;
                w1 = i;
            } else {
                w2 = i;
            }
        } else if (i == 2) {
            if (r[i] > r[w1]) {
                w3 = w2;
                w2 = w1;
                w1 = i;
            } else if (r[i] > r[w2]) {
                w3 = w2;
                w2 = i;
            } else {
                w3 = i;
            }
        } else if (r[i] > r[w1]) {
            w3 = w2;
            w2 = w1;
            w1 = i;
        } else if (r[i] > r[w2]) {
            w3 = w2;
            w2 = i;
        } else if (r[i] > r[w3]) {
            w3 = i;
        }
    }
    const bool three = r[w2] * 1.0e-8 > r[w3] + 1.0e-24;
    for (int i = 0; i < 5; ++i) physical[i] = !(three && (i == w1 || i == w2));
}

// derivative_error_indicator_from_roots (PSM:313-359).
double derivative_indicator(const Geometry& g, const cplx* roots, const bool* physical)
{
    double indicator = 0.0;
    const cplx a = {g.a, 0.0};
    const cplx m1 = {g.m1, 0.0};
    const cplx m2 = {g.m2, 0.0};
    const double inf = std::numeric_limits<double>::infinity();
    for (int i = 0; i < 5; ++i) {
        if (!physical[i]) continue;
        const cplx z = roots[i];
        const cplx dza = sub(z, a);
        const cplx za2 = mul(dza, dza);
        const cplx zb2 = mul(z, z);
        const cplx j1 = add(dvd(m1, za2), dvd(m2, zb2));
        const cplx j1c = {j1.re, -j1.im};
        const double det_j = 1.0 - mul(j1, j1c).re;
        if (det_j == 0.0 || !std::isfinite(det_j)) return inf;
        cplx j2 = scl(-2.0, add(dvd(m1, mul(za2, dza)), dvd(m2, mul(zb2, z))));
        cplx j3 = scl(6.0, add(dvd(m1, mul(za2, za2)), dvd(m2, mul(zb2, zb2))));
        const double det_j2 = det_j * det_j;
        const cplx j1c2 = mul(j1c, j1c);
        j3 = mul(j3, j1c2);
        const double ob2 = (j2.re * j2.re + j2.im * j2.im) * (6.0 - 6.0 * det_j + det_j2);
        j2 = mul(mul(mul(j2, j2), j1c2), j1c);
        const double den = std::fabs(det_j * det_j2 * det_j2);
        if (den == 0.0 || !std::isfinite(den)) return inf;
        const double cq =
            0.5 * (std::fabs(ob2 - 6.0 * j2.re - 2.0 * j3.re * det_j) + 3.0 * std::fabs(j2.im)) / den;
        if (!std::isfinite(cq)) return inf;
        indicator += cq;
    }
    return indicator;
}

void solve_binary(const Geometry& g, cplx* roots)
{
    cplx c[6];
    coefficients(g, c);
    roots_gen(roots, c, 5, true);
}

} // namespace

void roots_gen(cplx* roots, const cplx* poly, int degree, bool polish)
{
    cplx p2[6];
    for (int i = 0; i < degree; ++i) roots[i] = {0.0, 0.0};
    for (int i = 0; i <= degree; ++i) p2[i] = poly[i];
    if (degree <= 1) {
        if (degree == 1) roots[0] = dvd(scl(-1.0, poly[0]), poly[1]);
        return;
    }
    for (int n = degree; n >= 3; --n) {
        // Start from the smallest-modulus remaining guess (all zero on a cold start).
        int small = n - 1;
        double abs_small = norm2(roots[small]);
        for (int i = 0; i < n - 1; ++i) {
            if (norm2(roots[i]) < abs_small) {
                small = i;
                abs_small = norm2(roots[i]);
            }
        }
        const cplx tmp = roots[small];
        roots[small] = roots[n - 1];
        roots[n - 1] = tmp;
        bool ok = true;
        laguerre2newton(p2, n, &roots[n - 1], &ok);
        if (!ok) {
            roots[n - 1] = {0.0, 0.0};
            laguerre(p2, n, &roots[n - 1], &ok);
        }
        // Synthetic division by (z - root).
        cplx coef = p2[n];
        for (int i = n - 1; i >= 0; --i) {
            const cplx prev = p2[i];
            p2[i] = coef;
            coef = add(prev, mul(roots[n - 1], coef));
        }
    }
    quadratic(&roots[1], &roots[0], p2);
    if (polish) {
        for (int n = 0; n < degree - 1; ++n) newton_polish(poly, degree, &roots[n]);
    }
}

PointSource binary_mag0(double separation, double mass_ratio, double y1, double y2)
{
    if (separation == 0.0 || mass_ratio <= 0.0) return {0.0, 0};
    const Geometry g = make_geometry(separation, mass_ratio, y1, y2);
    cplx roots[5];
    solve_binary(g, roots);
    bool physical[5];
    select_physical(g, roots, physical);
    double A = 0.0;
    int n = 0;
    for (int i = 0; i < 5; ++i) {
        if (!physical[i]) continue;
        A += 1.0 / std::fabs(jacobian(g, roots[i]));
        ++n;
    }
    return {A, n};
}

PointSource binary_mag0_derivatives(double separation, double mass_ratio, double y1, double y2,
                                    double* indicator)
{
    *indicator = 0.0;
    if (separation == 0.0 || mass_ratio <= 0.0) return {0.0, 0};
    const Geometry g = make_geometry(separation, mass_ratio, y1, y2);
    cplx roots[5];
    solve_binary(g, roots);
    bool physical[5];
    select_physical(g, roots, physical);
    double A = 0.0;
    int n = 0;
    for (int i = 0; i < 5; ++i) {
        if (!physical[i]) continue;
        A += 1.0 / std::fabs(jacobian(g, roots[i]));
        ++n;
    }
    *indicator = derivative_indicator(g, roots, physical);
    return {A, n};
}

int binary_image_candidates(double separation, double mass_ratio, double y1, double y2,
                            double* out)
{
    if (separation == 0.0 || mass_ratio <= 0.0) return 0;
    const Geometry g = make_geometry(separation, mass_ratio, y1, y2);
    cplx roots[5];
    solve_binary(g, roots);
    struct Row {
        double x, y, det, res;
    } rows[5];
    for (int i = 0; i < 5; ++i) {
        rows[i] = {roots[i].re, roots[i].im, jacobian(g, roots[i]), std::sqrt(residual2(g, roots[i]))};
    }
    // Stable insertion sort by residual (the order std::sort leaves 5 items in).
    for (int i = 1; i < 5; ++i) {
        const Row v = rows[i];
        int k = i;
        while (k > 0 && v.res < rows[k - 1].res) {
            rows[k] = rows[k - 1];
            --k;
        }
        rows[k] = v;
    }
    int physical = 5;
    if (rows[3].res * 1.0e-4 > rows[2].res + 1.0e-12) physical = 3;
    for (int i = 0; i < 5; ++i) {
        out[5 * i + 0] = rows[i].x;
        out[5 * i + 1] = rows[i].y;
        out[5 * i + 2] = rows[i].det;
        out[5 * i + 3] = rows[i].res;
        out[5 * i + 4] = i < physical ? 1.0 : 0.0;
    }
    return 5;
}

} // namespace oracle
