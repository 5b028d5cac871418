// CPU oracle (test infrastructure only): finite-source restatement.  See oracle_fs.h.
#include "oracle_fs.h"

#include "oracle_ps.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <deque>
#include <limits>
#include <unordered_map>
#include <utility>
#include <vector>

namespace oracle {

thread_local PolarFixedSum* g_polar_fixed = nullptr;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrtHalf = 0.70710678118654752440;
constexpr int kLdTable = 20000;
constexpr int kRowKeyOffset = 2000000;
const double kInf = std::numeric_limits<double>::infinity();
const double kNaN = std::numeric_limits<double>::quiet_NaN();

// static_cast<int>(double) as x86-64 evaluates it (cvttsd2si): out-of-range
// and NaN inputs give INT_MIN.  The reference relies on it in grid queries
// with enormous search radii (FSM:4201-4216 with kinji_threshold = 1e18).
int to_int(double v)
{
    if (!(v > -2147483649.0 && v < 2147483648.0)) return INT_MIN;
    return static_cast<int>(v);
}

template <typename T>
T clampv(T v, T lo, T hi)
{
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
inline double dmin(double a, double b) { return (b < a) ? b : a; }
inline double dmax(double a, double b) { return (a < b) ? b : a; }

struct Mapper {
    double a, m1, m2;
};

// make_binary_lens_mapper (FSM:43-52).
Mapper make_mapper(double separation, double mass_ratio)
{
    const double s = std::fabs(separation);
    const double q_in = std::fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const double m1 = 1.0 / (1.0 + q);
    return {q_in < 1.0 ? -s : s, m1, q * m1};
}

// map_binary_lens_real (FSM:278-291).
Pt map_real(const Mapper& m, double x, double y)
{
    const double xa = x - m.a;
    const double den1 = xa * xa + y * y;
    const double den2 = x * x + y * y;
    return {x - m.m1 * xa / den1 - m.m2 * x / den2 - m.a * m.m1, y - m.m1 * y / den1 - m.m2 * y / den2};
}

double dist2(Pt a, Pt b)
{
    const double dx = a.x - b.x;
    const double dy = a.y - b.y;
    return dx * dx + dy * dy;
}

// mapped_binary_lens_distance2 (FSM:65-80).
double mapped_dist2(const Mapper& m, double x, double y, Pt src)
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

// evaluate_binary_lens_cell (FSM:121-153): distance and Jacobian from shared denominators.
void eval_cell(const Mapper& m, double x, double y, Pt src, double* d2, double* jac)
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
    *d2 = dx * dx + dy * dy;
    *jac = j;
}

// binary_jacobian (FSM:196-209).
double jacobian(const Mapper& m, double x, double y)
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

int jacobian_sign(const Mapper& m, double x, double y)
{
    const double j = jacobian(m, x, y);
    return j > 0.0 ? 1 : j < 0.0 ? -1 : 0;
}

// hypot of the host C library (Borges 2019, the non-fused correction).
double hyp(double x, double y) { return std::hypot(x, y); }

// point_segment_distance (FSM:330-342).
double seg_dist(Pt p, Pt a, Pt b)
{
    const double dx = b.x - a.x;
    const double dy = b.y - a.y;
    const double l2 = dx * dx + dy * dy;
    if (l2 == 0.0) return std::sqrt(dist2(p, a));
    const double t = clampv(((p.x - a.x) * dx + (p.y - a.y) * dy) / l2, 0.0, 1.0);
    return hyp(p.x - (a.x + t * dx), p.y - (a.y + t * dy));
}

// ----- limb darkening (FSM:344-384, 3979-4012) -----
double flux_factor(const FsSettings& st) { return 1.0 - st.ld_c / 3.0 - st.ld_d / 5.0; }

double ld_gamma(const FsSettings& st)
{
    const double den = 15.0 - 5.0 * st.ld_c - 3.0 * st.ld_d;
    return den == 0.0 ? 0.0 : 10.0 * st.ld_c / den;
}

double ld_lambda(const FsSettings& st)
{
    const double den = 15.0 - 5.0 * st.ld_c - 3.0 * st.ld_d;
    return den == 0.0 ? 0.0 : 12.0 * st.ld_d / den;
}

double surface_brightness(double r2, double c, double d)
{
    const double b = clampv(r2, 0.0, 1.0);
    const double mu = std::sqrt(dmax(0.0, 1.0 - b));
    return 1.0 - c * (1.0 - mu) - d * (1.0 - std::sqrt(mu));
}

double source_flux(double rho, const FsSettings& st)
{
    const double ff = flux_factor(st);
    if (ff <= 0.0 || !std::isfinite(ff)) return kNaN;
    return kPi * rho * rho * ff;
}

struct LdTable {
    std::vector<double> t;
    bool uniform;
    explicit LdTable(const FsSettings& st)
    {
        uniform = st.ld_c == 0.0 && st.ld_d == 0.0;
        t.resize(kLdTable + 1);
        for (int i = 0; i <= kLdTable; ++i)
            t[i] = surface_brightness(static_cast<double>(i) / static_cast<double>(kLdTable), st.ld_c, st.ld_d);
    }
    double operator()(double r2) const
    {
        if (r2 <= 0.0) return t[0];
        if (r2 >= 1.0) return t[kLdTable];
        return t[static_cast<int>(r2 * static_cast<double>(kLdTable) + 0.5)];
    }
};

// ----- critical curves and caustics -----

// critical_curve_polynomial_coefficients (FSM:528-545) with std::complex
// semantics (naive products for finite values).
void critical_poly(double separation, double mass_ratio, cplx phase, cplx* c)
{
    const double s = std::fabs(separation);
    const double q_in = std::fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const cplx a = {q_in < 1.0 ? -s : s, 0.0};
    const cplx m1 = {1.0 / (1.0 + q), 0.0};
    const cplx m2 = {m1.re * q, m1.im * q};
    const cplx a2 = mul(a, a);
    c[0] = mul(m2, a2);
    c[1] = mul(cplx{m2.re * -2.0, m2.im * -2.0}, a);
    c[2] = sub(add(m1, m2), mul(phase, a2));
    c[3] = mul(cplx{phase.re * 2.0, phase.im * 2.0}, a);
    c[4] = {-phase.re, -phase.im};
}

cplx polar1(double angle) { return {std::cos(angle), std::sin(angle)}; }

int critical_roots(double s, double q, double phi, cplx* roots)
{
    cplx c[5];
    critical_poly(s, q, polar1(phi), c);
    roots_gen(roots, c, 4, true);
    return 4;
}

// Smith (1962) complex quotient: libgcc's __divdc3 for finite operands.
cplx div_smith(cplx a, cplx b)
{
    const double c = b.re, d = b.im;
    if (std::fabs(c) < std::fabs(d)) {
        const double r = c / d;
        const double den = (c * r) + d;
        return {((a.re * r) + a.im) / den, ((a.im * r) - a.re) / den};
    }
    const double r = d / c;
    const double den = (d * r) + c;
    return {((a.im * r) + a.re) / den, (a.im - (a.re * r)) / den};
}

// PointSourceMagnifier::binary_lens_equation (PSM:780-792), std::complex arithmetic.
Pt lens_equation(double separation, double mass_ratio, cplx z)
{
    const double s = std::fabs(separation);
    const double q_in = std::fabs(mass_ratio);
    const double q = q_in < 1.0 ? q_in : 1.0 / q_in;
    const cplx a = {q_in < 1.0 ? -s : s, 0.0};
    const cplx m1 = {1.0 / (1.0 + q), 0.0};
    const cplx m2 = {m1.re * q, m1.im * q};
    const cplx zc = {z.re, -z.im};
    const cplx t1 = div_smith(m1, sub(zc, a));
    const cplx t2 = div_smith(m2, zc);
    const cplx shifted = sub(sub(z, t1), t2);
    const cplx src = sub(shifted, mul(a, m1));
    return {src.re, src.im};
}

bool less_by_angle(Pt l, Pt r) { return std::atan2(l.y, l.x) < std::atan2(r.y, r.x); }

// append_tracked_caustic_points (FSM:569-611).
void append_tracked(std::vector<Pt>* br, Pt* pts)
{
    if (br[0].empty()) {
        for (int i = 1; i < 4; ++i) {  // stable insertion sort by polar angle
            const Pt v = pts[i];
            int k = i;
            while (k > 0 && less_by_angle(v, pts[k - 1])) {
                pts[k] = pts[k - 1];
                --k;
            }
            pts[k] = v;
        }
        for (int i = 0; i < 4; ++i) br[i].push_back(pts[i]);
        return;
    }
    int perm[4] = {0, 1, 2, 3};
    int best[4] = {0, 1, 2, 3};
    double best_cost = kInf;
    do {
        double cost = 0.0;
        for (int i = 0; i < 4; ++i) cost += dist2(br[i].back(), pts[perm[i]]);
        if (cost < best_cost) {
            best_cost = cost;
            std::copy(perm, perm + 4, best);
        }
    } while (std::next_permutation(perm, perm + 4));
    for (int i = 0; i < 4; ++i) br[i].push_back(pts[best[i]]);
}

int grid_ix(double v, double lo, double step) { return clampv(to_int((v - lo) / step), 0, CausticCache::kGrid - 1); }

} // namespace

double ld_brightness(double c, double d, double r2)
{
    FsSettings st;
    st.ld_c = c;
    st.ld_d = d;
    return LdTable(st)(r2);
}

int critical_sources(double s, double q, double phi, Pt* out)
{
    const Mapper m = make_mapper(s, q);
    cplx r[4];
    critical_roots(s, q, phi, r);
    for (int i = 0; i < 4; ++i) out[i] = map_real(m, r[i].re, r[i].im);
    return 4;
}

void build_caustic_cache(double s, double q, int caustic_bins, CausticCache* cc)
{
    const int bins = std::max(caustic_bins, 32);
    for (auto& b : cc->branches) b.clear();
    cc->points.clear();
    cc->min_x = kInf;
    cc->max_x = -kInf;
    cc->min_y = kInf;
    cc->max_y = -kInf;
    for (int i = 0; i < bins; ++i) {
        const double phase = 2.0 * kPi * static_cast<double>(i) / static_cast<double>(bins);
        cplx r[4];
        critical_roots(s, q, phase, r);
        Pt pts[4];
        for (int k = 0; k < 4; ++k) {
            pts[k] = lens_equation(s, q, r[k]);
            cc->points.push_back(pts[k]);
            cc->min_x = dmin(cc->min_x, pts[k].x);
            cc->max_x = dmax(cc->max_x, pts[k].x);
            cc->min_y = dmin(cc->min_y, pts[k].y);
            cc->max_y = dmax(cc->max_y, pts[k].y);
        }
        append_tracked(cc->branches, pts);
    }
    const int G = CausticCache::kGrid;
    const double width = dmax(cc->max_x - cc->min_x, 1.0e-12);
    const double height = dmax(cc->max_y - cc->min_y, 1.0e-12);
    cc->step_x = width / static_cast<double>(G);
    cc->step_y = height / static_cast<double>(G);
    cc->grid.assign(G * G, {});
    for (size_t i = 0; i < cc->points.size(); ++i) {
        const Pt& p = cc->points[i];
        cc->grid[grid_ix(p.y, cc->min_y, cc->step_y) * G + grid_ix(p.x, cc->min_x, cc->step_x)].push_back(int(i));
    }
    cc->branch_grid.assign(G * G, {});
    double max_seg2 = 0.0;
    for (int b = 0; b < 4; ++b) {
        const auto& br = cc->branches[b];
        const int n = static_cast<int>(br.size());
        for (int j = 0; j < n; ++j) {
            if (j < n - 1) {
                const double seg2 = dist2(br[j], br[(j + 1) % n]);
                if (seg2 > max_seg2) max_seg2 = seg2;
            }
            cc->branch_grid[grid_ix(br[j].y, cc->min_y, cc->step_y) * G + grid_ix(br[j].x, cc->min_x, cc->step_x)]
                .push_back({b, j});
        }
    }
    cc->max_seg_len = std::sqrt(max_seg2);
}

// binary_sampled_caustic_distance (FSM:4183-4246).
double sampled_caustic_distance(const CausticCache& cc, double x, double y, double R)
{
    double d2 = kInf;
    if (R > 0.0 && (x < cc.min_x - R || x > cc.max_x + R || y < cc.min_y - R || y > cc.max_y + R)) return kInf;
    if (R > 0.0 && !cc.grid.empty()) {
        const int ix0 = grid_ix(x - R, cc.min_x, cc.step_x), ix1 = grid_ix(x + R, cc.min_x, cc.step_x);
        const int iy0 = grid_ix(y - R, cc.min_y, cc.step_y), iy1 = grid_ix(y + R, cc.min_y, cc.step_y);
        for (int iy = iy0; iy <= iy1; ++iy)
            for (int ix = ix0; ix <= ix1; ++ix)
                for (int idx : cc.grid[iy * CausticCache::kGrid + ix]) {
                    const double dx = x - cc.points[idx].x;
                    const double dy = y - cc.points[idx].y;
                    const double c = dx * dx + dy * dy;
                    if (c < d2) d2 = c;
                }
        if (d2 == kInf) return d2;
    } else {
        for (const Pt& p : cc.points) {
            const double dx = x - p.x;
            const double dy = y - p.y;
            const double c = dx * dx + dy * dy;
            if (c < d2) d2 = c;
        }
    }
    return std::sqrt(d2);
}

// binary_caustic_distance (FSM:4107-4181).
double caustic_distance(const CausticCache& cc, double x, double y, double hint)
{
    double nearest = hint;
    if (!std::isfinite(nearest)) {
        double n2 = kInf;
        for (const Pt& p : cc.points) {
            const double dx = x - p.x;
            const double dy = y - p.y;
            const double d2 = dx * dx + dy * dy;
            if (d2 < n2) n2 = d2;
        }
        nearest = std::sqrt(n2);
    }
    if (cc.branch_grid.empty()) return nearest;
    const double R = nearest + cc.max_seg_len;
    const int ix0 = grid_ix(x - R, cc.min_x, cc.step_x), ix1 = grid_ix(x + R, cc.min_x, cc.step_x);
    const int iy0 = grid_ix(y - R, cc.min_y, cc.step_y), iy1 = grid_ix(y + R, cc.min_y, cc.step_y);
    double d = nearest;
    const Pt src{x, y};
    for (int iy = iy0; iy <= iy1; ++iy)
        for (int ix = ix0; ix <= ix1; ++ix)
            for (const auto& ref : cc.branch_grid[iy * CausticCache::kGrid + ix]) {
                const auto& br = cc.branches[ref.branch];
                const int n = static_cast<int>(br.size());
                if (n < 2) continue;
                const int prev = ref.pos > 0 ? ref.pos - 1 : n - 1;
                const int next = (ref.pos + 1) % n;
                d = dmin(d, seg_dist(src, br[prev], br[ref.pos]));
                d = dmin(d, seg_dist(src, br[ref.pos], br[next]));
            }
    return d;
}

namespace {

// ----- seeding (FSM:1424-1871, 4845-4926) -----

// selected_point_images (FSM:1873-1889): candidates with residual^2 < 1e-12.
int selected_images(double s, double q, Pt src, Pt* out)
{
    double c[25];
    const int n = binary_image_candidates(s, q, src.x, src.y, c);
    int k = 0;
    for (int i = 0; i < n; ++i) {
        if (c[5 * i + 3] * c[5 * i + 3] < 1.0e-12) out[k++] = {c[5 * i], c[5 * i + 1]};
    }
    return k;
}

struct SeedCtx {
    double s, q, rho, rho2;
    Pt src;
    Mapper m;
    std::vector<Pt>* seeds;
};

// append_valid_probe_image_seeds (FSM:1449-1498).
void probe_seeds(SeedCtx& c, Pt probe)
{
    if (c.rho <= 0.0 || dist2(probe, c.src) >= c.rho2 * (1.0 + 1.0e-10)) return;
    Pt imgs[5];
    const int n = selected_images(c.s, c.q, probe, imgs);
    if (n <= 3) return;
    auto& seeds = *c.seeds;
    const size_t before = seeds.size();
    for (int k = 0; k < n; ++k) {
        const Pt img = imgs[k];
        const double md2 = dist2(map_real(c.m, img.x, img.y), c.src);
        if (md2 > c.rho2 * (1.0 + 1.0e-8)) continue;
        bool dup = false;
        for (size_t si = 0; si < before; ++si) {
            if (dist2(img, seeds[si]) < 0.0625 * c.rho2) {
                const double ed2 = dist2(map_real(c.m, seeds[si].x, seeds[si].y), c.src);
                if (md2 + 1.0e-16 < ed2) seeds[si] = img;
                dup = true;
                break;
            }
        }
        if (!dup) seeds.push_back(img);
    }
}

// append_caustic_probe_image_seeds (FSM:1500-1563).
void caustic_probe_seeds(SeedCtx& c, Pt cs)
{
    const double dx = cs.x - c.src.x;
    const double dy = cs.y - c.src.y;
    const double dist = hyp(dx, dy);
    if (dist <= 0.0 || dist >= c.rho) return;
    const double ux = dx / dist;
    const double uy = dy / dist;
    const double steps[4] = {0.02 * c.rho, 0.05 * c.rho, 0.15 * c.rho, 0.35 * c.rho};
    for (double st : steps) {
        probe_seeds(c, {cs.x + ux * st, cs.y + uy * st});
        probe_seeds(c, {cs.x - ux * st, cs.y - uy * st});
    }
    if (c.seeds->size() <= 3) {
        const double radial[5] = {0.02 * c.rho, 0.05 * c.rho, 0.10 * c.rho, 0.20 * c.rho, 0.35 * c.rho};
        for (double st : radial) {
            for (int i = 0; i < 16; ++i) {
                const double th = 2.0 * kPi * static_cast<double>(i) / static_cast<double>(16);
                probe_seeds(c, {cs.x + st * std::cos(th), cs.y + st * std::sin(th)});
                if (c.seeds->size() > 3) return;
            }
        }
    }
}

double nearest_critical_d2(SeedCtx& c, double phi, Pt* nearest)
{
    double best = kInf;
    Pt cs[4];
    critical_sources(c.s, c.q, phi, cs);
    for (int i = 0; i < 4; ++i) {
        const double d2 = dist2(cs[i], c.src);
        if (d2 < best) {
            best = d2;
            if (nearest) *nearest = cs[i];
        }
    }
    return best;
}

// refine_nearest_critical_source (FSM:1666-1707): 32 golden-section steps.
Pt refine_critical(SeedCtx& c, double center, double step)
{
    double left = center - step;
    double right = center + step;
    const double g = 0.61803398874989484820;
    double x1 = right - g * (right - left);
    double x2 = left + g * (right - left);
    Pt n1{}, n2{};
    double f1 = nearest_critical_d2(c, x1, &n1);
    double f2 = nearest_critical_d2(c, x2, &n2);
    for (int it = 0; it < 32; ++it) {
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            n1 = n2;
            x2 = left + g * (right - left);
            f2 = nearest_critical_d2(c, x2, &n2);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            n2 = n1;
            x1 = right - g * (right - left);
            f1 = nearest_critical_d2(c, x1, &n1);
        }
    }
    return f1 < f2 ? n1 : n2;
}

// augmented_image_seeds (FSM:1709-1871) without seed hints.
std::vector<Pt> augmented_seeds(double s, double q, Pt src, double rho)
{
    std::vector<Pt> seeds;
    {
        double c[25];
        const int n = binary_image_candidates(s, q, src.x, src.y, c);
        for (int i = 0; i < n; ++i)
            if (c[5 * i + 4] != 0.0) seeds.push_back({c[5 * i], c[5 * i + 1]});
    }
    if (rho <= 0.0) return seeds;
    SeedCtx c{s, q, rho, rho * rho, src, make_mapper(s, q), &seeds};
    const int samples = 1400;
    const double phase_step = 2.0 * kPi / static_cast<double>(samples);
    double best_d2 = kInf;
    double best_phase = 0.0;
    const int nskip = 40;
    bool found = false;
    for (int kphi = 0; kphi < nskip && !found; ++kphi) {
        for (int jphi = 0; jphi < samples / nskip && !found; ++jphi) {
            const int sample = jphi * nskip + kphi;
            const double phi = phase_step * static_cast<double>(sample);
            Pt cs[4];
            critical_sources(s, q, phi, cs);
            for (int i = 0; i < 4; ++i) {
                const double d2 = dist2(cs[i], src);
                if (d2 < best_d2) {
                    best_d2 = d2;
                    best_phase = phi;
                }
                if (d2 >= c.rho2 || d2 <= 0.0) continue;
                const size_t before = seeds.size();
                caustic_probe_seeds(c, cs[i]);
                found = seeds.size() > before;
            }
        }
    }
    if (!found && best_d2 < c.rho2 && best_d2 > 0.0) {
        caustic_probe_seeds(c, refine_critical(c, best_phase, phase_step));
    }
    if (seeds.size() >= 5) {
        // Sequential branch scan (FSM:1800-1865), kept literally.
        Pt prev[4];
        bool inside[4] = {false, false, false, false};
        for (auto& p : prev) p = {1.0e30, 1.0e30};
        for (int sample = 0; sample < samples; ++sample) {
            const double phi = phase_step * static_cast<double>(sample);
            Pt cs[4];
            const int ncur = critical_sources(s, q, phi, cs);
            int assign[4] = {-1, -1, -1, -1};
            bool used[4] = {false, false, false, false};
            for (int bi = 0; bi < 4; ++bi) {
                double bd = 1.0e60;
                int bj = -1;
                for (int j = 0; j < ncur; ++j) {
                    if (used[j]) continue;
                    const double d2 = dist2(cs[j], prev[bi]);
                    if (d2 < bd) {
                        bd = d2;
                        bj = j;
                    }
                }
                if (bj >= 0) {
                    assign[bi] = bj;
                    used[bj] = true;
                }
            }
            for (int bi = 0; bi < 4; ++bi) {
                const int j = assign[bi];
                if (j < 0) {
                    inside[bi] = false;
                    continue;
                }
                const double d2 = dist2(cs[j], src);
                const bool now = d2 < c.rho2 && d2 > 0.0;
                const bool arc = rho >= 2.0e-2 && now && (sample % 20 == 0);
                if ((now && !inside[bi]) || arc) caustic_probe_seeds(c, cs[j]);
                inside[bi] = now;
                prev[bi] = cs[j];
            }
        }
    }
    // Boundary probes (FSM:1565-1591).
    if (seeds.size() < 128) {
        const double pr = rho * (1.0 - 0.02);
        for (int i = 0; i < 400 && seeds.size() < 128; ++i) {
            const double phi = 2.0 * kPi * static_cast<double>(i) / static_cast<double>(400);
            probe_seeds(c, {src.x + pr * std::cos(phi), src.y + pr * std::sin(phi)});
        }
    }
    // Interior probes (FSM:1593-1620).
    if (rho >= 2.0e-2) {
        const double radii[3] = {0.25, 0.5, 0.75};
        for (double f : radii) {
            const double pr = rho * f;
            for (int i = 0; i < 64; ++i) {
                const double phi = 2.0 * kPi * static_cast<double>(i) / static_cast<double>(64);
                probe_seeds(c, {src.x + pr * std::cos(phi), src.y + pr * std::sin(phi)});
            }
        }
    }
    return seeds;
}

// augment_seeds_from_caustic_branches (FSM:4845-4926).
void augment_from_branches(const CausticCache& cc, double s, double q, Pt src, double rho, std::vector<Pt>& seeds)
{
    if (seeds.size() >= 5 || cc.branch_grid.empty()) return;
    const double R = rho + cc.max_seg_len;
    const int ix0 = grid_ix(src.x - R, cc.min_x, cc.step_x), ix1 = grid_ix(src.x + R, cc.min_x, cc.step_x);
    const int iy0 = grid_ix(src.y - R, cc.min_y, cc.step_y), iy1 = grid_ix(src.y + R, cc.min_y, cc.step_y);
    for (int iy = iy0; iy <= iy1 && seeds.size() < 5; ++iy) {
        for (int ix = ix0; ix <= ix1 && seeds.size() < 5; ++ix) {
            for (const auto& ref : cc.branch_grid[iy * CausticCache::kGrid + ix]) {
                const auto& br = cc.branches[ref.branch];
                const int n = static_cast<int>(br.size());
                if (n < 2) continue;
                const int next = (ref.pos + 1) % n;
                if (next == 0) continue;
                const Pt p0 = br[ref.pos];
                const Pt p1 = br[next];
                if (seg_dist(src, p0, p1) >= rho) continue;
                const double sx = p1.x - p0.x;
                const double sy = p1.y - p0.y;
                const double l2 = sx * sx + sy * sy;
                const double t = l2 > 0.0 ? clampv(((src.x - p0.x) * sx + (src.y - p0.y) * sy) / l2, 0.0, 1.0) : 0.0;
                const Pt nearest{p0.x + t * sx, p0.y + t * sy};
                const double dist = std::sqrt(dist2(nearest, src));
                if (dist <= 0.0 || dist >= rho) continue;
                const double step = rho * 0.05 / dist;
                const Pt probe{nearest.x + (nearest.x - src.x) * step, nearest.y + (nearest.y - src.y) * step};
                if (dist2(probe, src) >= rho * rho) continue;
                Pt imgs[5];
                const int k = selected_images(s, q, probe, imgs);
                if (static_cast<size_t>(k) > seeds.size()) seeds.assign(imgs, imgs + k);
            }
        }
    }
}

// ----- Cartesian row scan (FSM:911-930, 1891-2014, 2470-2768) -----

int g_max_rows = 0;  // largest row count of one seed's scans in the last call (diagnostics)

struct Rows {
    std::vector<double> xmin, xmax, ax, y, dys;
    std::unordered_map<int, std::vector<int>> keys;
    void ensure(size_t i)
    {
        if (xmin.size() <= i) {
            if (static_cast<int>(i + 1) > g_max_rows) g_max_rows = static_cast<int>(i + 1);
            xmin.resize(i + 1);
            xmax.resize(i + 1);
            ax.resize(i + 1);
            y.resize(i + 1);
            dys.resize(i + 1);
        }
    }
};

struct CartCtx {
    Mapper m;
    Pt src;
    double rho;
    const FsSettings* st;
    const LdTable* ld;
};

// cartesian_image_area_impl (FSM:1891-2014): one directional flood fill.
double image_area(const CartCtx& c, Pt seed, double dy, int& yi, Rows& r, int jsign)
{
    double countx = 0.0, countall = 0.0, dz2 = 99999999.9;
    const double incr = std::fabs(dy);
    const double inv_incr = 1.0 / incr;
    double dx = incr;
    Pt img = seed;
    double x0 = seed.x;
    const double rho2 = c.rho * c.rho;
    const double inv_rho2 = 1.0 / rho2;
    const int max_steps = std::max(100000, c.st->source_bins * c.st->source_bins * 2000);
    int guard = 0;
    while (++guard < max_steps) {
        const double last = dz2;
        double md2;
        bool ok = true;
        if (jsign == 0) {
            md2 = mapped_dist2(c.m, img.x, img.y, c.src);
        } else {
            double jac;
            eval_cell(c.m, img.x, img.y, c.src, &md2, &jac);
            const int es = jac > 0.0 ? 1 : jac < 0.0 ? -1 : 0;
            ok = es != -jsign;
        }
        dz2 = ok ? md2 : rho2 + 1.0;
        r.ensure(yi);
        if (dz2 <= rho2) {
            if (dx == -incr && countx == 0.0) r.xmax[yi] = img.x - dx;
            countx += c.ld->uniform ? 1.0 : (*c.ld)(md2 * inv_rho2);
        } else if (dx == incr) {
            if (last <= rho2) r.xmax[yi] = img.x;
            dx = -incr;
            img.x = x0;
            r.xmin[yi] = img.x + dx;
        } else {
            if (last <= rho2) r.xmin[yi] = img.x;
            if (yi != 0 && countx == 0.0) {
                r.ensure(yi - 1);
                if (img.x >= r.xmin[yi - 1] - dx) {
                    img.x += dx;
                    continue;
                }
            }
            countall += countx;
            r.ax[yi] = countx;
            r.y[yi] = img.y;
            r.dys[yi] = dy;
            if (countx == 0.0) {
                r.dys[yi] = -dy;
                break;
            }
            const int key = static_cast<int>(img.y * inv_incr + kRowKeyOffset);
            auto& list = r.keys[key];
            for (int e : list) {
                if (r.xmin[yi] + incr < r.xmax[e] && r.xmax[yi] - incr > r.xmin[e]) return countall - countx;
            }
            list.push_back(yi);
            ++yi;
            r.ensure(yi);
            dx = incr;
            x0 = r.xmax[yi - 1];
            img.x = x0 - dx;
            img.y += dy;
            countx = 0.0;
        }
        img.x += dx;
    }
    return countall;
}

// high_magnification_floor_coefficient (FSM:1017-1063).
double floor_coefficient(const CartesianDiagnostics& d, double mag, double rho)
{
    const double am = std::fabs(mag);
    if (rho >= 0.1 && (d.gap_repairs > 0 || d.max_jump > 50.0)) return 0.06;
    if (rho < 1.0e-2 && d.seed_count <= 5 && am <= 10.0 && d.gap_repairs > 0 && d.max_jump > 20.0) return 0.035;
    if (rho < 1.0e-2 && d.seed_count <= 5 && am <= 10.0 && d.max_jump > 1000.0) return 0.04;
    if (rho < 1.0e-2 && d.seed_count >= 16 && d.overlaps >= 8 && d.gap_repairs >= 100 && d.max_jump > 1000.0 &&
        am <= 50.0)
        return 0.035;
    if (rho < 1.0e-2 && am <= 300.0) return 0.02;
    if (rho < 1.0e-2 && am <= 1000.0) return 0.04;
    if (rho < 1.0e-2 && d.seed_count <= 5 && d.gap_repairs > 0 && d.max_jump > 20.0) return 0.04;
    if (am <= 80.0 || d.gap_repairs <= 1000) return 0.0;
    return rho >= 1.0e-2 ? 0.04 : 0.05;
}

// cartesian_area_error_indicator (FSM:1065-1106).
double area_error(const CartesianDiagnostics& d, double rho, const FsSettings& st)
{
    const int bins = std::max(st.source_bins, 1);
    const double flux = source_flux(rho, st);
    if (!std::isfinite(flux) || flux <= 0.0 || rho <= 0.0) return 0.0;
    const double gw = rho >= 2.0e-2 ? 0.005 : ((rho < 1.0e-2 && d.seed_count >= 16) ? 0.015 : 0.03);
    const double ow = rho >= 2.0e-2 ? 0.005 : 0.02;
    const double bw = rho >= 2.0e-2 ? 0.012 : 0.03;
    double u = bw * static_cast<double>(d.boundary_rows) + gw * static_cast<double>(d.gap_repairs) +
               ow * static_cast<double>(d.overlaps) + 0.02 * static_cast<double>(std::max(0, d.fold)) +
               0.002 * static_cast<double>(std::max(0, d.seed_count - 5));
    if (rho >= 1.0e-3 && d.seed_count >= 16 && d.overlaps >= 8) {
        const double iw = rho < 1.0e-2 ? 0.001 : 0.0005;
        u += iw * static_cast<double>(d.seed_count) * static_cast<double>(d.overlaps);
    }
    if (rho >= 1.0e-3 && d.max_jump > 10.0) {
        const double jw = rho >= 2.0e-2 ? 0.2 : 4.0;
        u += jw * std::log10(d.max_jump / 10.0);
    }
    const double cell = (rho / static_cast<double>(bins)) * (rho / static_cast<double>(bins));
    const double e = 1.25 * u * cell / flux;
    return std::isfinite(e) ? e : 0.0;
}

double cartesian_impl(const FsSettings& st, const LdTable& ld, double s, double q, Pt src, double rho,
                      const std::vector<Pt>& images, CartesianDiagnostics* diag)
{
    if (images.empty() || rho <= 0.0) return kNaN;
    const Mapper m = make_mapper(s, q);
    CartCtx c{m, src, rho, &st, &ld};
    CartesianDiagnostics d;
    d.seed_count = static_cast<int>(images.size());
    const double nbin = static_cast<double>(std::max(st.source_bins, 1));
    const double incr = rho / nbin;
    const double margin = 0.5 * incr * 1.01;
    double area = 0.0;
    std::vector<double> areaimage(images.size(), 0.0);
    std::vector<int> overlap(images.size(), 0);
    std::vector<char> subtracted(images.size(), 0);
    for (size_t ii = 0; ii < images.size(); ++ii) {
        if (overlap[ii] == 1) continue;
        Rows r;
        r.ensure(1);
        double areai = 0.0, area0 = 0.0;
        double dy = incr;
        int yi = 0;
        const Pt seed = images[ii];
        const double jseed = jacobian(m, seed.x, seed.y);
        const int js = (std::fabs(jseed) < 0.02) ? (jseed > 0.0 ? 1 : jseed < 0.0 ? -1 : 0) : 0;
        ++d.processed;
        if (js != 0) ++d.fold;
        r.xmin[0] = seed.x;
        r.xmax[0] = seed.x;
        areai = image_area(c, seed, dy, yi, r, js);
        dy = -incr;
        r.ensure(yi);
        const Pt lower{r.xmax[0], seed.y + dy};
        r.xmin[yi] = r.xmin[0];
        r.xmax[yi] = r.xmax[0];
        r.y[yi] = r.y[0];
        r.dys[yi] = dy;
        ++yi;
        areai += image_area(c, lower, dy, yi, r, js);
        int nyi = yi;
        double areabound = 0.0;
        for (int row = 0; row < nyi; ++row) {
            r.ensure(row + 1);
            const double dxmax = r.xmax[row + 1] - r.xmax[row];
            const double dxmin = r.xmin[row + 1] - r.xmin[row];
            if (r.ax[row + 1] > 0.0) d.max_jump = dmax(d.max_jump, dmax(std::fabs(dxmax), std::fabs(dxmin)) / incr);
            if (r.ax[row + 1] > 0.0) {
                if (dxmax > 1.1 * incr) {
                    ++d.gap_repairs;
                    const Pt es{r.xmax[row + 1], r.y[row]};
                    r.ensure(yi);
                    r.xmin[yi] = r.xmax[row];
                    r.xmax[yi] = r.xmax[row + 1];
                    dy = -r.dys[row];
                    r.dys[yi] = dy;
                    ++yi;
                    area0 = image_area(c, es, dy, yi, r, js);
                    areai += area0;
                    areabound += area0;
                    if (area0 <= 0.0) --yi;
                }
                if (dxmin > 1.1 * incr) {
                    ++d.gap_repairs;
                    const Pt es{r.xmin[row + 1] - incr, r.y[row + 1]};
                    r.ensure(yi);
                    r.xmin[yi] = r.xmin[row];
                    r.xmax[yi] = r.xmin[row + 1];
                    dy = r.dys[row];
                    r.dys[yi] = dy;
                    ++yi;
                    area0 = image_area(c, es, dy, yi, r, js);
                    areai += area0;
                    areabound += area0;
                    if (area0 <= 0.0) --yi;
                }
                if (dxmin < -1.1 * incr) {
                    ++d.gap_repairs;
                    const Pt es{r.xmin[row] - incr, r.y[row]};
                    r.ensure(yi);
                    r.xmin[yi] = r.xmin[row + 1];
                    r.xmax[yi] = r.xmin[row];
                    dy = -r.dys[row];
                    r.dys[yi] = dy;
                    ++yi;
                    area0 = image_area(c, es, dy, yi, r, js);
                    areai += area0;
                    areabound += area0;
                    if (area0 <= 0.0) --yi;
                }
                if (dxmax < -1.1 * incr) {
                    ++d.gap_repairs;
                    const Pt es{r.xmax[row + 1] + incr, r.y[row + 1]};
                    r.ensure(yi);
                    r.xmin[yi] = r.xmax[row + 1];
                    r.xmax[yi] = r.xmax[row];
                    dy = r.dys[row];
                    r.dys[yi] = dy;
                    ++yi;
                    area0 = image_area(c, es, dy, yi, r, js);
                    areai += area0;
                    areabound += area0;
                    if (area0 <= 0.0) --yi;
                }
            }
            if (row == nyi - 1 && areabound > 0.0 && yi > nyi) nyi = yi;
        }
        area += areai;
        areaimage[ii] = areai;
        for (int row = 0; row < nyi; ++row)
            if (r.ax[row] > 0.0) ++d.boundary_rows;
        for (size_t o = 0; o < images.size(); ++o) {
            if (o == ii) continue;
            const Pt p = images[o];
            if (js != 0) {
                if (jacobian_sign(m, p.x, p.y) == -js) continue;
                if (rho >= 4.0e-3 && st.source_bins >= 35 && o > ii && std::fabs(jseed) < 1.0e-3 &&
                    std::fabs(jacobian(m, p.x, p.y)) < 0.02)
                    continue;
            }
            for (int row = 0; row < nyi; ++row) {
                if (r.ax[row] <= 0.0) continue;
                if (p.y >= r.y[row] - margin && p.y <= r.y[row] + margin && p.x >= r.xmin[row] - margin &&
                    p.x <= r.xmax[row] + margin) {
                    ++d.overlaps;
                    if (o < ii) {
                        if (!subtracted[o]) {
                            subtracted[o] = 1;
                            area -= areaimage[o];
                        }
                    } else {
                        overlap[o] = 1;
                    }
                    break;
                }
            }
        }
    }
    const double scale = source_flux(rho, st) / (rho * rho) * nbin * nbin;
    const double mag = area / scale;
    d.estimated_error = area_error(d, rho, st);
    const double fc = floor_coefficient(d, mag, rho);
    if (fc > 0.0) d.estimated_error = dmax(d.estimated_error, std::fabs(mag) * (fc / static_cast<double>(std::max(st.source_bins, 1))));
    if (diag) *diag = d;
    return mag;
}

// ----- polar flood fill (FSM:1123-1364) -----

// When set, polar_impl also sums its terms the way the device does: each
// term rounded to a multiple of 2^-64 and added into a 128-bit two's
// complement integer (order-free, so exact), converted back to FP64 once.
// The reference's own sum (`total`) is the running FP64 sum below; the two
// differ only by that sum's rounding, so equality of the fixed-point value
// with the device's pins the device's cell set and per-cell terms bit for bit.
struct Fx128 {
    unsigned long long lo = 0;
    long long hi = 0;
    void add(double v)
    {
        const double f = std::floor(v);
        const double frac = v - f;  // exact, in [0, 1)
        const auto l = static_cast<unsigned long long>(std::nearbyint(frac * 18446744073709551616.0));
        const unsigned long long sum = lo + l;
        hi += static_cast<long long>(f) + (sum < l ? 1 : 0);
        lo = sum;
    }
    double value() const
    {
        return static_cast<double>(hi) + static_cast<double>(lo) * (1.0 / 18446744073709551616.0);
    }
};

double wrap_angle(double a)
{
    while (a < 0.0) a += 2.0 * kPi;
    while (a >= 2.0 * kPi) a -= 2.0 * kPi;
    return a;
}

bool polar_start(const Mapper& m, Pt src, double rho, Pt seed, double dr, double dphi, int phi_bins, double* sr,
                 double* sp)
{
    const double seed_r = hyp(seed.x, seed.y);
    const double seed_phi = wrap_angle(std::atan2(seed.y, seed.x));
    const int seed_ir = static_cast<int>(std::floor(seed_r / dr));
    const int seed_iphi = clampv(static_cast<int>(seed_phi / dphi), 0, phi_bins - 1);
    const double rho2 = rho * rho;
    for (int shell = 0; shell <= 10; ++shell) {
        for (int dir = -1; dir <= 1; dir += 2) {
            for (int dir_ = -shell; dir_ <= shell; ++dir_) {
                const int diphi = (shell - std::abs(dir_)) * dir;
                const int ir = seed_ir + dir_;
                if (ir < 0) continue;
                int iphi = (seed_iphi + diphi) % phi_bins;
                if (iphi < 0) iphi += phi_bins;
                const double radius = (static_cast<double>(ir) + 0.5) * dr;
                const double phi = (static_cast<double>(iphi) + 0.5) * dphi;
                const Pt mp = map_real(m, radius * std::cos(phi), radius * std::sin(phi));
                if (dist2(mp, src) <= rho2) {
                    *sr = radius;
                    *sp = phi;
                    return true;
                }
            }
        }
    }
    return false;
}

double polar_impl(const FsSettings& st, const LdTable& ld, double s, double q, Pt src, double rho,
                  const std::vector<Pt>& images)
{
    if (images.empty()) return kNaN;
    const int bins = std::max(st.polar_source_bins > 0 ? st.polar_source_bins : st.source_bins, 1);
    const double ratio = dmax(st.polar_grid_ratio > 0.0 ? st.polar_grid_ratio : st.grid_ratio, 1.0e-12);
    const double dr = rho / static_cast<double>(bins);
    double max_r = 1.0;
    for (const Pt& p : images) max_r = dmax(max_r, hyp(p.x, p.y) + 4.0 * rho);
    const int phi_bins = std::max(16, static_cast<int>(std::ceil(2.0 * kPi * max_r / (dr * ratio))));
    const double dphi = 2.0 * kPi / static_cast<double>(phi_bins);
    const double flux = source_flux(rho, st);
    if (!std::isfinite(flux)) return kNaN;
    const Mapper m = make_mapper(s, q);
    std::vector<std::vector<std::pair<int, int>>> visited(phi_bins);
    std::deque<std::pair<int, int>> queue;
    const double rho2 = rho * rho;
    const double inv_rho2 = 1.0 / rho2;
    auto wrap = [&](int i) {
        i %= phi_bins;
        if (i < 0) i += phi_bins;
        return i;
    };
    auto is_visited = [&](int ir, int iphi) {
        if (ir < 0) return true;
        for (const auto& iv : visited[wrap(iphi)])
            if (ir >= iv.first && ir <= iv.second) return true;
        return false;
    };
    auto add_run = [&](int iphi, int l, int r) {
        iphi = wrap(iphi);
        if (r < l) return;
        auto& v = visited[iphi];
        v.push_back({l, r});
        std::sort(v.begin(), v.end());
        size_t w = 0;
        for (size_t k = 0; k < v.size(); ++k) {
            if (w == 0 || v[k].first > v[w - 1].second + 1) v[w++] = v[k];
            else v[w - 1].second = std::max(v[w - 1].second, v[k].second);
        }
        v.resize(w);
    };
    auto enqueue = [&](int ir, int iphi) {
        if (!is_visited(ir, iphi)) queue.push_back({ir, wrap(iphi)});
    };
    auto inside = [&](int ir, int iphi, double* dz2) {
        if (ir < 0) return false;
        iphi = wrap(iphi);
        const double radius = (static_cast<double>(ir) + 0.5) * dr;
        const double phi = (static_cast<double>(iphi) + 0.5) * dphi;
        const Pt mp = map_real(m, radius * std::cos(phi), radius * std::sin(phi));
        const double d2 = dist2(mp, src);
        if (dz2) *dz2 = d2;
        return d2 <= rho2;
    };
    for (const Pt& p : images) {
        double gr = 0.0, gp = 0.0;
        if (!polar_start(m, src, rho, p, dr, dphi, phi_bins, &gr, &gp)) continue;
        const int ir = std::max(0, static_cast<int>(std::floor(gr / dr)));
        const int iphi = clampv(static_cast<int>(gp / dphi), 0, phi_bins - 1);
        enqueue(ir, iphi);
    }
    double total = 0.0;
    Fx128 fixed;
    unsigned long long cells = 0;
    while (!queue.empty()) {
        const auto [ir, iphi] = queue.front();
        queue.pop_front();
        if (is_visited(ir, iphi) || !inside(ir, iphi, nullptr)) continue;
        int l = ir;
        while (l > 0 && !is_visited(l - 1, iphi) && inside(l - 1, iphi, nullptr)) --l;
        int r = ir;
        while (!is_visited(r + 1, iphi) && inside(r + 1, iphi, nullptr)) ++r;
        add_run(iphi, l, r);
        for (int cur = l; cur <= r; ++cur) {
            double dz2 = 0.0;
            inside(cur, iphi, &dz2);
            const double radius = (static_cast<double>(cur) + 0.5) * dr;
            const double b = ld.uniform ? 1.0 : ld(dz2 * inv_rho2);
            total += b * radius;
            if (g_polar_fixed) {
                fixed.add(b * radius);
                ++cells;
            }
            enqueue(cur, iphi - 1);
            enqueue(cur, iphi + 1);
        }
    }
    if (g_polar_fixed) {
        g_polar_fixed->value = fixed.value() * dr * dphi / flux;
        g_polar_fixed->cells = cells;
    }
    return total * dr * dphi / flux;
}

// hexadecapole_binary (FSM:792-847).
void hex_impl(const FsSettings& st, double s, double q, Pt src, double rho, const double* known, double* out)
{
    const double sineta[8] = {0.0, 1.0, 0.0, -1.0, kSqrtHalf, kSqrtHalf, -kSqrtHalf, -kSqrtHalf};
    const double coseta[8] = {1.0, 0.0, -1.0, 0.0, kSqrtHalf, -kSqrtHalf, -kSqrtHalf, kSqrtHalf};
    const double a0 = known ? *known : binary_mag0(s, q, src.x, src.y).magnification;
    double a1p = 0.0, a2p = 0.0, a1c = 0.0;
    for (int i = 0; i < 4; ++i) {
        a1p += binary_mag0(s, q, src.x + rho * coseta[i], src.y + rho * sineta[i]).magnification;
        a2p += binary_mag0(s, q, src.x + 0.5 * rho * coseta[i], src.y + 0.5 * rho * sineta[i]).magnification;
        a1c += binary_mag0(s, q, src.x + rho * coseta[i + 4], src.y + rho * sineta[i + 4]).magnification;
    }
    a1p = a1p / 4.0 - a0;
    a2p = a2p / 4.0 - a0;
    a1c = a1c / 4.0 - a0;
    const double a2rho2 = (16.0 * a2p - a1p) / 3.0;
    const double a4rho4 = (a1p + a1c) / 2.0 - a2rho2;
    const double g = ld_gamma(st);
    const double l = ld_lambda(st);
    const double quad = 0.5 * a2rho2 * (1.0 - 0.2 * g - l / 9.0);
    const double hexc = a4rho4 / 3.0 * (1.0 - 11.0 * g / 35.0 - 7.0 * l / 39.0);
    const double mag = a0 + quad + hexc;
    out[0] = mag;
    out[1] = std::fabs(hexc) / dmax(std::fabs(mag), 1.0e-10);
}

} // namespace

std::vector<Pt> seeds(const FsSettings& st, double s, double q, double x, double y, double rho)
{
    auto v = augmented_seeds(s, q, {x, y}, rho);
    CausticCache cc;
    build_caustic_cache(s, q, st.caustic_bins, &cc);
    augment_from_branches(cc, s, q, {x, y}, rho, v);
    return v;
}

int last_max_rows() { return g_max_rows; }

double cartesian(const FsSettings& st, double s, double q, double x, double y, double rho,
                 const std::vector<Pt>& sd, CartesianDiagnostics* diag)
{
    g_max_rows = 0;
    const LdTable ld(st);
    return cartesian_impl(st, ld, s, q, {x, y}, rho, sd, diag);
}

double polar(const FsSettings& st, double s, double q, double x, double y, double rho, const std::vector<Pt>& sd)
{
    const LdTable ld(st);
    return polar_impl(st, ld, s, q, {x, y}, rho, sd);
}

void hexadecapole(const FsSettings& st, double s, double q, double x, double y, double rho, const double* a0,
                  double* out)
{
    hex_impl(st, s, q, {x, y}, rho, a0, out);
}

// fixed_inverse_ray_binary (FSM:3042-3296) for fixed grids (no adaptive tape).
static FsResult fixed_inverse_ray(const FsSettings& st, const CausticCache& cc, double s, double q, Pt src,
                                  double rho, int method)
{
    auto sd = augmented_seeds(s, q, src, rho);
    augment_from_branches(cc, s, q, src, rho, sd);
    const LdTable ld(st);
    if (method == kPolar) {
        const double A = polar_impl(st, ld, s, q, src, rho, sd);
        if (!std::isfinite(A)) return {A, method, kNaN, 0, false};
        return {A, method, 0.0, 0, true};
    }
    CartesianDiagnostics d;
    const double A = cartesian_impl(st, ld, s, q, src, rho, sd, &d);
    if (!std::isfinite(A)) return {A, method, kNaN, 0, false};
    const double target = st.tol + st.reltol * dmax(std::fabs(A), 1.0);
    const bool conv = d.estimated_error <= 0.999 * target;
    return {A, method, d.estimated_error, 0, conv};
}

FsResult binary_mag(const FsSettings& st, double s, double q, double x, double y, double rho, double a_ps,
                    bool ps_exact)
{
    const Pt src{x, y};
    if (rho <= 0.0) return {binary_mag0(s, q, x, y).magnification, kPointSource, 0.0, 0, true};
    if (st.finite_mode <= 0) return {a_ps, kPointSource, 0.0, 0, true};
    CausticCache cc;
    build_caustic_cache(s, q, st.caustic_bins, &cc);
    const double margin = st.kinji_threshold * rho;
    const bool adaptive = st.adaptive_source_bins != 0 && (st.tol > 0.0 || st.reltol > 0.0);
    const double amargin = adaptive ? dmax(margin, 60.0 * rho) : margin;
    const double sampled = sampled_caustic_distance(cc, x, y, amargin);
    if (x < cc.min_x - amargin || x > cc.max_x + amargin || y < cc.min_y - amargin || y > cc.max_y + amargin)
        return {a_ps, kPointSource, 0.0, 0, true};
    const double refined = caustic_distance(cc, x, y, sampled);
    const bool near = refined < st.hex_threshold * rho;
    if (!near) {
        double safety = 1.0;
        if (rho >= 1.0e-3 && std::isfinite(refined) && rho > 0.0) {
            const double ratio = refined / rho;
            const double t = st.hex_threshold / dmax(ratio, st.hex_threshold);
            safety = dmax(1.0, 30.0 * t * t * t);
        }
        double req = st.adaptive_hex_threshold > 0.0 ? st.adaptive_hex_threshold : 1.0e-3;
        if (adaptive) req = st.reltol + st.tol / dmax(std::fabs(a_ps), 1.0);
        if (st.hex_threshold > 0.0) {
            double ind = 0.0;
            const PointSource dp = binary_mag0_derivatives(s, q, x, y, &ind);
            const double rel = ind * rho * rho / dmax(std::fabs(dp.magnification), 1.0e-10);
            if (std::isfinite(rel) && rel <= req / safety)
                return {dp.magnification, kPointSource, rel * dmax(std::fabs(dp.magnification), 1.0), 0, true};
        }
        double hx[2];
        hex_impl(st, s, q, src, rho, ps_exact ? &a_ps : nullptr, hx);
        double thr = st.adaptive_hex_threshold;
        if (adaptive) {
            req = st.reltol + st.tol / dmax(std::fabs(hx[0]), 1.0);
            thr = std::min(thr, req / safety);
        }
        if (hx[1] <= thr) return {hx[0], kHexadecapole, hx[1] * dmax(std::fabs(hx[0]), 1.0), 0, true};
    }
    const bool auto_polar = st.finite_mode == 4 && std::fabs(a_ps) >= 100.0;
    if (st.finite_mode == 2 || auto_polar) {
        FsSettings ir = st;
        if (auto_polar) ir.polar_grid_ratio = dmax(dmax(ir.polar_grid_ratio > 0.0 ? ir.polar_grid_ratio : ir.grid_ratio, 1.0e-12), 12.0);
        return fixed_inverse_ray(ir, cc, s, q, src, rho, kPolar);
    }
    return fixed_inverse_ray(st, cc, s, q, src, rho, kCartesian);
}

} // namespace oracle
