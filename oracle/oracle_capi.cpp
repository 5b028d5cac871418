// C entry points of the CPU oracle library (oracle/_build/liblcbi_oracle.so).
// Test infrastructure only: loaded by tests/, __graft_entry__.smoke() and the
// CPU baseline arm of bench.py, never by the product.
#include "oracle_fs.h"
#include "oracle_ps.h"

#include <cmath>

extern "C" {

void orc_binary_mag0_many(int n, const double* s, const double* q, const double* x, const double* y,
                          double* A, int* nimg)
{
    for (int i = 0; i < n; ++i) {
        const auto r = oracle::binary_mag0(s[i], q[i], x[i], y[i]);
        A[i] = r.magnification;
        if (nimg) nimg[i] = r.image_count;
    }
}

void orc_binary_mag0_derivatives_many(int n, const double* s, const double* q, const double* x,
                                      const double* y, double* A, int* nimg, double* indicator)
{
    for (int i = 0; i < n; ++i) {
        const auto r = oracle::binary_mag0_derivatives(s[i], q[i], x[i], y[i], &indicator[i]);
        A[i] = r.magnification;
        nimg[i] = r.image_count;
    }
}

int orc_image_candidates(double s, double q, double x, double y, double* out)
{
    return oracle::binary_image_candidates(s, q, x, y, out);
}

void orc_roots(const double* coef, int degree, double* roots, int polish)
{
    oracle::cplx p[6], r[5];
    for (int i = 0; i <= degree; ++i) p[i] = {coef[2 * i], coef[2 * i + 1]};
    oracle::roots_gen(r, p, degree, polish != 0);
    for (int i = 0; i < degree; ++i) {
        roots[2 * i] = r[i].re;
        roots[2 * i + 1] = r[i].im;
    }
}

} // extern "C"

// ----- finite source -----
namespace {
struct CSettings {
    int source_bins;
    int caustic_bins;
    double grid_ratio;
    int polar_source_bins;
    double polar_grid_ratio;
    int finite_mode;
    double kinji_threshold;
    double hex_threshold;
    double adaptive_hex_threshold;
    double limb_darkening_c;
    double limb_darkening_d;
    int adaptive_source_bins;
    int max_source_bins;
    double finite_source_tol;
    double finite_source_reltol;
};

oracle::FsSettings conv(const CSettings* c)
{
    oracle::FsSettings s;
    s.source_bins = c->source_bins;
    s.caustic_bins = c->caustic_bins;
    s.grid_ratio = c->grid_ratio;
    s.polar_source_bins = c->polar_source_bins;
    s.polar_grid_ratio = c->polar_grid_ratio;
    s.finite_mode = c->finite_mode;
    s.kinji_threshold = c->kinji_threshold;
    s.hex_threshold = c->hex_threshold;
    s.adaptive_hex_threshold = c->adaptive_hex_threshold;
    s.ld_c = c->limb_darkening_c;
    s.ld_d = c->limb_darkening_d;
    s.adaptive_source_bins = c->adaptive_source_bins;
    s.max_source_bins = c->max_source_bins;
    s.tol = c->finite_source_tol;
    s.reltol = c->finite_source_reltol;
    return s;
}
} // namespace

extern "C" {

void orc_binary_mag(const CSettings* st, double s, double q, double x, double y, double rho, double a_ps,
                    int ps_exact, double* dout, int* iout)
{
    const auto r = oracle::binary_mag(conv(st), s, q, x, y, rho, a_ps, ps_exact != 0);
    dout[0] = r.magnification;
    dout[1] = r.error_estimate;
    iout[0] = r.method;
    iout[1] = r.refinement_level;
    iout[2] = r.converged ? 1 : 0;
    iout[3] = 0;
}

// lcbinint.binary_inverse_ray semantics (python/lcbinint_pybind.cpp:3826-3847), batched.
void orc_inverse_ray_many(const CSettings* cst, int n, const double* s, const double* q, const double* x,
                          const double* y, const double* rho, double* A, int* method)
{
    oracle::FsSettings st = conv(cst);
    st.kinji_threshold = 1e18;
    st.hex_threshold = 0.0;
    st.adaptive_hex_threshold = 0.0;
    for (int i = 0; i < n; ++i) {
        const double aps = oracle::binary_mag0(s[i], q[i], x[i], y[i]).magnification;
        const auto r = oracle::binary_mag(st, s[i], q[i], x[i], y[i], std::fabs(rho[i]), aps, true);
        A[i] = r.magnification;
        if (method) method[i] = r.method;
    }
}

// orc_inverse_ray_many, and for each polar point also its integral with the
// cells summed exactly as the device sums them (NaN for other methods) and
// the number of cells counted.
void orc_inverse_ray_many_fixed(const CSettings* cst, int n, const double* s, const double* q, const double* x,
                                const double* y, const double* rho, double* A, int* method, double* A_fixed,
                                unsigned long long* cells)
{
    oracle::PolarFixedSum fx;
    for (int i = 0; i < n; ++i) {
        fx.value = std::nan("");
        fx.cells = 0;
        oracle::g_polar_fixed = &fx;
        orc_inverse_ray_many(cst, 1, s + i, q + i, x + i, y + i, rho + i, A + i, method ? method + i : nullptr);
        oracle::g_polar_fixed = nullptr;
        A_fixed[i] = fx.value;
        cells[i] = fx.cells;
    }
}

int orc_seeds(const CSettings* st, double s, double q, double x, double y, double rho, double* out, int cap)
{
    const auto v = oracle::seeds(conv(st), s, q, x, y, rho);
    const int n = static_cast<int>(v.size());
    for (int i = 0; i < n && i < cap; ++i) {
        out[2 * i] = v[i].x;
        out[2 * i + 1] = v[i].y;
    }
    return n;
}

double orc_cartesian(const CSettings* st, double s, double q, double x, double y, double rho, const double* seeds,
                     int n, double* diag)
{
    std::vector<oracle::Pt> v(n);
    for (int i = 0; i < n; ++i) v[i] = {seeds[2 * i], seeds[2 * i + 1]};
    oracle::CartesianDiagnostics d;
    const double A = oracle::cartesian(conv(st), s, q, x, y, rho, v, &d);
    if (diag) {
        diag[0] = d.seed_count;
        diag[1] = d.processed;
        diag[2] = d.fold;
        diag[3] = d.boundary_rows;
        diag[4] = d.gap_repairs;
        diag[5] = d.overlaps;
        diag[6] = d.max_jump;
        diag[7] = d.estimated_error;
    }
    return A;
}

double orc_polar(const CSettings* st, double s, double q, double x, double y, double rho, const double* seeds, int n)
{
    std::vector<oracle::Pt> v(n);
    for (int i = 0; i < n; ++i) v[i] = {seeds[2 * i], seeds[2 * i + 1]};
    return oracle::polar(conv(st), s, q, x, y, rho, v);
}

void orc_hexadecapole(const CSettings* st, double s, double q, double x, double y, double rho, const double* a0,
                      double* out)
{
    oracle::hexadecapole(conv(st), s, q, x, y, rho, a0, out);
}

int orc_caustic_cache(double s, double q, int bins, double* branch_xy, int cap, double* bbox, double* max_seg)
{
    oracle::CausticCache cc;
    oracle::build_caustic_cache(s, q, bins, &cc);
    int per = 0;
    for (int b = 0; b < 4; ++b) {
        per = static_cast<int>(cc.branches[b].size());
        for (int j = 0; j < per && j < cap; ++j) {
            branch_xy[(b * cap + j) * 2] = cc.branches[b][j].x;
            branch_xy[(b * cap + j) * 2 + 1] = cc.branches[b][j].y;
        }
    }
    bbox[0] = cc.min_x;
    bbox[1] = cc.max_x;
    bbox[2] = cc.min_y;
    bbox[3] = cc.max_y;
    *max_seg = cc.max_seg_len;
    return per;
}

void orc_caustic_distances(double s, double q, int bins, double x, double y, double R, double* out)
{
    oracle::CausticCache cc;
    oracle::build_caustic_cache(s, q, bins, &cc);
    out[0] = oracle::sampled_caustic_distance(cc, x, y, R);
    out[1] = oracle::caustic_distance(cc, x, y, out[0]);
}

int orc_critical_sources(double s, double q, double phi, double* out)
{
    oracle::Pt p[4];
    const int n = oracle::critical_sources(s, q, phi, p);
    for (int i = 0; i < n; ++i) {
        out[2 * i] = p[i].x;
        out[2 * i + 1] = p[i].y;
    }
    return n;
}

double orc_ld_brightness(double c, double d, double r2) { return oracle::ld_brightness(c, d, r2); }

int orc_last_max_rows() { return oracle::last_max_rows(); }

// Static-binary light curve in VBM convention (python/lcbinint_pybind.cpp:1087-1174).
int orc_light_curve_static(const CSettings* cst, const double* times, int n, double t0, double tE, double u0,
                           double alpha, double s, double q, double rho, double* out, int* method)
{
    const oracle::FsSettings st = conv(cst);
    const double ca = std::cos(alpha);
    const double sa = std::sin(alpha);
    const double itE = 1.0 / tE;
    const double eq = q != 0.0 ? 1.0 / q : q;
    for (int i = 0; i < n; ++i) {
        const double tau = (times[i] - t0) * itE;
        const double x = tau * ca - u0 * sa;
        const double y = tau * sa + u0 * ca;
        const double aps = oracle::binary_mag0(s, eq, x, y).magnification;
        if (rho == 0.0) {
            out[i] = aps;
            if (method) method[i] = 0;
            continue;
        }
        const auto r = oracle::binary_mag(st, s, eq, x, y, std::fabs(rho), aps, true);
        out[i] = r.magnification;
        if (method) method[i] = r.method;
        if (!std::isfinite(r.magnification)) return 1;
    }
    return 0;
}

} // extern "C"
