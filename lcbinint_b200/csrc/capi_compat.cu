// The reference's own C ABI (include/lcbinint/lcbinint.h:15-136) on the GPU.
//
// lcbi_magnification_array evaluates LensModel::magnification
// (src/lcbinint/model/lens_model.cpp:83-236) for every epoch in one batch:
// the host forms the source positions with the same arithmetic and C library
// calls as the reference (so they are bit-identical), and the device computes
// the point-source or finite-source magnifications through the library's own
// entry points.  Contexts are kept per host thread, on the thread's current
// CUDA device.
#include "../../include/lcbinint_b200.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <limits>
#include <thread>
#include <vector>

#include "lcbi_internal.h"
#include "lcbi_trajectory.h"

namespace {

struct ThreadContext {
    lcbi_gpu_context* ctx = nullptr;
    int device = -1;
    ~ThreadContext()
    {
        if (ctx) lcbi_gpu_destroy(ctx);
    }
};

lcbi_gpu_context* thread_context()
{
    thread_local ThreadContext tc;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    if (tc.ctx && tc.device == dev) return tc.ctx;
    if (tc.ctx) {
        lcbi_gpu_destroy(tc.ctx);
        tc.ctx = nullptr;
    }
    if (lcbi_gpu_create(dev, &tc.ctx) != LCBI_OK) {
        tc.ctx = nullptr;
        return nullptr;
    }
    tc.device = dev;
    return tc.ctx;
}

// LensParameters::is_valid (src/lcbinint/model/lens_parameters.cpp:7-11).
bool params_valid(const lcbi_params& p)
{
    return std::isfinite(p.tE) && p.tE != 0.0 && std::isfinite(p.q) && std::isfinite(p.sep) &&
           p.orbital_motion_mode >= LCBI_ORBIT_STATIC && p.orbital_motion_mode <= LCBI_ORBIT_KEPLER;
}

// has_unsupported_dynamic_effects (lens_model.cpp:16-27).
bool unsupported_dynamic(const lcbi_params& p, const lcbi_options& o)
{
    const bool piEN_xa = (p.piEN_xa != 0.0 || p.piEE_xa != 0.0) && o.xallarap_param_type != LCBI_XALLARAP_ORBITAL_ELEMENTS;
    const bool xi = (p.xi_1 != 0.0 || p.xi_2 != 0.0) && o.xallarap_param_type != LCBI_XALLARAP_ANGULAR_VELOCITY;
    return piEN_xa || xi || p.omega != 0.0 || p.v_sep != 0.0;
}

// wide_binary_offset (lens_model.cpp:29-41).
double wide_binary_offset(double separation, const lcbi_params& p, const lcbi_options& o)
{
    const double projected = std::abs(separation);
    if (o.center_of_mass != 0 || projected <= 1.0) return 0.0;
    const double q = std::abs(p.q);
    const double m2 = q / (1.0 + q);
    return m2 * projected - m2 / projected;
}

// Lens orbital motion (src/lcbinint/model/orbital_motion.cpp): projected
// separation and angle of the binary axis at `time`, restated with the same
// arithmetic and C library calls so the values are bit-identical.
struct Orbit {
    double separation, angle;
    double line_of_sight = 0.0;
};

constexpr double kBranchEps = 1.0e-8;

double clamp1(double v) { return v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v); }
double sqrt0(double v) { return std::sqrt(v > 0.0 ? v : 0.0); }

// circular_orbital_motion_3d (orbital_motion.cpp:69-115).
Orbit circular_orbit(double time, double separation, double angle, double w1, double w2, double w3, double t_ref)
{
    const double w13_sq = w1 * w1 + w3 * w3;
    const double w13 = std::sqrt(w13_sq);
    const double w123 = std::sqrt(w13_sq + w2 * w2);
    double w_orb = w2, inc = 0.0, phi0 = 0.0;
    if (w13 > kBranchEps) {
        const double w3_eff = w3 > kBranchEps ? w3 : kBranchEps;
        w_orb = w3_eff * w123 / w13;
        inc = std::acos(clamp1(w2 * w3_eff / (w13 * w123)));
        phi0 = std::atan2(-w1 * w123, w3_eff * w13);
    }
    const double c_phi0 = std::cos(phi0), s_phi0 = std::sin(phi0);
    const double c_inc = std::cos(inc);
    const double den0 = std::sqrt(c_phi0 * c_phi0 + c_inc * c_inc * s_phi0 * s_phi0);
    const double s_true = separation / den0;
    const double c_a0 = std::cos(angle), s_a0 = std::sin(angle);
    const double c_om = (c_phi0 * c_a0 + c_inc * s_a0 * s_phi0) / den0;
    const double s_om = (c_phi0 * s_a0 - c_inc * c_a0 * s_phi0) / den0;
    const double phi = w_orb * (time - t_ref) + phi0;
    const double c_phi = std::cos(phi), s_phi = std::sin(phi);
    const double den = std::sqrt(c_phi * c_phi + c_inc * c_inc * s_phi * s_phi);
    Orbit o;
    o.separation = s_true * den;
    const double sin_angle = (c_phi * s_om + c_inc * s_phi * c_om) / den;
    const double cos_angle = (c_phi * c_om - c_inc * s_phi * s_om) / den;
    o.angle = std::atan2(sin_angle, cos_angle);
    o.line_of_sight = s_true * std::sin(inc) * s_phi;
    return o;
}

// kepler_orbital_motion_3d (orbital_motion.cpp:117-183), Newton's method on
// Kepler's equation (:46-60).
Orbit kepler_orbit(double time, double separation, double angle, double w1, double w2, double w3, double szs,
                   double ar, double t_ref)
{
    ar += kBranchEps;
    const double smix = 1.0 + szs * szs;
    const double sqsmix = std::sqrt(smix);
    const double w11 = w1 * w1, w22 = w2 * w2, w33 = w3 * w3;
    const double w12 = w11 + w22;
    const double wt2 = w12 + w33;
    const double arm1 = ar - 1.0;
    const double arm2 = 2.0 * ar - 1.0;
    const double mean_motion = std::sqrt(wt2 / arm2 / smix) / ar;
    double z[3] = {-szs * w2, szs * w1 - w3, w2};
    {
        const double nz = sqrt0(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
        const double nan = std::numeric_limits<double>::quiet_NaN();
        if (nz == 0.0 || !std::isfinite(nz)) {
            z[0] = z[1] = z[2] = nan;
        } else {
            const double f = 1.0 / nz;
            z[0] = z[0] * f;
            z[1] = z[1] * f;
            z[2] = z[2] * f;
        }
    }
    double x[3] = {-ar * w11 + arm1 * w22 - arm2 * szs * w1 * w3 + arm1 * w33, -arm2 * w2 * (w1 + szs * w3),
                   arm1 * szs * w12 - arm2 * w1 * w3 - ar * szs * w33};
    const double x_norm = sqrt0(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    {
        const double f = 1.0 / x_norm;
        x[0] = x[0] * f;
        x[1] = x[1] * f;
        x[2] = x[2] * f;
    }
    const double ecc = x_norm / (ar * sqsmix * wt2);
    const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    const double conu = (x[0] + x[2] * szs) / sqsmix;
    const double cos_e0 = clamp1((conu + ecc) / (1.0 + ecc * conu));
    const double sign = (y[0] + y[2] * szs) > 0.0 ? 1.0 : -1.0;
    const double e0 = std::acos(cos_e0) * sign;
    const double sin_e0 = sqrt0(1.0 - cos_e0 * cos_e0) * sign;
    const double t_peri = t_ref - (e0 - ecc * sin_e0) / mean_motion;
    const double semi_major = ar * separation * sqsmix;
    const double mean_anomaly = mean_motion * (time - t_peri);
    double E = mean_anomaly + ecc * std::sin(mean_anomaly);
    for (int i = 0; i < 10; ++i) {
        const double f = E - ecc * std::sin(E) - mean_anomaly;
        const double fp = 1.0 - ecc * std::cos(E);
        const double delta = f / fp;
        E -= delta;
        if (std::abs(delta) <= 1.0e-13) break;
    }
    const double cos_e = std::cos(E), sin_e = std::sin(E);
    const double r0 = semi_major * (cos_e - ecc);
    const double r1 = semi_major * sqrt0(1.0 - ecc * ecc) * sin_e;
    const double x0 = r0 * x[0] + r1 * y[0];
    const double x1 = r0 * x[1] + r1 * y[1];
    const double x2 = r0 * x[2] + r1 * y[2];
    Orbit o;
    o.separation = std::sqrt(x0 * x0 + x1 * x1);
    o.angle = angle + std::atan2(x1, x0);
    o.line_of_sight = x2;
    return o;
}

// orbital_state (orbital_motion.cpp:185-199).
Orbit orbit_at(const lcbi_params& p, double time)
{
    const double t_ref = p.tfix != 0.0 ? p.tfix : p.t0;
    switch (p.orbital_motion_mode) {
    case LCBI_ORBIT_CIRCULAR:
        return circular_orbit(time, p.sep, p.theta, p.g1, p.g2, p.g3, t_ref);
    case LCBI_ORBIT_KEPLER:
        return kepler_orbit(time, p.sep, p.theta, p.g1, p.g2, p.g3, p.lom_szs, p.lom_ar, t_ref);
    default:
        return Orbit{p.sep, p.theta};
    }
}

void set_unevaluated(lcbi_result& r, double sx, double sy)
{
    const double nan = std::numeric_limits<double>::quiet_NaN();
    r.magnification = nan;
    r.point_source_magnification = nan;
    r.finite_source_magnification = nan;
    r.source_x = sx;
    r.source_y = sy;
    r.image_count = 0;
    r.finite_source_error_estimate = 0.0;
    r.finite_source_refinement_level = 0;
    r.finite_source_converged = 1;
}

// What LensModel::magnification (lens_model.cpp:83-236) settles for one
// parameter set before the magnifier call.
struct SetInfo {
    int status = LCBI_OK;     // LCBI_OK: the first n_valid epochs go to the device
    long long n_valid = 0;
    double bad_x = 0.0, bad_y = 0.0;  // trajectory source of the first epoch without a finite orbit
    bool write_first = false;  // results[0] is written as unevaluated at (first_x, first_y)
    double first_x = 0.0, first_y = 0.0;
    int settings = 0;
};

lcbi_fs_settings fs_settings_of(const lcbi_options& o, double c, double d)
{
    lcbi_fs_settings fs{};
    fs.source_bins = o.source_bins;
    fs.caustic_bins = o.caustic_bins;
    fs.grid_ratio = o.grid_ratio;
    fs.polar_source_bins = o.polar_source_bins;
    fs.polar_grid_ratio = o.polar_grid_ratio;
    fs.finite_mode = o.mode;
    fs.kinji_threshold = o.point_source_threshold;
    fs.hex_threshold = o.hexadecapole_threshold;
    fs.adaptive_hex_threshold = o.adaptive_hex_threshold;
    fs.limb_darkening_c = c;
    fs.limb_darkening_d = d;
    fs.adaptive_source_bins = o.adaptive_source_bins;
    fs.max_source_bins = o.max_source_bins;
    fs.finite_source_tol = o.finite_source_tol;
    fs.finite_source_reltol = o.finite_source_reltol;
    return fs;
}

// A cheap placeholder for an epoch that is not evaluated (a point source at
// the centre of an equal-mass binary); its result is never read.
void placeholder(lcbi_fs_point& pt)
{
    pt.s = 1.0;
    pt.q = 1.0;
    pt.y1 = 0.0;
    pt.y2 = 0.0;
    pt.rho = 0.0;
    pt.point_source_magnification = 0.0;
    pt.settings = 0;
    pt.model = 0;
    pt.flags = 0;
    pt.reserved = 0;
}

// The static trajectory (lens_model.cpp:90-99), the orbit at each epoch
// (:104-118) and the source in the orbit's frame (:162-190) for one set;
// epochs that are not evaluated get placeholders.  The first epoch whose orbit
// is not finite ends the set, as in the reference.
void prepare_set(const lcbi_params& p, const lcbi_options& o, bool keyword_route, const double* times, long long n,
                 double* sx, double* sy, lcbi_fs_point* pts, SetInfo& info)
{
    for (long long i = 0; i < n; ++i) placeholder(pts[i]);
    if (n == 0) return;
    if (!params_valid(p)) {
        info.status = LCBI_INVALID_ARGUMENT;
        return;
    }
    const bool vbm = o.vbm_compatible != 0;
    const bool has_xallarap = o.xallarap_param_type != LCBI_XALLARAP_NONE &&
                              (o.xallarap_param_type == LCBI_XALLARAP_ANGULAR_VELOCITY
                                   ? (p.xi_1 != 0.0 || p.xi_2 != 0.0)
                                   : (p.piEN_xa != 0.0 || p.piEE_xa != 0.0));
    const bool parallax = p.piEN != 0.0 || p.piEE != 0.0;
    if (p.q2 > 0.0) {
        // Triple lenses are not built here: the first epoch is reported as
        // unsupported.
        const double nan = std::numeric_limits<double>::quiet_NaN();
        info.status = LCBI_UNSUPPORTED;
        info.write_first = true;
        info.first_x = nan;
        info.first_y = nan;
        return;
    }
    const double cos_t = std::cos(p.theta);
    const double sin_t = std::sin(p.theta);
    const bool static_orbit = p.orbital_motion_mode == LCBI_ORBIT_STATIC;
    const double beta = p.umin;
    const double eff_q = (vbm && p.q != 0.0) ? 1.0 / p.q : p.q;
    const double rho = std::abs(p.rho);
    long long n_valid = n;
    // Parallax or xallarap: Trajectory::source_position (trajectory.cpp:436-463).
    const bool dynamic_source = parallax || has_xallarap;
    const lcbi::Trajectory traj = dynamic_source ? lcbi::make_trajectory(p) : lcbi::Trajectory{};
    for (long long i = 0; i < n; ++i) {
        const double tn = (times[i] - p.t0) / p.tE;
        double x, y;
        if (dynamic_source) {
            lcbi::source_position(traj, times[i], vbm, o.xallarap_param_type, &x, &y);
        } else if (vbm) {
            x = tn * cos_t - beta * sin_t;
            y = tn * sin_t + beta * cos_t;
        } else {
            x = beta * sin_t + tn * cos_t;
            y = beta * cos_t - tn * sin_t;
        }
        const Orbit orb = static_orbit ? Orbit{p.sep, p.theta} : orbit_at(p, times[i]);
        if (!std::isfinite(orb.separation) || !std::isfinite(orb.angle) || !std::isfinite(x) ||
            !std::isfinite(y)) {
            // A non-finite orbit ends the array (lens_model.cpp:116-119); so
            // does a source outside the ephemeris, whose magnification is NaN.
            n_valid = i;
            info.bad_x = x;
            info.bad_y = y;
            break;
        }
        if (!static_orbit) {
            if (vbm) {
                // LensModel rotates (tau, beta) directly unless parallax moved
                // the source (lens_model.cpp:164-178); the keyword route always
                // takes them back out of the trajectory point.
                double tau = tn, b = beta;
                if (keyword_route || parallax) {
                    tau = x * cos_t + y * sin_t;
                    b = -x * sin_t + y * cos_t;
                }
                const double nx = tau * std::cos(orb.angle) - b * std::sin(orb.angle);
                const double ny = b * std::cos(orb.angle) + tau * std::sin(orb.angle);
                x = nx;
                y = ny;
            } else {
                // rotate_source_to_orbital_frame (orbital_motion.cpp:201-206).
                const double c = std::cos(orb.angle - p.theta);
                const double s = std::sin(orb.angle - p.theta);
                const double rx = x * c + y * s;
                const double ry = y * c - x * s;
                x = rx;
                y = ry;
            }
        }
        sx[i] = x;
        sy[i] = y;
        lcbi_fs_point& pt = pts[i];
        pt.s = orb.separation;
        pt.q = eff_q;
        pt.y1 = vbm ? x : x - wide_binary_offset(orb.separation, p, o);
        pt.y2 = y;
        pt.rho = rho;
        pt.settings = info.settings;
    }
    if (n_valid == 0) {
        info.status = LCBI_NUMERICAL_ERROR;
        info.write_first = true;
        info.first_x = info.bad_x;
        info.first_y = info.bad_y;
        return;
    }
    if (unsupported_dynamic(p, o)) {
        for (long long i = 0; i < n_valid; ++i) placeholder(pts[i]);
        info.status = LCBI_UNSUPPORTED;
        info.write_first = true;
        info.first_x = sx[0];
        info.first_y = sy[0];
        return;
    }
    for (long long i = n_valid; i < n; ++i) placeholder(pts[i]);
    info.n_valid = n_valid;
}

// Runs fn(m) for every set, on several host threads when the batch is large
// (each set writes only its own epochs).
template <typename F>
void parallel_sets(int n_sets, long long n_times, F fn)
{
    unsigned hw = std::thread::hardware_concurrency();
    int threads = static_cast<int>(hw == 0 ? 1 : (hw > 32 ? 32 : hw));
    if (threads > n_sets) threads = n_sets;
    if (n_times < (1 << 16) || threads <= 1) {
        for (int m = 0; m < n_sets; ++m) fn(m);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            for (int m = next.fetch_add(1); m < n_sets; m = next.fetch_add(1)) fn(m);
        });
    for (auto& th : pool) th.join();
}

} // namespace

extern "C" {

lcbi_params lcbi_default_params(void)
{
    lcbi_params p = {};
    p.tE = 1.0;
    p.q = 1.0;
    p.sep = 1.0;
    p.orbital_motion_mode = LCBI_ORBIT_STATIC;
    p.lom_ar = 1.0;
    return p;
}

lcbi_options lcbi_default_options(void)
{
    lcbi_options o = {};
    o.orbit_pair = 23;
    o.caustic_bins = 1400;
    o.source_bins = 50;
    o.mode = 4;
    o.grid_ratio = 4.0;
    o.polar_source_bins = 0;
    o.polar_grid_ratio = 0.0;
    o.point_source_threshold = 20.0;
    o.hexadecapole_threshold = 3.0;
    o.adaptive_hex_threshold = 0.001;
    o.adaptive_source_bins = 0;
    o.max_source_bins = 400;
    o.finite_source_reltol = 0.0;
    o.xallarap_param_type = LCBI_XALLARAP_NONE;
    return o;
}

lcbi_status lcbi_magnification_array(const double* times, int count, const lcbi_params* params,
                                     const lcbi_options* options, lcbi_result* results)
{
    if (count < 0) return LCBI_INVALID_ARGUMENT;
    if (count == 0) return LCBI_OK;
    if (times == nullptr || params == nullptr || results == nullptr) return LCBI_INVALID_ARGUMENT;
    lcbi_gpu_context* ctx = thread_context();
    if (!ctx) return static_cast<lcbi_status>(LCBI_GPU_ERROR);
    const int64_t first = 0;
    const int32_t n = count;
    int32_t status = LCBI_OK;
    const int rc = lcbi_gpu_magnification_arrays(ctx, 1, params, options, &first, &n, times, count, 0, results, &status);
    return static_cast<lcbi_status>(rc != LCBI_OK ? rc : status);
}

int lcbi_gpu_magnification_arrays(lcbi_gpu_context* ctx, int32_t n_sets, const lcbi_params* params,
                                  const lcbi_options* options, const int64_t* first, const int32_t* count,
                                  const double* times, int64_t n_times, unsigned flags, lcbi_result* results,
                                  int32_t* status)
{
    if (!ctx || n_sets < 0 || n_times < 0) return LCBI_INVALID_ARGUMENT;
    if (n_sets == 0) return LCBI_OK;
    if (!params || !first || !count || !status || (n_times > 0 && (!times || !results))) return LCBI_INVALID_ARGUMENT;
    for (int m = 0; m < n_sets; ++m)
        if (first[m] < 0 || count[m] < 0 || first[m] + count[m] > n_times) return LCBI_INVALID_ARGUMENT;
    // from_c_options (lens_parameters.cpp:59-85): no options means the defaults.
    const lcbi_options o = options ? *options : lcbi_default_options();
    const bool keyword_route = (flags & LCBI_ARRAYS_KEYWORD_ROUTE) != 0;

    // One settings entry per distinct limb darkening.
    std::vector<lcbi_fs_settings> sts;
    std::vector<SetInfo> info(static_cast<size_t>(n_sets));
    for (int m = 0; m < n_sets; ++m) {
        const double c = params[m].limb_darkening_c, d = params[m].limb_darkening_d;
        int idx = -1;
        for (size_t k = 0; k < sts.size() && idx < 0; ++k)
            if (sts[k].limb_darkening_c == c && sts[k].limb_darkening_d == d) idx = static_cast<int>(k);
        if (idx < 0) {
            idx = static_cast<int>(sts.size());
            sts.push_back(fs_settings_of(o, c, d));
        }
        info[m].settings = idx;
    }

    const size_t n = static_cast<size_t>(n_times);
    std::vector<double> sx(n), sy(n), a_ps(n);
    std::vector<int32_t> nimg(n), levels(n, 0);
    std::vector<lcbi_fs_point> pts(n);
    std::vector<lcbi_fs_result> res(n);
    parallel_sets(n_sets, n_times, [&](int m) {
        prepare_set(params[m], o, keyword_route, times + first[m], count[m], sx.data() + first[m],
                    sy.data() + first[m], pts.data() + first[m], info[m]);
    });
    if (n_times > 0) {
        const int rc = lcbi::binary_mag_images(ctx, sts.data(), static_cast<int>(sts.size()), pts.data(), n_times,
                                               res.data(), a_ps.data(), nimg.data(), levels.data());
        if (rc != LCBI_OK) return rc;
    }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int m = 0; m < n_sets; ++m) {
        const SetInfo& in = info[m];
        lcbi_result* r = results + first[m];
        status[m] = in.status;
        if (in.write_first) set_unevaluated(r[0], in.first_x, in.first_y);
        if (in.status != LCBI_OK) continue;
        const long long k0 = first[m];
        const double rho = params[m].rho;
        for (long long i = 0; i < in.n_valid; ++i) {
            const lcbi_fs_result& f = res[k0 + i];
            // A device limit (status 17-19) leaves no magnification.
            const double A = (f.status != LCBI_OK && f.status != LCBI_NUMERICAL_ERROR) ? nan : f.magnification;
            lcbi_result& ri = r[i];
            ri.magnification = A;
            ri.point_source_magnification = a_ps[k0 + i];
            ri.finite_source_magnification = rho == 0.0 ? nan : A;
            ri.source_x = sx[k0 + i];
            ri.source_y = sy[k0 + i];
            ri.image_count = nimg[k0 + i];
            ri.finite_source_error_estimate = f.error_estimate;
            ri.finite_source_refinement_level = rho == 0.0 ? 0 : levels[k0 + i];
            ri.finite_source_converged = f.converged ? 1 : 0;
            if (!std::isfinite(A)) {
                status[m] = LCBI_NUMERICAL_ERROR;
                break;
            }
        }
        if (status[m] == LCBI_OK && in.n_valid < count[m]) {
            set_unevaluated(r[in.n_valid], in.bad_x, in.bad_y);
            status[m] = LCBI_NUMERICAL_ERROR;
        }
    }
    return LCBI_OK;
}

int lcbi_source_trajectory(const lcbi_params* params, const lcbi_options* options, const double* times, int64_t n,
                           double* x, double* y)
{
    if (!params || n < 0 || (n > 0 && (!times || !x || !y))) return LCBI_INVALID_ARGUMENT;
    const lcbi_params& p = *params;
    const lcbi_options o = options ? *options : lcbi_default_options();
    const bool vbm = o.vbm_compatible != 0;
    // Only parallax moves the source off the straight line here; the
    // trajectory applies no xallarap on this route (trajectory.hpp:12-13).
    const bool parallax = p.piEN != 0.0 || p.piEE != 0.0;
    const lcbi::Trajectory traj = parallax ? lcbi::make_trajectory(p) : lcbi::Trajectory{};
    const double cos_t = std::cos(p.theta);
    const double sin_t = std::sin(p.theta);
    for (int64_t i = 0; i < n; ++i) {
        double sx, sy;
        if (!parallax) {
            const double tau = (times[i] - p.t0) / p.tE;
            const double beta = p.umin;
            if (vbm) {
                sx = tau * cos_t - beta * sin_t;
                sy = tau * sin_t + beta * cos_t;
            } else {
                sx = beta * sin_t + tau * cos_t;
                sy = beta * cos_t - tau * sin_t;
            }
        } else {
            lcbi::source_position(traj, times[i], vbm, LCBI_XALLARAP_NONE, &sx, &sy);
        }
        if (p.orbital_motion_mode != LCBI_ORBIT_STATIC) {
            const Orbit orb = orbit_at(p, times[i]);
            if (vbm) {
                // (tau, beta) are taken back out of the trajectory point and
                // turned by the orbit's angle.
                const double tau = sx * cos_t + sy * sin_t;
                const double beta = -sx * sin_t + sy * cos_t;
                const double nx = tau * std::cos(orb.angle) - beta * std::sin(orb.angle);
                const double ny = beta * std::cos(orb.angle) + tau * std::sin(orb.angle);
                sx = nx;
                sy = ny;
            } else {
                const double c = std::cos(orb.angle - p.theta);
                const double s = std::sin(orb.angle - p.theta);
                const double rx = sx * c + sy * s;
                const double ry = sy * c - sx * s;
                sx = rx;
                sy = ry;
            }
        }
        x[i] = sx;
        y[i] = sy;
    }
    return LCBI_OK;
}

lcbi_status lcbi_magnification(double time, const lcbi_params* params, const lcbi_options* options,
                               lcbi_result* result)
{
    if (params == nullptr || result == nullptr) return LCBI_INVALID_ARGUMENT;
    return lcbi_magnification_array(&time, 1, params, options, result);
}

int lcbi_circular_orbital_motion(double time, double separation, double angle, double g1, double g2, double g3,
                                 double reference_time, double* state)
{
    if (!state) return LCBI_INVALID_ARGUMENT;
    const Orbit o = circular_orbit(time, separation, angle, g1, g2, g3, reference_time);
    state[0] = o.separation;
    state[1] = o.angle;
    state[2] = o.line_of_sight;
    return LCBI_OK;
}

int lcbi_kepler_orbital_motion(double time, double separation, double angle, double g1, double g2, double g3,
                               double szs, double ar, double reference_time, double* state)
{
    if (!state) return LCBI_INVALID_ARGUMENT;
    const Orbit o = kepler_orbit(time, separation, angle, g1, g2, g3, szs, ar, reference_time);
    state[0] = o.separation;
    state[1] = o.angle;
    state[2] = o.line_of_sight;
    return LCBI_OK;
}

const char* lcbi_status_string(lcbi_status status)
{
    switch (static_cast<int>(status)) {
    case LCBI_OK:
        return "ok";
    case LCBI_INVALID_ARGUMENT:
        return "invalid argument";
    case LCBI_NUMERICAL_ERROR:
        return "numerical error";
    case LCBI_UNSUPPORTED:
        return "unsupported";
    case LCBI_GPU_ERROR:
        return "gpu error";
    default:
        return "unknown status";
    }
}

} // extern "C"
