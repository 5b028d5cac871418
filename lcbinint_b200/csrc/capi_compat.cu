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

#include <cmath>
#include <limits>
#include <vector>

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
    Orbit o;
    o.separation = std::sqrt(x0 * x0 + x1 * x1);
    o.angle = angle + std::atan2(x1, x0);
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
    const lcbi_params p = *params;
    if (!params_valid(p)) return LCBI_INVALID_ARGUMENT;
    // from_c_options (lens_parameters.cpp:59-85): no options means the defaults.
    const lcbi_options o = options ? *options : lcbi_default_options();
    const bool vbm = o.vbm_compatible != 0;
    const size_t n = static_cast<size_t>(count);

    const bool has_xallarap = o.xallarap_param_type != LCBI_XALLARAP_NONE &&
                              (o.xallarap_param_type == LCBI_XALLARAP_ANGULAR_VELOCITY
                                   ? (p.xi_1 != 0.0 || p.xi_2 != 0.0)
                                   : (p.piEN_xa != 0.0 || p.piEE_xa != 0.0));
    if (p.piEN != 0.0 || p.piEE != 0.0 || has_xallarap || p.q2 > 0.0) {
        // Parallax, xallarap and triple lenses are not built here: report the
        // first epoch as unsupported.
        const double nan = std::numeric_limits<double>::quiet_NaN();
        set_unevaluated(results[0], nan, nan);
        return LCBI_UNSUPPORTED;
    }

    // Static trajectory (lens_model.cpp:90-99), the orbit at each epoch
    // (:113-115) and the source in the orbit's frame (:172-190).  The first
    // epoch whose orbit is not finite ends the array, as in the reference.
    const double cos_t = std::cos(p.theta);
    const double sin_t = std::sin(p.theta);
    const bool static_orbit = p.orbital_motion_mode == LCBI_ORBIT_STATIC;
    std::vector<double> sx(n), sy(n), mx(n), s_arr(n), q_arr(n);
    const double beta = p.umin;
    const double eff_q = (vbm && p.q != 0.0) ? 1.0 / p.q : p.q;
    size_t n_valid = n;
    double bad_x = 0.0, bad_y = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double tn = (times[i] - p.t0) / p.tE;
        double x, y;
        if (vbm) {
            x = tn * cos_t - beta * sin_t;
            y = tn * sin_t + beta * cos_t;
        } else {
            x = beta * sin_t + tn * cos_t;
            y = beta * cos_t - tn * sin_t;
        }
        const Orbit orb = static_orbit ? Orbit{p.sep, p.theta} : orbit_at(p, times[i]);
        if (!std::isfinite(orb.separation) || !std::isfinite(orb.angle)) {
            n_valid = i;
            bad_x = x;
            bad_y = y;
            break;
        }
        if (!static_orbit) {
            if (vbm) {
                const double nx = tn * std::cos(orb.angle) - beta * std::sin(orb.angle);
                const double ny = beta * std::cos(orb.angle) + tn * std::sin(orb.angle);
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
        mx[i] = vbm ? x : x - wide_binary_offset(orb.separation, p, o);
        s_arr[i] = orb.separation;
        q_arr[i] = eff_q;
    }
    if (n_valid == 0) {
        set_unevaluated(results[0], bad_x, bad_y);
        return LCBI_NUMERICAL_ERROR;
    }
    if (unsupported_dynamic(p, o)) {
        set_unevaluated(results[0], sx[0], sy[0]);
        return LCBI_UNSUPPORTED;
    }
    const int count_valid = static_cast<int>(n_valid);
    lcbi_gpu_context* ctx = thread_context();
    if (!ctx) return static_cast<lcbi_status>(LCBI_GPU_ERROR);
    std::vector<double> A(n), A_ps(n), err(n, 0.0);
    std::vector<int32_t> nimg(n), st(n, LCBI_OK), conv(n, 1);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (p.rho == 0.0) {
        // supports_binary_point_source (lens_model.cpp:43-46): binary_mag0.
        const int rc = lcbi_gpu_binary_mag0(ctx, count_valid, s_arr.data(), q_arr.data(), mx.data(), sy.data(), A.data(),
                                            nimg.data(), nullptr, 0);
        if (rc != LCBI_OK) return static_cast<lcbi_status>(rc);
        A_ps = A;
    } else {
        // binary_images seeds and point-source value, then the finite-source
        // decision tree (lens_model.cpp:209-226).
        int rc = lcbi_gpu_binary_images_mag(ctx, count_valid, s_arr.data(), q_arr.data(), mx.data(), sy.data(),
                                            A_ps.data(), nimg.data(), 0);
        if (rc != LCBI_OK) return static_cast<lcbi_status>(rc);
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
        fs.limb_darkening_c = p.limb_darkening_c;
        fs.limb_darkening_d = p.limb_darkening_d;
        fs.adaptive_source_bins = o.adaptive_source_bins;
        fs.max_source_bins = o.max_source_bins;
        fs.finite_source_tol = o.finite_source_tol;
        fs.finite_source_reltol = o.finite_source_reltol;
        std::vector<lcbi_fs_point> pts(n);
        std::vector<lcbi_fs_result> res(n);
        const double rho = std::abs(p.rho);
        for (size_t i = 0; i < n; ++i) {
            lcbi_fs_point& pt = pts[i];
            pt.s = s_arr[i];
            pt.q = eff_q;
            pt.y1 = mx[i];
            pt.y2 = sy[i];
            pt.rho = rho;
            pt.point_source_magnification = A_ps[i];
            pt.settings = 0;
            pt.model = 0;
            pt.flags = LCBI_FS_PS_EXACT | LCBI_FS_SEED_HINTS;
            pt.reserved = 0;
        }
        rc = lcbi_gpu_binary_mag(ctx, &fs, 1, nullptr, 0, count_valid, pts.data(), res.data(), 0);
        if (rc != LCBI_OK) return static_cast<lcbi_status>(rc);
        for (size_t i = 0; i < n; ++i) {
            A[i] = res[i].magnification;
            err[i] = res[i].error_estimate;
            conv[i] = res[i].converged;
            // A device limit (status 17-19) leaves no magnification.
            if (res[i].status != LCBI_OK && res[i].status != LCBI_NUMERICAL_ERROR) A[i] = nan;
        }
    }
    for (size_t i = 0; i < n_valid; ++i) {
        lcbi_result& r = results[i];
        r.magnification = A[i];
        r.point_source_magnification = A_ps[i];
        r.finite_source_magnification = p.rho == 0.0 ? nan : A[i];
        r.source_x = sx[i];
        r.source_y = sy[i];
        r.image_count = nimg[i];
        r.finite_source_error_estimate = err[i];
        r.finite_source_refinement_level = 0;
        r.finite_source_converged = conv[i] ? 1 : 0;
        if (!std::isfinite(r.magnification)) return LCBI_NUMERICAL_ERROR;
    }
    if (n_valid < n) {
        set_unevaluated(results[n_valid], bad_x, bad_y);
        return LCBI_NUMERICAL_ERROR;
    }
    return LCBI_OK;
}

lcbi_status lcbi_magnification(double time, const lcbi_params* params, const lcbi_options* options,
                               lcbi_result* result)
{
    if (params == nullptr || result == nullptr) return LCBI_INVALID_ARGUMENT;
    return lcbi_magnification_array(&time, 1, params, options, result);
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
