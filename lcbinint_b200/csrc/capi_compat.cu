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
    if (p.piEN != 0.0 || p.piEE != 0.0 || has_xallarap || p.q2 > 0.0 ||
        p.orbital_motion_mode != LCBI_ORBIT_STATIC) {
        // Parallax, xallarap, triple lenses and lens orbital motion are not
        // built here: report the first epoch as unsupported.
        const double nan = std::numeric_limits<double>::quiet_NaN();
        set_unevaluated(results[0], nan, nan);
        return LCBI_UNSUPPORTED;
    }

    // Static trajectory (lens_model.cpp:90-99) and the static orbit.
    const double cos_t = std::cos(p.theta);
    const double sin_t = std::sin(p.theta);
    std::vector<double> sx(n), sy(n), mx(n), s_arr(n), q_arr(n);
    const double beta = p.umin;
    for (size_t i = 0; i < n; ++i) {
        const double tn = (times[i] - p.t0) / p.tE;
        if (vbm) {
            sx[i] = tn * cos_t - beta * sin_t;
            sy[i] = tn * sin_t + beta * cos_t;
        } else {
            sx[i] = beta * sin_t + tn * cos_t;
            sy[i] = beta * cos_t - tn * sin_t;
        }
    }
    if (!std::isfinite(p.sep) || !std::isfinite(p.theta)) {
        set_unevaluated(results[0], sx[0], sy[0]);
        return LCBI_NUMERICAL_ERROR;
    }
    if (unsupported_dynamic(p, o)) {
        set_unevaluated(results[0], sx[0], sy[0]);
        return LCBI_UNSUPPORTED;
    }
    const double offset = vbm ? 0.0 : wide_binary_offset(p.sep, p, o);
    const double eff_q = (vbm && p.q != 0.0) ? 1.0 / p.q : p.q;
    for (size_t i = 0; i < n; ++i) {
        mx[i] = sx[i];
        if (!vbm) mx[i] -= offset;
        s_arr[i] = p.sep;
        q_arr[i] = eff_q;
    }

    lcbi_gpu_context* ctx = thread_context();
    if (!ctx) return static_cast<lcbi_status>(LCBI_GPU_ERROR);
    std::vector<double> A(n), A_ps(n), err(n, 0.0);
    std::vector<int32_t> nimg(n), st(n, LCBI_OK), conv(n, 1);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (p.rho == 0.0) {
        // supports_binary_point_source (lens_model.cpp:43-46): binary_mag0.
        const int rc = lcbi_gpu_binary_mag0(ctx, count, s_arr.data(), q_arr.data(), mx.data(), sy.data(), A.data(),
                                            nimg.data(), nullptr, 0);
        if (rc != LCBI_OK) return static_cast<lcbi_status>(rc);
        A_ps = A;
    } else {
        // binary_images seeds and point-source value, then the finite-source
        // decision tree (lens_model.cpp:209-226).
        int rc = lcbi_gpu_binary_images_mag(ctx, count, s_arr.data(), q_arr.data(), mx.data(), sy.data(),
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
            pt.s = p.sep;
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
        rc = lcbi_gpu_binary_mag(ctx, &fs, 1, nullptr, 0, count, pts.data(), res.data(), 0);
        if (rc != LCBI_OK) return static_cast<lcbi_status>(rc);
        for (size_t i = 0; i < n; ++i) {
            A[i] = res[i].magnification;
            err[i] = res[i].error_estimate;
            conv[i] = res[i].converged;
            // A device limit (status 17-19) leaves no magnification.
            if (res[i].status != LCBI_OK && res[i].status != LCBI_NUMERICAL_ERROR) A[i] = nan;
        }
    }
    for (size_t i = 0; i < n; ++i) {
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
