/* C++ entry points of lcbinint's magnification core, served by the GPU
 * library through its C ABI (lcbinint_b200.h).
 *
 * The classes keep the names, member functions and argument meanings of the
 * reference's C++ core so that code written against it needs only this
 * header (and `namespace lcbinint = lcbinint_b200;` where it spells the
 * namespace):
 *   PointSourceMagnifier  <- src/lcbinint/magnification/point_source_magnifier.hpp:47-85
 *   FiniteSourceMagnifier <- src/lcbinint/magnification/finite_source_magnifier.hpp:62-90
 *   FiniteSourceSettings, FiniteSourceResult, FiniteSourceMethod
 *                         <- finite_source_magnifier.hpp:13-60
 *   SourcePosition        <- src/lcbinint/types.hpp:15
 * Each magnifier owns a GPU context (device, stream, workspaces); one object
 * per host thread, as with the reference's objects, which keep caches.
 * Results are those of the reference for the same inputs.  Batched forms
 * (binary_mag0_batch, binary_mag over many points) are where the GPU pays:
 * a single evaluation is one launch sequence and one synchronisation.
 * Failures of the GPU itself throw std::runtime_error; numerical failures
 * come back as NaN magnifications, as in the reference. */
#ifndef LCBININT_B200_HPP
#define LCBININT_B200_HPP

#include "lcbinint_b200.h"

#include <cmath>
#include <complex>
#include <cstddef>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace lcbinint_b200 {

struct SourcePosition {
    double x = 0.0;
    double y = 0.0;
};

namespace detail {

struct ContextDeleter {
    void operator()(lcbi_gpu_context* c) const { lcbi_gpu_destroy(c); }
};
using ContextPtr = std::shared_ptr<lcbi_gpu_context>;

inline ContextPtr make_context(int device)
{
    lcbi_gpu_context* c = nullptr;
    const int rc = lcbi_gpu_create(device, &c);
    if (rc != LCBI_OK || c == nullptr)
        throw std::runtime_error("lcbi_gpu_create failed (status " + std::to_string(rc) + ")");
    return ContextPtr(c, ContextDeleter{});
}

inline void check(const ContextPtr& c, int rc, const char* what)
{
    if (rc != LCBI_OK) {
        throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(rc) +
                                 "): " + lcbi_gpu_last_error(c.get()));
    }
}

}  // namespace detail

namespace magnification {

struct PointSourceResult {
    double magnification = 0.0;
    int image_count = 0;
};

struct PointSourceDerivativeResult {
    double magnification = 0.0;
    int image_count = 0;
    double derivative_error_indicator = 0.0;
};

struct BinaryImage {
    SourcePosition position;
    double jacobian_determinant = 0.0;
};

struct BinaryImageCandidate {
    SourcePosition position;
    double jacobian_determinant = 0.0;
    double residual = 0.0;
    bool physical = false;
};

/* Separation and mass ratio in the core convention (mass_ratio < 1: the
 * heavier lens at -separation; > 1 is inverted), source in the
 * centre-of-mass frame, as in the reference. */
class PointSourceMagnifier {
public:
    explicit PointSourceMagnifier(int device = 0) : ctx_(detail::make_context(device)) {}

    PointSourceResult binary_mag0(double separation, double mass_ratio, SourcePosition source) const
    {
        double A = 0.0;
        int32_t n = 0;
        detail::check(ctx_, lcbi_gpu_binary_mag0(ctx_.get(), 1, &separation, &mass_ratio, &source.x, &source.y,
                                                 &A, &n, nullptr, 0),
                      "lcbi_gpu_binary_mag0");
        return {A, n};
    }

    /* The reference warm-starts from the previous call's roots and re-solves
     * cold when they do not converge (point_source_magnifier.cpp:666-681); a
     * cold solve gives the same result. */
    PointSourceResult binary_mag0_cached(double separation, double mass_ratio, SourcePosition source) const
    {
        return binary_mag0(separation, mass_ratio, source);
    }

    PointSourceDerivativeResult binary_mag0_with_derivatives(double separation, double mass_ratio,
                                                             SourcePosition source) const
    {
        double A = 0.0, ind = 0.0;
        int32_t n = 0;
        detail::check(ctx_, lcbi_gpu_binary_mag0_derivatives(ctx_.get(), 1, &separation, &mass_ratio, &source.x,
                                                             &source.y, &A, &n, &ind, 0),
                      "lcbi_gpu_binary_mag0_derivatives");
        return {A, n, ind};
    }

    PointSourceDerivativeResult binary_mag0_with_derivatives_cached(double separation, double mass_ratio,
                                                                    SourcePosition source) const
    {
        return binary_mag0_with_derivatives(separation, mass_ratio, source);
    }

    /* count sources of one lens in one launch. */
    void binary_mag0_batch(double separation, double mass_ratio, const SourcePosition* sources,
                           double* magnifications, std::size_t count) const
    {
        if (count == 0) return;
        std::vector<double> s(count, separation), q(count, mass_ratio), x(count), y(count);
        for (std::size_t i = 0; i < count; ++i) {
            x[i] = sources[i].x;
            y[i] = sources[i].y;
        }
        detail::check(ctx_, lcbi_gpu_binary_mag0(ctx_.get(), static_cast<int64_t>(count), s.data(), q.data(),
                                                 x.data(), y.data(), magnifications, nullptr, nullptr, 0),
                      "lcbi_gpu_binary_mag0");
    }

    std::vector<BinaryImageCandidate> binary_image_candidates(double separation, double mass_ratio,
                                                              SourcePosition source) const
    {
        double rec[20];
        int32_t nphys = 0;
        detail::check(ctx_, lcbi_gpu_binary_image_candidates(ctx_.get(), 1, &separation, &mass_ratio, &source.x,
                                                             &source.y, rec, &nphys, 0),
                      "lcbi_gpu_binary_image_candidates");
        std::vector<BinaryImageCandidate> out;
        if (nphys == 0) return out;
        if (nphys < 0) {
            // The source on the lighter lens: the reference's solver does not
            // terminate there; this reports the case instead.
            throw std::domain_error("binary_image_candidates: source on the lighter lens");
        }
        for (int k = 0; k < 5; ++k) {
            BinaryImageCandidate c;
            c.position = {rec[4 * k], rec[4 * k + 1]};
            c.jacobian_determinant = rec[4 * k + 2];
            c.residual = rec[4 * k + 3];
            c.physical = k < nphys;
            out.push_back(c);
        }
        return out;
    }

    std::vector<BinaryImage> binary_images(double separation, double mass_ratio, SourcePosition source) const
    {
        std::vector<BinaryImage> images;
        for (const auto& c : binary_image_candidates(separation, mass_ratio, source))
            if (c.physical) images.push_back({c.position, c.jacobian_determinant});
        return images;
    }

    /* point_source_magnifier.cpp:780-792: the source of an image position, in
     * the frame of the lens-equation roots.  Host arithmetic with the
     * reference's complex types and operations (make_vbm_geometry, :140-150),
     * so the result is the reference's to the bit. */
    SourcePosition binary_lens_equation(double separation, double mass_ratio, SourcePosition image) const
    {
        using Complex = std::complex<double>;
        const double s = std::abs(separation);
        const double q_input = std::abs(mass_ratio);
        const double q = q_input < 1.0 ? q_input : 1.0 / q_input;
        const Complex a = q_input < 1.0 ? Complex(-s, 0.0) : Complex(s, 0.0);
        const Complex m1 = 1.0 / (1.0 + q);
        const Complex m2 = q * m1;
        const Complex z(image.x, image.y);
        const Complex zc = std::conj(z);
        const Complex shifted = z - m1 / (zc - a) - m2 / zc;
        const Complex src = shifted - a * m1;
        return {src.real(), src.imag()};
    }

    lcbi_gpu_context* context() const { return ctx_.get(); }

private:
    detail::ContextPtr ctx_;
};

enum class FiniteSourceMethod {
    point_source,
    hexadecapole,
    inverse_ray_cartesian,
    inverse_ray_polar,
    inverse_ray_spine,
    source_plane_quadrature,
};

/* The reference's defaults (finite_source_magnifier.hpp:22-38). */
struct FiniteSourceSettings {
    int source_bins = 50;
    int caustic_bins = 1400;
    double grid_ratio = 4.0;
    int polar_source_bins = 0;
    double polar_grid_ratio = 0.0;
    int finite_mode = 1;
    double kinji_threshold = 20.0;
    double hex_threshold = 3.0;
    double adaptive_hex_threshold = 0.001;
    double limb_darkening_c = 0.0;
    double limb_darkening_d = 0.0;
    int adaptive_source_bins = 0;
    int max_source_bins = 400;
    double finite_source_tol = 0.0;
    double finite_source_reltol = 0.0;
};

struct FiniteSourceDecision {
    FiniteSourceMethod method = FiniteSourceMethod::point_source;
    int estimated_evaluations = 0;
    std::string reason;
};

struct FiniteSourceResult {
    double magnification = 0.0;
    int image_count = 0;
    FiniteSourceDecision decision;
    double error_estimate = 0.0;
    int refinement_level = 0;
    bool converged = true;
};

/* One point of a batched binary_mag call. */
struct FiniteSourcePoint {
    double separation = 1.0;
    double mass_ratio = 1.0;
    SourcePosition source;
    double source_radius = 0.0;
    double point_source_magnification = 0.0;
    bool point_source_magnification_is_exact = false;
};

class FiniteSourceMagnifier {
public:
    explicit FiniteSourceMagnifier(FiniteSourceSettings settings, int device = 0)
        : settings_(settings), ctx_(detail::make_context(device))
    {
    }

    const FiniteSourceSettings& settings() const { return settings_; }

    /* FiniteSourceMagnifier::binary_mag (finite_source_magnifier.cpp:4633-4843).
     * center_image_seeds, when given, are taken to be the point-source images
     * of `source`, which is what the reference's own caller passes
     * (src/lcbinint/model/lens_model.cpp:209-226); the device derives them
     * again.  point_magnifier_hint is not needed. */
    FiniteSourceResult binary_mag(double separation, double mass_ratio, SourcePosition source, double source_radius,
                                  double point_source_magnification,
                                  const std::vector<SourcePosition>* center_image_seeds = nullptr,
                                  bool point_source_magnification_is_exact = false,
                                  const PointSourceMagnifier* point_magnifier_hint = nullptr) const
    {
        (void)point_magnifier_hint;
        FiniteSourcePoint p;
        p.separation = separation;
        p.mass_ratio = mass_ratio;
        p.source = source;
        p.source_radius = source_radius;
        p.point_source_magnification = point_source_magnification;
        p.point_source_magnification_is_exact = point_source_magnification_is_exact;
        std::vector<FiniteSourceResult> r = binary_mag(&p, 1, center_image_seeds != nullptr);
        return r[0];
    }

    /* count points in one batched launch sequence. */
    std::vector<FiniteSourceResult> binary_mag(const FiniteSourcePoint* points, std::size_t count,
                                               bool seed_with_point_images = false) const
    {
        std::vector<FiniteSourceResult> out(count);
        if (count == 0) return out;
        const lcbi_fs_settings st = c_settings();
        std::vector<lcbi_fs_point> pts(count);
        for (std::size_t i = 0; i < count; ++i) {
            lcbi_fs_point& q = pts[i];
            q.s = points[i].separation;
            q.q = points[i].mass_ratio;
            q.y1 = points[i].source.x;
            q.y2 = points[i].source.y;
            q.rho = points[i].source_radius;
            q.point_source_magnification = points[i].point_source_magnification;
            q.settings = 0;
            q.model = 0;
            q.flags = (points[i].point_source_magnification_is_exact ? LCBI_FS_PS_EXACT : 0) |
                      (seed_with_point_images ? LCBI_FS_SEED_HINTS : 0);
            q.reserved = 0;
        }
        std::vector<lcbi_fs_result> res(count);
        detail::check(ctx_, lcbi_gpu_binary_mag(ctx_.get(), &st, 1, nullptr, 0, static_cast<int64_t>(count),
                                                pts.data(), res.data(), 0),
                      "lcbi_gpu_binary_mag");
        std::vector<int32_t> levels(count, 0);
        detail::check(ctx_, lcbi_gpu_last_refinement_levels(ctx_.get(), static_cast<int64_t>(count), levels.data()),
                      "lcbi_gpu_last_refinement_levels");
        for (std::size_t i = 0; i < count; ++i) {
            const lcbi_fs_result& r = res[i];
            FiniteSourceResult& o = out[i];
            o.magnification = r.magnification;
            o.decision.method = static_cast<FiniteSourceMethod>(r.method);
            o.decision.reason = method_name(r.method);
            o.error_estimate = r.error_estimate;
            o.refinement_level = levels[i];
            o.converged = r.converged != 0;
            if (r.status != LCBI_OK && r.status != LCBI_NUMERICAL_ERROR)
                o.magnification = std::numeric_limits<double>::quiet_NaN();
        }
        return out;
    }

    lcbi_gpu_context* context() const { return ctx_.get(); }

private:
    static const char* method_name(int m)
    {
        switch (m) {
        case 0: return "point source";
        case 1: return "hexadecapole";
        case 2: return "cartesian inverse-ray";
        case 3: return "polar inverse-ray";
        default: return "";
        }
    }

    lcbi_fs_settings c_settings() const
    {
        lcbi_fs_settings s{};
        s.source_bins = settings_.source_bins;
        s.caustic_bins = settings_.caustic_bins;
        s.grid_ratio = settings_.grid_ratio;
        s.polar_source_bins = settings_.polar_source_bins;
        s.polar_grid_ratio = settings_.polar_grid_ratio;
        s.finite_mode = settings_.finite_mode;
        s.kinji_threshold = settings_.kinji_threshold;
        s.hex_threshold = settings_.hex_threshold;
        s.adaptive_hex_threshold = settings_.adaptive_hex_threshold;
        s.limb_darkening_c = settings_.limb_darkening_c;
        s.limb_darkening_d = settings_.limb_darkening_d;
        s.adaptive_source_bins = settings_.adaptive_source_bins;
        s.max_source_bins = settings_.max_source_bins;
        s.finite_source_tol = settings_.finite_source_tol;
        s.finite_source_reltol = settings_.finite_source_reltol;
        return s;
    }

    FiniteSourceSettings settings_;
    detail::ContextPtr ctx_;
};

}  // namespace magnification
}  // namespace lcbinint_b200

#endif /* LCBININT_B200_HPP */
