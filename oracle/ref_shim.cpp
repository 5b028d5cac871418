// Test-only C shim over the reference lcbinint sources (oracle/_ref).
//
// This translation unit is compiled together with the reference's own source
// files (see oracle/Makefile) and is linked ONLY into oracle/_ref, which the
// parity tests, smoke() and the bench reference arm use as the checker.  It
// exposes, through plain C entry points, the reference functions that the
// B200 implementation must reproduce, including the ones that live in the
// anonymous namespace of finite_source_magnifier.cpp (hence the #include of
// that .cpp file below: those functions are otherwise unreachable).
//
// Nothing here is product code; the product never links or loads it.

// Standard headers first, so the access override below only touches the
// reference's own class definitions.
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <limits>
#include <memory>
#include <numeric>
#include <queue>
#include <set>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#define private public
#include "lcbinint/magnification/finite_source_magnifier.hpp"
#undef private
#include "lcbinint/magnification/finite_source_magnifier.cpp"

#include "SkowronGould.h"

namespace mag = lcbinint::magnification;

extern "C" {

// Flat mirror of FiniteSourceSettings (finite_source_magnifier.hpp:22-38).
typedef struct ref_fs_settings {
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
} ref_fs_settings;

static mag::FiniteSourceSettings to_settings(const ref_fs_settings* s)
{
    mag::FiniteSourceSettings o;
    o.source_bins = s->source_bins;
    o.caustic_bins = s->caustic_bins;
    o.grid_ratio = s->grid_ratio;
    o.polar_source_bins = s->polar_source_bins;
    o.polar_grid_ratio = s->polar_grid_ratio;
    o.finite_mode = s->finite_mode;
    o.kinji_threshold = s->kinji_threshold;
    o.hex_threshold = s->hex_threshold;
    o.adaptive_hex_threshold = s->adaptive_hex_threshold;
    o.limb_darkening_c = s->limb_darkening_c;
    o.limb_darkening_d = s->limb_darkening_d;
    o.adaptive_source_bins = s->adaptive_source_bins;
    o.max_source_bins = s->max_source_bins;
    o.finite_source_tol = s->finite_source_tol;
    o.finite_source_reltol = s->finite_source_reltol;
    return o;
}

void ref_default_settings(ref_fs_settings* s)
{
    const mag::FiniteSourceSettings d;
    s->source_bins = d.source_bins;
    s->caustic_bins = d.caustic_bins;
    s->grid_ratio = d.grid_ratio;
    s->polar_source_bins = d.polar_source_bins;
    s->polar_grid_ratio = d.polar_grid_ratio;
    s->finite_mode = d.finite_mode;
    s->kinji_threshold = d.kinji_threshold;
    s->hex_threshold = d.hex_threshold;
    s->adaptive_hex_threshold = d.adaptive_hex_threshold;
    s->limb_darkening_c = d.limb_darkening_c;
    s->limb_darkening_d = d.limb_darkening_d;
    s->adaptive_source_bins = d.adaptive_source_bins;
    s->max_source_bins = d.max_source_bins;
    s->finite_source_tol = d.finite_source_tol;
    s->finite_source_reltol = d.finite_source_reltol;
}

// PointSourceMagnifier::binary_mag0 over arrays (point_source_magnifier.cpp:652-693).
void ref_binary_mag0_many(int n, const double* s, const double* q, const double* x,
                          const double* y, double* A, int* nimg)
{
    const mag::PointSourceMagnifier pm;
    for (int i = 0; i < n; ++i) {
        const auto r = pm.binary_mag0(s[i], q[i], {x[i], y[i]});
        A[i] = r.magnification;
        if (nimg) nimg[i] = r.image_count;
    }
}

// binary_mag0_with_derivatives (point_source_magnifier.cpp:583-611).
void ref_binary_mag0_derivatives_many(int n, const double* s, const double* q, const double* x,
                                      const double* y, double* A, int* nimg, double* indicator)
{
    const mag::PointSourceMagnifier pm;
    for (int i = 0; i < n; ++i) {
        const auto r = pm.binary_mag0_with_derivatives(s[i], q[i], {x[i], y[i]});
        A[i] = r.magnification;
        nimg[i] = r.image_count;
        indicator[i] = r.derivative_error_indicator;
    }
}

// binary_image_candidates (point_source_magnifier.cpp:739-778); out rows: x, y, detJ, residual, physical.
int ref_image_candidates(double s, double q, double x, double y, double* out)
{
    const mag::PointSourceMagnifier pm;
    const auto c = pm.binary_image_candidates(s, q, {x, y});
    for (std::size_t i = 0; i < c.size(); ++i) {
        out[5 * i + 0] = c[i].position.x;
        out[5 * i + 1] = c[i].position.y;
        out[5 * i + 2] = c[i].jacobian_determinant;
        out[5 * i + 3] = c[i].residual;
        out[5 * i + 4] = c[i].physical ? 1.0 : 0.0;
    }
    return static_cast<int>(c.size());
}

// cmplx_roots_gen (SkowronGould.cpp:79-168) on interleaved (re, im) coefficients.
void ref_roots(const double* coef, int degree, double* roots, int polish)
{
    std::vector<complex> p(static_cast<std::size_t>(degree) + 1);
    std::vector<complex> r(static_cast<std::size_t>(degree));
    for (int i = 0; i <= degree; ++i) p[i] = complex(coef[2 * i], coef[2 * i + 1]);
    cmplx_roots_gen(r.data(), p.data(), degree, polish != 0, false);
    for (int i = 0; i < degree; ++i) {
        roots[2 * i] = r[i].re;
        roots[2 * i + 1] = r[i].im;
    }
}

// FiniteSourceMagnifier::binary_mag (finite_source_magnifier.cpp:4633-4843) with a fresh
// magnifier.  dout = {A, error_estimate}; iout = {method, refinement_level, converged, image_count}.
void ref_binary_mag(const ref_fs_settings* st, double s, double q, double x, double y, double rho,
                    double a_ps, int ps_exact, double* dout, int* iout)
{
    const mag::FiniteSourceMagnifier fm(to_settings(st));
    const auto r = fm.binary_mag(s, q, {x, y}, rho, a_ps, nullptr, ps_exact != 0, nullptr);
    dout[0] = r.magnification;
    dout[1] = r.error_estimate;
    iout[0] = static_cast<int>(r.decision.method);
    iout[1] = r.refinement_level;
    iout[2] = r.converged ? 1 : 0;
    iout[3] = r.image_count;
}

// The lcbinint.binary_inverse_ray free function (python/lcbinint_pybind.cpp:3826-3847),
// batched: forced thresholds, PS magnification from binary_mag0 passed as exact.
void ref_inverse_ray_many(const ref_fs_settings* st, int n, const double* s, const double* q,
                          const double* x, const double* y, const double* rho, double* A,
                          int* method)
{
    mag::FiniteSourceSettings settings = to_settings(st);
    settings.kinji_threshold = 1e18;
    settings.hex_threshold = 0.0;
    settings.adaptive_hex_threshold = 0.0;
    for (int i = 0; i < n; ++i) {
        const mag::PointSourceMagnifier pm;
        const mag::FiniteSourceMagnifier fm(settings);
        const lcbinint::SourcePosition src {x[i], y[i]};
        const auto point = pm.binary_mag0(s[i], q[i], src);
        const auto r = fm.binary_mag(s[i], q[i], src, std::abs(rho[i]), point.magnification,
                                     nullptr, true);
        A[i] = r.magnification;
        if (method) method[i] = static_cast<int>(r.decision.method);
    }
}

// Seeds exactly as fixed_inverse_ray_binary builds them (finite_source_magnifier.cpp:3055-3064).
int ref_seeds(const ref_fs_settings* st, double s, double q, double x, double y, double rho,
              double* out, int cap)
{
    const mag::FiniteSourceMagnifier fm(to_settings(st));
    const mag::PointSourceMagnifier pm;
    const auto mapper = mag::make_binary_lens_mapper(s, q);
    auto seeds = mag::augmented_image_seeds(pm, mapper, s, q, {x, y}, rho);
    fm.augment_seeds_from_caustic_branches(s, q, {x, y}, rho, seeds);
    const int n = static_cast<int>(seeds.size());
    for (int i = 0; i < n && i < cap; ++i) {
        out[2 * i] = seeds[i].x;
        out[2 * i + 1] = seeds[i].y;
    }
    return n;
}

// Seeds before the caustic-branch augmentation (augmented_image_seeds only).
int ref_seeds_phase12(double s, double q, double x, double y, double rho, double* out, int cap)
{
    const mag::PointSourceMagnifier pm;
    const auto mapper = mag::make_binary_lens_mapper(s, q);
    const auto seeds = mag::augmented_image_seeds(pm, mapper, s, q, {x, y}, rho);
    const int n = static_cast<int>(seeds.size());
    for (int i = 0; i < n && i < cap; ++i) {
        out[2 * i] = seeds[i].x;
        out[2 * i + 1] = seeds[i].y;
    }
    return n;
}

// inverse_ray_cartesian_binary_mag with given seeds (finite_source_magnifier.cpp:2470-2768).
// diag = {seed_count, processed, fold, boundary_rows, gap_repairs, overlaps, max_jump, est_err}.
double ref_cartesian(const ref_fs_settings* st, double s, double q, double x, double y, double rho,
                     const double* seeds, int nseeds, double* diag)
{
    const mag::FiniteSourceMagnifier fm(to_settings(st));
    const mag::PointSourceMagnifier pm;
    std::vector<lcbinint::SourcePosition> sv(static_cast<std::size_t>(nseeds));
    for (int i = 0; i < nseeds; ++i) sv[i] = {seeds[2 * i], seeds[2 * i + 1]};
    mag::LegacyAreaDiagnostics d;
    const double A = mag::inverse_ray_cartesian_binary_mag(
        pm, s, q, {x, y}, rho, fm.settings(), &fm, &sv, &d, nullptr);
    if (diag) {
        diag[0] = d.seed_count;
        diag[1] = d.processed_images;
        diag[2] = d.fold_seed_count;
        diag[3] = d.boundary_rows;
        diag[4] = d.gap_repairs;
        diag[5] = d.overlaps;
        diag[6] = d.max_jump_cells;
        diag[7] = d.estimated_error;
    }
    return A;
}

// inverse_ray_polar_boundary_binary with given seeds (finite_source_magnifier.cpp:1156-1319).
double ref_polar(const ref_fs_settings* st, double s, double q, double x, double y, double rho,
                 const double* seeds, int nseeds)
{
    const mag::FiniteSourceMagnifier fm(to_settings(st));
    const mag::PointSourceMagnifier pm;
    std::vector<lcbinint::SourcePosition> sv(static_cast<std::size_t>(nseeds));
    for (int i = 0; i < nseeds; ++i) sv[i] = {seeds[2 * i], seeds[2 * i + 1]};
    return mag::inverse_ray_polar_boundary_binary(pm, s, q, {x, y}, rho, fm.settings(), &fm,
                                                  nullptr, &sv);
}

// hexadecapole_binary (finite_source_magnifier.cpp:792-847); out = {A, rel_err}.
void ref_hexadecapole(const ref_fs_settings* st, double s, double q, double x, double y, double rho,
                      const double* known_a0, double* out)
{
    const mag::PointSourceMagnifier pm;
    const auto r = mag::hexadecapole_binary(pm, s, q, {x, y}, rho, to_settings(st), known_a0);
    out[0] = r.magnification;
    out[1] = r.relative_error;
}

// ensure_binary_caustic_cache (finite_source_magnifier.cpp:4014-4105): flattened branches,
// bbox {min_x, max_x, min_y, max_y}, max segment length; returns points per branch.
int ref_caustic_cache(double s, double q, int bins, double* branch_xy, int cap_per_branch,
                      double* bbox, double* max_seg)
{
    mag::FiniteSourceSettings settings;
    settings.caustic_bins = bins;
    const mag::FiniteSourceMagnifier fm(settings);
    fm.ensure_binary_caustic_cache(s, q);
    int per = 0;
    for (std::size_t b = 0; b < fm.caustic_cache_branches_.size(); ++b) {
        const auto& br = fm.caustic_cache_branches_[b];
        per = static_cast<int>(br.size());
        for (int j = 0; j < per && j < cap_per_branch; ++j) {
            branch_xy[(b * cap_per_branch + j) * 2] = br[j].x;
            branch_xy[(b * cap_per_branch + j) * 2 + 1] = br[j].y;
        }
    }
    bbox[0] = fm.caustic_cache_min_x_;
    bbox[1] = fm.caustic_cache_max_x_;
    bbox[2] = fm.caustic_cache_min_y_;
    bbox[3] = fm.caustic_cache_max_y_;
    *max_seg = fm.caustic_cache_max_seg_len_;
    return per;
}

// Caustic distances used by the decision tree: out = {sampled, refined}.
void ref_caustic_distances(double s, double q, int bins, double x, double y, double search_radius,
                           double* out)
{
    mag::FiniteSourceSettings settings;
    settings.caustic_bins = bins;
    const mag::FiniteSourceMagnifier fm(settings);
    const double sampled = fm.binary_sampled_caustic_distance(s, q, {x, y}, search_radius);
    out[0] = sampled;
    out[1] = fm.binary_caustic_distance(s, q, {x, y}, sampled);
}

// critical_sources_at_phase (finite_source_magnifier.cpp:1622-1641); returns the count.
int ref_critical_sources(double s, double q, double phi, double* out)
{
    const auto mapper = mag::make_binary_lens_mapper(s, q);
    const auto v = mag::critical_sources_at_phase(mapper, s, q, phi);
    for (std::size_t i = 0; i < v.size(); ++i) {
        out[2 * i] = v[i].x;
        out[2 * i + 1] = v[i].y;
    }
    return static_cast<int>(v.size());
}

// LD table brightness (finite_source_magnifier.cpp:3979-4012).
double ref_ld_brightness(double c, double d, double r2)
{
    mag::FiniteSourceSettings settings;
    settings.limb_darkening_c = c;
    settings.limb_darkening_d = d;
    const mag::FiniteSourceMagnifier fm(settings);
    fm.ensure_limb_darkening_table();
    return fm.limb_darkening_table_brightness(r2);
}

// The static-binary light-curve loop of evaluate_binary_light_curve_numpy
// (python/lcbinint_pybind.cpp:1087-1174, the direct_static_binary branch, VBM convention):
// tau, source position, effective_q = 1/q, binary_mag0 then binary_mag with one
// magnifier reused across epochs.  Returns 0, or 1 on a non-finite magnification.
int ref_light_curve_static(const ref_fs_settings* st, const double* times, int n, double t0,
                           double tE, double u0, double alpha, double s, double q, double rho,
                           double* out, int* method)
{
    const mag::PointSourceMagnifier pm;
    const mag::FiniteSourceMagnifier fm(to_settings(st));
    const double cos_alpha = std::cos(alpha);
    const double sin_alpha = std::sin(alpha);
    const double inverse_tE = 1.0 / tE;
    const double effective_q = q != 0.0 ? 1.0 / q : q;
    for (int i = 0; i < n; ++i) {
        const double tau = (times[i] - t0) * inverse_tE;
        const lcbinint::SourcePosition src {tau * cos_alpha - u0 * sin_alpha,
                                       tau * sin_alpha + u0 * cos_alpha};
        const auto point = pm.binary_mag0(s, effective_q, src);
        if (rho == 0.0) {
            out[i] = point.magnification;
            if (method) method[i] = 0;
            continue;
        }
        const auto r = fm.binary_mag(s, effective_q, src, std::abs(rho), point.magnification,
                                     nullptr, true);
        out[i] = r.magnification;
        if (method) method[i] = static_cast<int>(r.decision.method);
        if (!std::isfinite(r.magnification)) return 1;
    }
    return 0;
}

} // extern "C"
