// CPU oracle (test infrastructure only): restatement of the lcbinint
// finite-source path -- decision tree, caustic sampling, image seeding,
// Cartesian row-scan and polar flood-fill inverse-ray integration, limb
// darkening and the hexadecapole approximation.  Only tests/, smoke() and
// bench.py's CPU arm load the library built from it.
//
// Citations: FSM = src/lcbinint/magnification/finite_source_magnifier.cpp,
// PSM = src/lcbinint/magnification/point_source_magnifier.cpp of
// NunotaKansuke/lcbinint.  Arithmetic follows the reference operation by
// operation (compiled without contraction) so results are bit-identical on
// the same host.
#pragma once

#include <vector>

namespace oracle {

// FiniteSourceSettings (finite_source_magnifier.hpp:22-38).
struct FsSettings {
    int source_bins = 50;
    int caustic_bins = 1400;
    double grid_ratio = 4.0;
    int polar_source_bins = 0;
    double polar_grid_ratio = 0.0;
    int finite_mode = 1;
    double kinji_threshold = 20.0;
    double hex_threshold = 3.0;
    double adaptive_hex_threshold = 0.001;
    double ld_c = 0.0;
    double ld_d = 0.0;
    int adaptive_source_bins = 0;
    int max_source_bins = 400;
    double tol = 0.0;
    double reltol = 0.0;
};

struct Pt {
    double x, y;
};

// FiniteSourceMethod enum values (finite_source_magnifier.hpp:12-19).
enum Method { kPointSource = 0, kHexadecapole = 1, kCartesian = 2, kPolar = 3 };

struct FsResult {
    double magnification;
    int method;
    double error_estimate;
    int refinement_level;
    bool converged;
};

struct CartesianDiagnostics {
    int seed_count = 0, processed = 0, fold = 0, boundary_rows = 0, gap_repairs = 0, overlaps = 0;
    double max_jump = 0.0, estimated_error = 0.0;
};

// FiniteSourceMagnifier::binary_mag (FSM:4633-4843) for one source position,
// with a fresh magnifier (its caches only memoise).
FsResult binary_mag(const FsSettings& st, double s, double q, double x, double y, double rho, double a_ps,
                    bool ps_exact);

// Seeds as fixed_inverse_ray_binary builds them (FSM:3055-3064).
std::vector<Pt> seeds(const FsSettings& st, double s, double q, double x, double y, double rho);

// inverse_ray_cartesian_binary_mag with given seeds (FSM:2470-2768).
double cartesian(const FsSettings& st, double s, double q, double x, double y, double rho,
                 const std::vector<Pt>& seeds, CartesianDiagnostics* diag);

// The polar integral with its cells summed exactly (a 128-bit fixed-point
// accumulator with 64 fraction bits, as the device sums them) and how many
// cells it counted; filled by every polar integration while the pointer is set.
struct PolarFixedSum {
    double value = 0.0;
    unsigned long long cells = 0;
};
extern thread_local PolarFixedSum* g_polar_fixed;

// inverse_ray_polar_boundary_binary with given seeds (FSM:1156-1319).
double polar(const FsSettings& st, double s, double q, double x, double y, double rho, const std::vector<Pt>& seeds);

// hexadecapole_binary (FSM:792-847): {magnification, relative error}.
void hexadecapole(const FsSettings& st, double s, double q, double x, double y, double rho, const double* a0,
                  double* out);

// Caustic cache (FSM:4014-4105): 4 tracked branches, bbox, max segment.
struct CausticCache {
    std::vector<Pt> branches[4];
    std::vector<Pt> points;
    double min_x, max_x, min_y, max_y, step_x, step_y, max_seg_len;
    static constexpr int kGrid = 128;
    std::vector<std::vector<int>> grid;
    struct Ref {
        int branch, pos;
    };
    std::vector<std::vector<Ref>> branch_grid;
};
void build_caustic_cache(double s, double q, int caustic_bins, CausticCache* cc);
double sampled_caustic_distance(const CausticCache& cc, double x, double y, double search_radius);
double caustic_distance(const CausticCache& cc, double x, double y, double hint);

// Critical-curve sources at one phase (FSM:1622-1641).
int critical_sources(double s, double q, double phi, Pt* out);

double ld_brightness(double c, double d, double r2);

// Largest row count one seed's scans reached in the last cartesian() call.
int last_max_rows();

} // namespace oracle
