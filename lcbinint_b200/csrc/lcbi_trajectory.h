// Source trajectories with annual and terrestrial parallax and xallarap, on
// the host (not public ABI).  Trajectory::source_position
// (src/lcbinint/model/trajectory.cpp:436-463) restated with the reference's
// arithmetic and C library calls, so positions are bit-identical.
#pragma once

#include "../../include/lcbinint_b200.h"

#include <array>
#include <vector>

namespace lcbi {

struct EarthState {
    double time = 0.0;
    std::array<double, 3> position{};
    std::array<double, 3> velocity{};
};

// The Earth's ephemeris (JPL Horizons vector table: JD, x, y, z, vx, vy, vz
// between $$SOE and $$EOE, trajectory.cpp:147-177).  Loaded once from the file
// named by LCBININT_EARTH_EPHEMERIS, as the reference does, unless set first
// with set_earth_ephemeris.  Returns the number of states, or -1 if the file
// could not be read.
int set_earth_ephemeris(const char* path);
const std::vector<EarthState>& earth_ephemeris();

// One parameter set's trajectory: the annual-parallax projector is built once
// (the reference caches it per thread for the same sky position and time).
struct Trajectory {
    lcbi_params p{};
    const std::vector<EarthState>* eph = nullptr;  // the ephemeris, fetched once per set
    bool annual = false;
    double time_offset = 0.0, eph_reference_time = 0.0;
    std::array<double, 3> north{}, east{}, event{};
    double ref_pn = 0.0, ref_pe = 0.0, ref_vn = 0.0, ref_ve = 0.0;  // projected reference state
};

Trajectory make_trajectory(const lcbi_params& p);
// Source position at `time`; xallarap_type as lcbi_options::xallarap_param_type.
void source_position(const Trajectory& tr, double time, bool vbm, int xallarap_type, double* x, double* y);

} // namespace lcbi
