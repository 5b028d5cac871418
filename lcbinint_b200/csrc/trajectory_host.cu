// Host-side source trajectories: annual parallax from an Earth ephemeris with
// light-time correction, terrestrial parallax, and xallarap (angular velocity
// or orbital elements) -- src/lcbinint/model/trajectory.cpp restated with the
// same operation order and C library calls, so the positions are the
// reference's bit for bit.  The per-epoch positions feed the GPU pipeline.
#include "lcbi_trajectory.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <mutex>
#include <sstream>
#include <string>

namespace lcbi {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kDegreeToRadian = kPi / 180.0;
constexpr double kReducedJulianDateOrigin = 2450000.0;
constexpr double kAuLightTravelDays = 0.005775518331436995;
constexpr double kEarthRadiusAU = 4.2635212e-5;
constexpr double kSiderealDegPerDay = 360.98564736629;

using V3 = std::array<double, 3>;

double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

V3 cross3(const V3& a, const V3& b)
{
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

V3 unit3(const V3& v)
{
    const double norm = std::sqrt(dot3(v, v));
    if (norm == 0.0 || !std::isfinite(norm)) {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        return {nan, nan, nan};
    }
    const double f = 1.0 / norm;
    return {v[0] * f, v[1] * f, v[2] * f};
}

V3 event_unit(double ra_deg, double dec_deg)
{
    const double ra = ra_deg * kDegreeToRadian;
    const double dec = dec_deg * kDegreeToRadian;
    const double cd = std::cos(dec);
    return {std::cos(ra) * cd, std::sin(ra) * cd, std::sin(dec)};
}

V3 east_of(double ra_deg, double dec_deg) { return unit3(cross3(V3{0.0, 0.0, 1.0}, event_unit(ra_deg, dec_deg))); }

V3 north_of(double ra_deg, double dec_deg) { return cross3(event_unit(ra_deg, dec_deg), east_of(ra_deg, dec_deg)); }

std::string strip(const std::string& s)
{
    const auto b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return "";
    const auto e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

// Comma-separated numbers of one table line, the second column (the calendar
// date) skipped, unparsable tokens dropped (trajectory.cpp:104-126).
std::vector<double> numeric_fields(const std::string& line)
{
    std::vector<double> out;
    std::stringstream in(line);
    std::string tok;
    int column = 0;
    while (std::getline(in, tok, ',')) {
        tok = strip(tok);
        if (tok.empty()) continue;
        if (column == 1) {
            ++column;
            continue;
        }
        try {
            out.push_back(std::stod(tok));
        } catch (const std::exception&) {
        }
        ++column;
    }
    return out;
}

std::vector<EarthState> read_table(const char* path, bool* ok)
{
    std::vector<EarthState> states;
    std::ifstream in(path ? path : "");
    *ok = static_cast<bool>(in);
    if (!in) return states;
    bool block = false;
    std::string line;
    while (std::getline(in, line)) {
        const std::string s = strip(line);
        if (!block) {
            if (s.rfind("$$SOE", 0) == 0) block = true;
            continue;
        }
        if (s.rfind("$$EOE", 0) == 0) break;
        const auto f = numeric_fields(s);
        if (f.size() < 7) continue;
        states.push_back({f[0], {f[1], f[2], f[3]}, {f[4], f[5], f[6]}});
    }
    return states;
}

std::mutex g_eph_mutex;
bool g_eph_loaded = false;
std::vector<EarthState> g_eph;

// interpolate_earth_state (trajectory.cpp:185-207): linear between the
// bracketing states, NaN outside the table.  A time equal to the last state's
// reads the last interval.
void interpolate(const std::vector<EarthState>& st, double time, V3* pos, V3* vel)
{
    if (st.size() < 2 || time < st.front().time || time > st.back().time) {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        *pos = {nan, nan, nan};
        *vel = {nan, nan, nan};
        return;
    }
    auto upper = std::upper_bound(st.begin(), st.end(), time,
                                  [](double v, const EarthState& s) { return v < s.time; });
    if (upper == st.end()) --upper;
    const auto hi = upper == st.begin() ? st.begin() + 1 : upper;
    const auto lo = hi - 1;
    const double dt = hi->time - lo->time;
    const double w = dt != 0.0 ? (time - lo->time) / dt : 0.0;
    for (int k = 0; k < 3; ++k) {
        (*pos)[k] = lo->position[k] + (hi->position[k] - lo->position[k]) * w;
        (*vel)[k] = lo->velocity[k] + (hi->velocity[k] - lo->velocity[k]) * w;
    }
}

double time_offset_of(double reference_time)
{
    return reference_time < kReducedJulianDateOrigin ? kReducedJulianDateOrigin : 0.0;
}

// light_time_corrected_time (trajectory.cpp:259-268): five fixed-point steps.
double emit_time(const Trajectory& tr, double observation_time)
{
    double emit = observation_time;
    for (int i = 0; i < 5; ++i) {
        V3 pos, vel;
        interpolate(*tr.eph, emit, &pos, &vel);
        const double light = dot3(pos, tr.event) * kAuLightTravelDays;
        emit = observation_time - light;
    }
    return emit;
}

void projected(const Trajectory& tr, double time, double* pn, double* pe, double* vn, double* ve)
{
    V3 pos, vel;
    interpolate(*tr.eph, time, &pos, &vel);
    *pn = -dot3(pos, tr.north);
    *pe = -dot3(pos, tr.east);
    *vn = -dot3(vel, tr.north);
    *ve = -dot3(vel, tr.east);
}

double solve_kepler(double mean_anomaly, double ecc)
{
    double E = mean_anomaly + ecc * std::sin(mean_anomaly);
    for (int i = 0; i < 10; ++i) {
        const double f = E - ecc * std::sin(E) - mean_anomaly;
        const double fp = 1.0 - ecc * std::cos(E);
        const double delta = f / fp;
        E -= delta;
        if (std::abs(delta) < 1.0e-13) break;
    }
    return E;
}

std::array<double, 2> kepler_xy(double time, double t0, double period, double ecc, double peri)
{
    const double mean_anom = 2.0 * kPi / period * (time - t0) + peri;
    const double E = solve_kepler(mean_anom, ecc);
    const double cE = std::cos(E);
    const double sE = std::sin(E);
    const double r = 1.0 - ecc * cE;
    const double sq = std::sqrt(std::max(0.0, 1.0 - ecc * ecc));
    const double cf = (cE - ecc) / r;
    const double sf = sq * sE / r;
    return {r * cf, r * sf};
}

} // namespace

int set_earth_ephemeris(const char* path)
{
    std::lock_guard<std::mutex> lock(g_eph_mutex);
    bool ok = false;
    g_eph = read_table(path, &ok);
    g_eph_loaded = true;
    return ok ? static_cast<int>(g_eph.size()) : -1;
}

const std::vector<EarthState>& earth_ephemeris()
{
    std::lock_guard<std::mutex> lock(g_eph_mutex);
    if (!g_eph_loaded) {
        const char* env = std::getenv("LCBININT_EARTH_EPHEMERIS");
        bool ok = false;
        if (env && env[0] != '\0') g_eph = read_table(env, &ok);
        g_eph_loaded = true;
    }
    return g_eph;
}

// The projector of EarthOrbitalParallaxProjector (trajectory.cpp:221-285).
Trajectory make_trajectory(const lcbi_params& p)
{
    Trajectory tr;
    tr.p = p;
    tr.eph = &earth_ephemeris();
    tr.annual = p.piEN != 0.0 || p.piEE != 0.0;
    if (tr.annual) {
        const double reference_time = p.tfix != 0.0 ? p.tfix : p.t0;
        tr.time_offset = time_offset_of(reference_time);
        tr.eph_reference_time = reference_time + tr.time_offset;
        tr.north = north_of(p.ra, p.dec);
        tr.east = east_of(p.ra, p.dec);
        tr.event = event_unit(p.ra, p.dec);
        projected(tr, emit_time(tr, tr.eph_reference_time), &tr.ref_pn, &tr.ref_pe, &tr.ref_vn, &tr.ref_ve);
    }
    return tr;
}

void source_position(const Trajectory& tr, double time, bool vbm, int xallarap_type, double* x, double* y)
{
    const lcbi_params& p = tr.p;
    double tn = (time - p.t0) / p.tE;
    double beta = p.umin;
    if (tr.annual) {
        // apply_annual_parallax (trajectory.cpp:403-432).
        const double eph_time = time + tr.time_offset;
        double pn, pe, vn, ve;
        projected(tr, emit_time(tr, eph_time), &pn, &pe, &vn, &ve);
        const double dt = eph_time - tr.eph_reference_time;
        const double dn = pn - tr.ref_pn - tr.ref_vn * dt;
        const double de = pe - tr.ref_pe - tr.ref_ve * dt;
        tn += p.piEN * dn + p.piEE * de;
        beta += -p.piEE * dn + p.piEN * de;
        // apply_terrestrial_parallax (trajectory.cpp:361-401).
        if (p.obs_lat != 0.0 || p.obs_lon != 0.0) {
            const double lat = p.obs_lat * kDegreeToRadian;
            const double lon = p.obs_lon * kDegreeToRadian;
            const double jd = time + time_offset_of(time);
            const double gmst = (280.46061837 + kSiderealDegPerDay * (jd - 2451545.0)) * kDegreeToRadian;
            const double ha = gmst + lon;
            const double cl = std::cos(lat);
            const V3 r_tel = {kEarthRadiusAU * cl * std::cos(ha), kEarthRadiusAU * cl * std::sin(ha),
                              kEarthRadiusAU * std::sin(lat)};
            const double proj_n = -dot3(r_tel, north_of(p.ra, p.dec));
            const double proj_e = -dot3(r_tel, east_of(p.ra, p.dec));
            tn += p.piEN * proj_n + p.piEE * proj_e;
            beta += -p.piEE * proj_n + p.piEN * proj_e;
        }
    }
    if (xallarap_type == LCBI_XALLARAP_ANGULAR_VELOCITY && (p.xi_1 != 0.0 || p.xi_2 != 0.0)) {
        // apply_xallarap_angular_velocity (trajectory.cpp:287-300).
        const double phit = p.omega_xa * (time - p.t0);
        const double phi = p.phi_xa;
        const double s_inc = std::sin(p.inc_xa);
        const double disp0 = s_inc * (-std::cos(phi) + std::cos(phi + phit) + phit * std::sin(phi));
        const double disp1 = -phit * std::cos(phi) - std::sin(phi) + std::sin(phi + phit);
        tn += p.xi_1 * disp0 + p.xi_2 * disp1;
        beta += p.xi_2 * disp0 - p.xi_1 * disp1;
    } else if (xallarap_type == LCBI_XALLARAP_ORBITAL_ELEMENTS && (p.piEN_xa != 0.0 || p.piEE_xa != 0.0) &&
               p.period_xa > 0.0) {
        // apply_xallarap_orbital_elements (trajectory.cpp:331-359).
        const auto pos_t = kepler_xy(time, p.t0, p.period_xa, p.ecc_xa, p.peri_xa);
        const auto pos_0 = kepler_xy(p.t0, p.t0, p.period_xa, p.ecc_xa, p.peri_xa);
        const double dt_small = p.period_xa * 1.0e-7;
        const auto pos_dt = kepler_xy(p.t0 + dt_small, p.t0, p.period_xa, p.ecc_xa, p.peri_xa);
        const double vx0 = (pos_dt[0] - pos_0[0]) / dt_small;
        const double vy0 = (pos_dt[1] - pos_0[1]) / dt_small;
        const double elapsed = time - p.t0;
        const double dev_x = pos_t[0] - pos_0[0] - vx0 * elapsed;
        const double dev_y = pos_t[1] - pos_0[1] - vy0 * elapsed;
        const double s_inc = std::sin(p.inc_xa);
        const double disp0 = s_inc * dev_x;
        const double disp1 = dev_y;
        tn += p.piEN_xa * disp0 + p.piEE_xa * disp1;
        beta += p.piEE_xa * disp0 - p.piEN_xa * disp1;
    }
    const double ct = std::cos(p.theta);
    const double st = std::sin(p.theta);
    if (vbm) {
        *x = tn * ct - beta * st;
        *y = tn * st + beta * ct;
    } else {
        *x = beta * st + tn * ct;
        *y = beta * ct - tn * st;
    }
}

} // namespace lcbi

extern "C" int lcbi_set_earth_ephemeris(const char* path) { return lcbi::set_earth_ephemeris(path); }
