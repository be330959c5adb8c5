// Host-only parts of the engine: lunar ephemeris rows and constants. Built with -ffp-contract=off and no
// -march, so every operation is a separately rounded IEEE double operation,
// as in the reference's CPU build.
#include <cmath>
#include <cstdint>

#include "kessler_b200.h"
#include "ks_host.h"

namespace ks {

double j2_numerator() {
    // Left to right, each product rounded: the value the reference's constant
    // expression folds to (src/core/orbital.cpp:96).
    volatile double k = 1.5;
    k = k * kJ2;
    k = k * kMuEarth;
    k = k * kREarth;
    k = k * kREarth;
    return k;
}

namespace {

double wrap360(double d) { return std::fmod(std::fmod(d, 360.0) + 360.0, 360.0); }

}  // namespace

// Meeus, Astronomical Algorithms ch. 47: mean elements of the Moon and the
// principal periodic terms in longitude, latitude and distance, rotated from
// ecliptic to equatorial by the mean obliquity. The term selection and the
// evaluation order are those of the reference (src/core/orbital.cpp:53-85),
// so both programs feed RK4 the same lunar positions bit for bit.
void moon_position(double jd, double out[3]) {
    const double T = (jd - 2451545.0) / 36525.0;
    const double Lp = wrap360(218.3164477 + 481267.88123421 * T);
    double D = wrap360(297.8501921 + 445267.1114034 * T);
    double M = wrap360(357.5291092 + 35999.0502909 * T);
    double Mp = wrap360(134.9633964 + 477198.8675055 * T);
    double F = wrap360(93.2720950 + 483202.0175233 * T);
    D *= kDeg;
    M *= kDeg;
    Mp *= kDeg;
    F *= kDeg;
    const double lon = Lp + 6.288774 * std::sin(Mp) + 1.274027 * std::sin(2 * D - Mp)
                     + 0.658314 * std::sin(2 * D) + 0.213618 * std::sin(2 * Mp)
                     - 0.185116 * std::sin(M) - 0.114332 * std::sin(2 * F)
                     + 0.058793 * std::sin(2 * D - 2 * Mp) + 0.057066 * std::sin(2 * D - M - Mp)
                     + 0.053322 * std::sin(2 * D + Mp) + 0.045758 * std::sin(2 * D - M);
    const double lat = 5.128122 * std::sin(F) + 0.280602 * std::sin(Mp + F)
                     + 0.277693 * std::sin(Mp - F) + 0.173237 * std::sin(2 * D - F)
                     + 0.055413 * std::sin(2 * D - Mp + F) + 0.046271 * std::sin(2 * D - Mp - F);
    const double dist = 385000.56 - 20905.355 * std::cos(Mp) - 3699.111 * std::cos(2 * D - Mp)
                      - 2955.968 * std::cos(2 * D) - 569.925 * std::cos(2 * Mp)
                      + 48.888 * std::cos(M) - 3.149 * std::cos(2 * F)
                      + 246.158 * std::cos(2 * D - 2 * Mp) - 152.138 * std::cos(2 * D - M - Mp)
                      - 170.733 * std::cos(2 * D + Mp) - 204.586 * std::cos(2 * D - M);
    const double l = lon * kDeg, b = lat * kDeg;
    const double eps = (23.439291 - 0.0130042 * T) * kDeg;
    const double xe = dist * std::cos(b) * std::cos(l);
    const double ye = dist * std::cos(b) * std::sin(l);
    const double ze = dist * std::sin(b);
    out[0] = xe;
    out[1] = ye * std::cos(eps) - ze * std::sin(eps);
    out[2] = ye * std::sin(eps) + ze * std::cos(eps);
}

void moon_stage_at(double jd, MoonStage& out) {
    double p[3];
    moon_position(jd, p);
    const double mn = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    const double s = kMuMoon / (mn * mn * mn);
    out.mx = p[0];
    out.my = p[1];
    out.mz = p[2];
    out.ix = p[0] * s;
    out.iy = p[1] * s;
    out.iz = p[2] * s;
}

void moon_stages(double epoch_jd, double t, double dt, MoonStage out[3]) {
    const double jd[3] = {epoch_jd + t / 86400.0, epoch_jd + (t + dt / 2) / 86400.0,
                          epoch_jd + (t + dt) / 86400.0};
    for (int k = 0; k < 3; ++k) moon_stage_at(jd[k], out[k]);
}

void moon_stages_from(double jd0, double span_s, MoonStage out[3]) {
    moon_stage_at(jd0, out[0]);
    moon_stage_at(jd0 + span_s / 2 / 86400.0, out[1]);
    moon_stage_at(jd0 + span_s / 86400.0, out[2]);
}

}  // namespace ks

extern "C" {

void ks_moon_position(double jd, double out[3]) { ks::moon_position(jd, out); }

}  // extern "C"
