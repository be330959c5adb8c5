// Host-only helpers of the engine: physical constants, lunar ephemeris rows
// and the synthetic population generator. Compiled without FMA contraction
// (ks_host.cpp) so the per-step lunar terms match the reference bit for bit.
#pragma once

#include <cstdint>

#include "ks_types.h"

namespace ks {

// src/core/orbital.hpp:19-30
constexpr double kPi = 3.14159265358979323846;
constexpr double kDeg = kPi / 180.0;
constexpr double kMuEarth = 398600.4418;
constexpr double kMuMoon = 4902.800066;
constexpr double kREarth = 6378.137;
constexpr double kJ2 = 1.08262668e-3;
constexpr double kDefaultEpochJd = 2461253.916666667;

// 1.5 * J2 * MU_EARTH * R_EARTH * R_EARTH, evaluated left to right
// (src/core/orbital.cpp:96).
double j2_numerator();

// Moon position (ECI km) at Julian date jd.
void moon_position(double jd, double out[3]);

// The three lunar stages of the step starting at t (src/core/orbital.cpp:287-289),
// each with its indirect term rm * (MU_MOON / |rm|^3) (src/core/orbital.cpp:103).
void moon_stages(double epoch_jd, double t, double dt, MoonStage out[3]);

// One lunar stage at Julian date jd (position and indirect term).
void moon_stage_at(double jd, MoonStage& out);

// The stages of a sub-step of span_s seconds from Julian date jd0, with the
// Julian dates formed as src/core/breakup.cpp:211-214 forms them for fragments.
void moon_stages_from(double jd0, double span_s, MoonStage out[3]);

}  // namespace ks
