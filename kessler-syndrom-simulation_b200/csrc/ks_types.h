// Plain data types shared by host and device code of the engine.
#pragma once

namespace ks {

// Per-stage lunar quantities, computed on the host with the same operations:
// position rm and the indirect term rm * (MU_MOON / (|rm|^3)).
struct MoonStage {
    double mx, my, mz;
    double ix, iy, iz;
};

// Physical constants (src/core/orbital.hpp:22-26), plus the J2 numerator
// 1.5 * J2 * MU_EARTH * R_EARTH * R_EARTH evaluated left to right on the host.
struct ForceConsts {
    double neg_mu_earth;  // -MU_EARTH
    double k_j2;          // ((((1.5 * J2) * MU_EARTH) * R_EARTH) * R_EARTH)
    double mu_moon;
    double r_earth;
};

constexpr double kGravityGradient = 2e-6;  // src/core/collision_filter.hpp:26

}  // namespace ks
