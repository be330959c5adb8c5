// NASA Standard Breakup Model fragmentation of one collision, on the host.
//
// Follows the reference's Fragmentation (src/core/breakup.cpp:121-360), which
// implements Johnson, Krisko, Liou & Anz-Meador, "NASA's new breakup model of
// EVOLVE 4.0", Adv. Space Res. 28(9), 2001: catastrophic test at a specific
// energy threshold, N(>L) = 0.1 M^0.75 L^-1.71 fragments above L_c, power-law
// sizes, the SBM area-to-mass distributions, log-normal isotropic delta-v,
// per-parent mass budgets and hyperbolic escapes dropped.
//
// Every draw is taken in the reference's order from a 64-bit Mersenne Twister
// (the engine the C++ standard fixes bit for bit) with 53-bit uniforms,
// Box-Muller normals and Knuth / Hormann-PTRS Poisson draws, and every
// expression keeps the reference's operation order (this file is compiled
// without FMA contraction): a run fragments exactly as the reference does.
//
// Fragments are returned at their birth state; the engine advances them to the
// end of the step on the device (the reference's rk4 over the remaining time,
// src/core/breakup.cpp:304-306).
#pragma once

#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "ks_records.h"

namespace ks {

// src/core/breakup.hpp:64-77
class SbmRng {
public:
    explicit SbmRng(uint64_t seed = 1) : engine_(seed) {}
    double uniform();              // [0, 1), 53 bits
    double normal();               // N(0, 1), Box-Muller on (1 - u1, u2)
    long long poisson(double mean);  // Knuth below a mean of 10, Hormann's PTRS above
    std::string state() const;                // engine state, as the standard library prints it
    bool set_state(const std::string& text);  // restores a printed state

private:
    std::mt19937_64 engine_;
};

struct SbmParams {
    double lc_m = 0.10;                 // smallest fragment followed (m)
    double catastrophic_j_per_g = 40.0;  // specific-energy threshold
};

struct SbmParent {
    int64_t index = -1;  // object index; -1 for the fictitious projectile of a forced impact
    double s[6] = {0, 0, 0, 0, 0, 0};
    double mass_kg = 0;
    double size_m = 0;
};

struct SbmFragment {
    double s[6];          // birth state
    double size_m, mass_kg, area_to_mass;
};

// What one event does to its parents.
struct SbmOutcome {
    bool kill_target = false, kill_projectile = false;
    bool reduce_target = false;
    double target_mass_after = 0;
};

// Default mass of an object whose mass is not known (src/core/breakup.cpp:19, 30-32).
double sbm_mass_or_default(double mass_kg);

// One collision (src/core/breakup.cpp:192-314). Fills ev's physical fields
// (t, catastrophic, v_rel, energy, masses, M, expected and created fragments,
// fragment mass, escapes, position); the caller owns id, step, realisation,
// target/projectile indices and first_fragment.
void sbm_fragment(SbmRng& rng, const SbmParams& p, const SbmParent& target, const SbmParent& projectile, double t,
                  ks_breakup_event& ev, std::vector<SbmFragment>& out, SbmOutcome& outcome);

// Parents of a forced impact (src/core/breakup.cpp:340-360): the fictitious
// projectile moves at the target's speed, turned about the local vertical so
// that the relative speed is v_rel; the heavier of the two is the target.
// Consumes one uniform draw (the side of the crossing).
void sbm_impact_parents(SbmRng& rng, int64_t target_index, const double s[6], double target_mass_kg,
                        double target_size_m, double projectile_mass_kg, double v_rel_km_s, SbmParent& tgt,
                        SbmParent& prj);

// State at fraction s of a step from the states and velocities at both ends
// (cubic Hermite, src/core/collision.cpp:77-90, 289-292).
void interpolate_state(const double a[6], const double b[6], double dt, double s, double out[6]);

}  // namespace ks
