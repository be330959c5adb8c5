// NASA Standard Breakup Model on the host; see ks_breakup.h. Compiled without
// FMA contraction: each expression keeps the operation order of
// src/core/breakup.cpp so that fragments are identical to the reference's.
#include "ks_breakup.h"

#include <algorithm>
#include <cmath>
#include <sstream>

#include "ks_host.h"

namespace ks {

namespace {

// src/core/breakup.cpp:19, 24, 28
constexpr double kFallbackMassKg = 100.0;
constexpr double kProjectileDensityKgM3 = 300.0;
constexpr long long kMaxFragmentsPerEvent = 200000;
// Number law exponent and area of a fragment of size L (A = 0.540424 L^2), SBM.
constexpr double kSizeExponent = 1.71;
constexpr double kAreaCoeff = 0.540424;

// Piecewise-linear in x, constant outside [x0, x1] (src/core/breakup.cpp:35-39).
double lerp_clamped(double x, double x0, double y0, double x1, double y1) {
    if (x <= x0) return y0;
    if (x >= x1) return y1;
    return y0 + (y1 - y0) * (x - x0) / (x1 - x0);
}

// log10(A/m) of a fragment of size 10^lam (src/core/breakup.cpp:165-190):
// above 11 cm a two-component normal mixture, below 8 cm one normal, and in
// between one or the other with a probability linear in the size.
double draw_log_area_to_mass(SbmRng& rng, double lam) {
    const double size = std::pow(10.0, lam);
    auto mixture = [&]() {
        const double w = lerp_clamped(lam, -1.95, 0.0, 0.55, 1.0);
        const double mu_a = lerp_clamped(lam, -1.1, -0.6, 0.0, -0.95);
        const double sd_a = lerp_clamped(lam, -1.3, 0.1, -0.3, 0.3);
        const double mu_b = lerp_clamped(lam, -0.7, -1.2, -0.1, -2.0);
        const double sd_b = lerp_clamped(lam, -0.5, 0.5, -0.3, 0.3);
        if (rng.uniform() < w) return mu_a + sd_a * rng.normal();
        return mu_b + sd_b * rng.normal();
    };
    auto single = [&]() {
        const double mu = lerp_clamped(lam, -1.75, -0.3, -1.25, -1.0);
        const double sd = lam <= -3.5 ? 0.2 : 0.2 + 0.1333 * (lam + 3.5);
        return mu + sd * rng.normal();
    };
    if (size >= 0.11) return mixture();
    if (size <= 0.08) return single();
    return rng.uniform() < (size - 0.08) / 0.03 ? mixture() : single();
}

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

std::string SbmRng::state() const {
    std::ostringstream os;
    os << engine_;
    return os.str();
}

bool SbmRng::set_state(const std::string& text) {
    std::istringstream is(text);
    std::mt19937_64 e;
    is >> e;
    if (!is) return false;
    engine_ = e;
    return true;
}

double SbmRng::uniform() { return static_cast<double>(engine_() >> 11) * 0x1.0p-53; }

double SbmRng::normal() {
    const double u1 = 1.0 - uniform();  // (0, 1]: finite logarithm
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
}

long long SbmRng::poisson(double mean) {
    if (mean <= 0.0) return 0;
    if (mean < 10.0) {
        // Knuth: multiply uniforms until the product drops to exp(-mean).
        const double stop = std::exp(-mean);
        long long k = 0;
        double prod = uniform();
        while (prod > stop) {
            ++k;
            prod *= uniform();
        }
        return k;
    }
    // Transformed rejection with squeeze, PTRS (W. Hormann, "The transformed
    // rejection method for generating Poisson random variables", Insurance:
    // Mathematics and Economics 12, 1993), constants from the paper.
    const double sq = std::sqrt(mean), lmean = std::log(mean);
    const double b = 0.931 + 2.53 * sq;
    const double a = -0.059 + 0.02483 * b;
    const double ainv = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (;;) {
        const double u = uniform() - 0.5;
        const double v = uniform();
        const double us = 0.5 - std::fabs(u);
        if (us <= 0.0 || v <= 0.0) continue;
        const double k = std::floor((2.0 * a / us + b) * u + mean + 0.43);
        if (us >= 0.07 && v <= vr) return static_cast<long long>(k);
        if (k < 0.0 || (us < 0.013 && v > us)) continue;
        if (std::log(v) + std::log(ainv) - std::log(a / (us * us) + b) <= -mean + k * lmean - std::lgamma(k + 1.0))
            return static_cast<long long>(k);
    }
}

double sbm_mass_or_default(double mass_kg) { return mass_kg > 0 ? mass_kg : kFallbackMassKg; }

void sbm_fragment(SbmRng& rng, const SbmParams& p, const SbmParent& tgt, const SbmParent& prj, double t,
                  ks_breakup_event& ev, std::vector<SbmFragment>& out, SbmOutcome& outcome) {
    ev.t = t;
    ev.target_mass_kg = tgt.mass_kg;
    ev.projectile_mass_kg = prj.mass_kg;
    for (int q = 0; q < 3; ++q) ev.position[q] = tgt.s[q];

    const double dv3[3] = {tgt.s[3] - prj.s[3], tgt.s[4] - prj.s[4], tgt.s[5] - prj.s[5]};
    const double vrel = std::sqrt(dot3(dv3, dv3));  // km/s
    ev.v_rel_km_s = vrel;
    // 1/2 m_p (1000 v)^2 [J] per gram of target
    ev.energy_j_per_g = 500.0 * prj.mass_kg * vrel * vrel / tgt.mass_kg;
    const bool catastrophic = ev.energy_j_per_g >= p.catastrophic_j_per_g;
    ev.catastrophic = catastrophic ? 1 : 0;

    // Mass each parent contributes: both whole parents in a catastrophic
    // event; otherwise the projectile plus the ejecta m_p v^2 - m_p.
    double budget[2];
    if (catastrophic) {
        budget[0] = tgt.mass_kg;
        budget[1] = prj.mass_kg;
    } else {
        budget[1] = prj.mass_kg;
        budget[0] = std::max(0.0, prj.mass_kg * vrel * vrel - prj.mass_kg);
    }
    const double msbm = budget[0] + budget[1];
    ev.sbm_mass_kg = msbm;

    outcome = SbmOutcome{};
    outcome.kill_projectile = prj.index >= 0;
    if (tgt.index >= 0) {
        if (catastrophic) outcome.kill_target = true;
        else {
            outcome.reduce_target = true;
            outcome.target_mass_after = std::max(tgt.mass_kg - budget[0], 0.0);
        }
    }

    const double lc = p.lc_m;
    ev.expected_fragments = msbm > 0 ? 0.1 * std::pow(msbm, 0.75) * std::pow(lc, -kSizeExponent) : 0.0;
    long long count = 0;
    if (ev.expected_fragments > 0) count = std::min(rng.poisson(ev.expected_fragments), kMaxFragmentsPerEvent);

    const SbmParent* parent[2] = {&tgt, &prj};
    double used[2] = {0.0, 0.0};
    const double p_target = msbm > 0 ? budget[0] / msbm : 0.0;
    ev.fragments = 0;
    ev.escaped = 0;
    ev.fragments_mass_kg = 0.0;
    out.reserve(out.size() + static_cast<size_t>(count));
    for (long long k = 0; k < count; ++k) {
        const int side = rng.uniform() < p_target ? 0 : 1;
        const SbmParent& par = *parent[side];
        // Size from N(>L) ~ L^-1.71 truncated to [L_c, parent size], by inversion.
        const double lmax = par.size_m;
        if (lmax <= lc) continue;
        const double tail = std::pow(lmax / lc, -kSizeExponent);
        const double size = lc * std::pow(1.0 - rng.uniform() * (1.0 - tail), -1.0 / kSizeExponent);

        const double chi = draw_log_area_to_mass(rng, std::log10(size));
        const double area = kAreaCoeff * size * size;
        const double mass = area / std::pow(10.0, chi);
        if (used[side] + mass > budget[side]) continue;  // this parent's budget is spent for this size
        used[side] += mass;

        // Delta-v: log-normal magnitude capped at the impact speed, isotropic direction.
        double dv_ms = std::pow(10.0, 0.9 * chi + 2.9 + 0.4 * rng.normal());
        dv_ms = std::min(dv_ms, vrel * 1000.0);
        const double cz = 2.0 * rng.uniform() - 1.0;
        const double phi = 2.0 * kPi * rng.uniform();
        const double sz = std::sqrt(std::max(0.0, 1.0 - cz * cz));
        const double dir[3] = {sz * std::cos(phi), sz * std::sin(phi), cz};
        SbmFragment f;
        for (int q = 0; q < 3; ++q) {
            f.s[q] = par.s[q];
            f.s[3 + q] = par.s[3 + q] + dir[q] * (dv_ms * 1e-3);
        }
        // Hyperbolic (non-negative orbital energy): leaves Earth, dropped.
        if (0.5 * dot3(f.s + 3, f.s + 3) - kMuEarth / std::sqrt(dot3(f.s, f.s)) >= 0.0) {
            ++ev.escaped;
            continue;
        }
        f.size_m = size;
        f.mass_kg = mass;
        f.area_to_mass = std::pow(10.0, chi);
        out.push_back(f);
        ++ev.fragments;
        ev.fragments_mass_kg += mass;
    }
}

void sbm_impact_parents(SbmRng& rng, int64_t target_index, const double s[6], double target_mass_kg,
                        double target_size_m, double projectile_mass_kg, double v_rel_km_s, SbmParent& tgt,
                        SbmParent& prj) {
    const double* r = s;
    const double* v = s + 3;
    const double rn = std::sqrt(dot3(r, r));
    const double up[3] = {r[0] * (1.0 / rn), r[1] * (1.0 / rn), r[2] * (1.0 / rn)};
    const double vu = dot3(v, up);
    const double vhz[3] = {v[0] - up[0] * vu, v[1] - up[1] * vu, v[2] - up[2] * vu};
    const double vh = std::sqrt(dot3(vhz, vhz));
    // |v_p - v| = 2 |v_h| sin(theta / 2)
    double theta = v_rel_km_s >= 2.0 * vh ? kPi : 2.0 * std::asin(v_rel_km_s / (2.0 * vh));
    if (rng.uniform() < 0.5) theta = -theta;
    const double c = std::cos(theta), sn = std::sin(theta);
    const double kxv[3] = {up[1] * v[2] - up[2] * v[1], up[2] * v[0] - up[0] * v[2], up[0] * v[1] - up[1] * v[0]};
    const double kv = dot3(up, v);
    double vp[3];
    for (int q = 0; q < 3; ++q) vp[q] = v[q] * c + kxv[q] * sn + up[q] * (kv * (1.0 - c));  // Rodrigues

    SbmParent a, b;
    a.index = target_index;
    for (int q = 0; q < 6; ++q) a.s[q] = s[q];
    a.mass_kg = sbm_mass_or_default(target_mass_kg);
    a.size_m = target_size_m;
    b.index = -1;
    for (int q = 0; q < 3; ++q) {
        b.s[q] = r[q];
        b.s[3 + q] = vp[q];
    }
    b.mass_kg = projectile_mass_kg;
    b.size_m = std::cbrt(projectile_mass_kg / kProjectileDensityKgM3);
    if (b.mass_kg > a.mass_kg) {
        tgt = b;
        prj = a;
    } else {
        tgt = a;
        prj = b;
    }
}

void interpolate_state(const double a[6], const double b[6], double dt, double s, double out[6]) {
    const double s2 = s * s, s3 = s2 * s;
    const double h00 = 2 * s3 - 3 * s2 + 1, h10 = s3 - 2 * s2 + s, h01 = -2 * s3 + 3 * s2, h11 = s3 - s2;
    const double d00 = 6 * s2 - 6 * s, d10 = 3 * s2 - 4 * s + 1, d01 = -6 * s2 + 6 * s, d11 = 3 * s2 - 2 * s;
    const double inv_dt = 1.0 / dt;
    for (int q = 0; q < 3; ++q) {
        const double p0 = a[q], m0 = a[3 + q] * dt, p1 = b[q], m1 = b[3 + q] * dt;
        out[q] = p0 * h00 + m0 * h10 + p1 * h01 + m1 * h11;
        out[3 + q] = (p0 * d00 + m0 * d10 + p1 * d01 + m1 * d11) * inv_dt;
    }
}

}  // namespace ks
