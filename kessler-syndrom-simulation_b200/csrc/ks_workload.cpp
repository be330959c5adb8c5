// Seeded synthetic population (ks_generate_population): the workload
// generator of the tests and the benchmark, not part of the per-step path.
// A self-contained translation unit, built with -ffp-contract=off and no
// -march like the rest of the host code, so that every build of it (the
// engine library, and the copy the CPU-baseline harness links so that it
// loads nothing of the engine) produces the same populations bit for bit.
#include <cmath>
#include <cstdint>
#include <vector>

#include "kessler_b200.h"
#include "ks_host.h"

namespace ks {
// ---------------------------------------------------------------------------
// Synthetic population
// ---------------------------------------------------------------------------

namespace {

// Counter-based random numbers: splitmix64 finaliser over (seed, object, draw).
uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t seed;
    uint64_t stream;  // object or cloud identifier
    uint64_t draw = 0;
    uint64_t next() {
        return mix64(mix64(seed ^ (stream * 0x9e3779b97f4a7c15ull)) + 0x632be59bd9b4e019ull * (++draw));
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
    double normal() {  // Box-Muller
        const double u1 = 1.0 - uniform();  // (0, 1]
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
};

enum Orbit { LEO = 0, MEO = 1, GEO = 2, GTO = 3 };

struct Elements {
    double a, e, inc, raan, argp, M;
};

double solve_kepler(double M, double e) {
    double E = e < 0.8 ? M : kPi;
    for (int it = 0; it < 60; ++it) {
        const double f = E - e * std::sin(E) - M;
        const double d = f / (1.0 - e * std::cos(E));
        E -= d;
        if (std::fabs(d) < 1e-15) break;
    }
    return E;
}

// Keplerian elements (angles in radians) -> ECI position and velocity.
void elements_to_state(const Elements& el, double s[6]) {
    const double E = solve_kepler(el.M, el.e);
    const double cE = std::cos(E), sE = std::sin(E);
    const double b = std::sqrt(1.0 - el.e * el.e);
    const double r = el.a * (1.0 - el.e * cE);
    const double xp = el.a * (cE - el.e), yp = el.a * b * sE;
    const double k = std::sqrt(kMuEarth * el.a) / r;
    const double vxp = -k * sE, vyp = k * b * cE;
    const double cO = std::cos(el.raan), sO = std::sin(el.raan);
    const double ci = std::cos(el.inc), si = std::sin(el.inc);
    const double cw = std::cos(el.argp), sw = std::sin(el.argp);
    // Columns of R3(-raan) R1(-inc) R3(-argp): perigee direction P and Q.
    const double P[3] = {cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si};
    const double Q[3] = {-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si};
    for (int q = 0; q < 3; ++q) {
        s[q] = xp * P[q] + yp * Q[q];
        s[3 + q] = vxp * P[q] + vyp * Q[q];
    }
}

// Two-body propagation over dt by Lagrange f and g coefficients in the
// eccentric-anomaly difference (Battin, An Introduction to the Mathematics and
// Methods of Astrodynamics, sec. 4.3). Returns false for non-elliptic motion.
bool kepler_propagate(const double s0[6], double dt, double s1[6]) {
    const double r0 = std::sqrt(s0[0] * s0[0] + s0[1] * s0[1] + s0[2] * s0[2]);
    const double v2 = s0[3] * s0[3] + s0[4] * s0[4] + s0[5] * s0[5];
    const double alpha = 2.0 / r0 - v2 / kMuEarth;  // 1/a
    if (!(alpha > 0.0)) return false;
    const double a = 1.0 / alpha;
    const double sqmu = std::sqrt(kMuEarth);
    const double sigma0 = (s0[0] * s0[3] + s0[1] * s0[4] + s0[2] * s0[5]) / sqmu;
    const double n = std::sqrt(kMuEarth / (a * a * a));
    double M = n * dt;
    // Reduce whole revolutions away before solving.
    const double rev = std::floor(M / (2.0 * kPi) + 0.5);
    const double Mred = M - rev * 2.0 * kPi;
    const double sqa = std::sqrt(a);
    double dE = Mred;
    for (int it = 0; it < 100; ++it) {
        const double c = std::cos(dE), s = std::sin(dE);
        const double f = dE + sigma0 / sqa * (1.0 - c) - (1.0 - r0 / a) * s - Mred;
        const double fp = 1.0 + sigma0 / sqa * s - (1.0 - r0 / a) * c;
        const double d = f / fp;
        dE -= d;
        if (std::fabs(d) < 1e-14) break;
    }
    const double c = std::cos(dE), s = std::sin(dE);
    const double r = a + (r0 - a) * c + sigma0 * sqa * s;
    const double F = 1.0 - a / r0 * (1.0 - c);
    const double G = (dt - rev * 2.0 * kPi / n) - std::sqrt(a * a * a / kMuEarth) * (dE - s);
    const double Fd = -std::sqrt(kMuEarth * a) / (r * r0) * s;
    const double Gd = 1.0 - a / r * (1.0 - c);
    for (int q = 0; q < 3; ++q) {
        s1[q] = F * s0[q] + G * s0[3 + q];
        s1[3 + q] = Fd * s0[q] + Gd * s0[3 + q];
    }
    return true;
}

Orbit draw_base(Rng& g, Elements& el, double& radius_m) {
    const double u = g.uniform();
    Orbit kind;
    if (u < 0.75) {
        kind = LEO;
        const double hp = 300.0 + 1700.0 * g.uniform();
        const double e = std::exp(std::log(1e-4) + (std::log(0.02) - std::log(1e-4)) * g.uniform());
        el.a = (kREarth + hp) / (1.0 - e);
        el.e = e;
        static const double clusters[4] = {51.6, 53.0, 70.0, 86.4};
        const int c = static_cast<int>(g.uniform() * 5.0);
        const double base = c < 4 ? clusters[c] : 97.0 + 2.0 * g.uniform();
        el.inc = (base + (g.uniform() - 0.5)) * kDeg;
    } else if (u < 0.81) {
        kind = MEO;
        el.a = 26560.0;
        el.e = 0.01 * g.uniform();
        el.inc = 55.0 * kDeg;
    } else if (u < 0.87) {
        kind = GEO;
        el.a = 42164.0;
        el.e = 1e-3 * g.uniform();
        el.inc = 2.0 * g.uniform() * kDeg;
    } else {
        kind = GTO;
        const double rp = kREarth + 250.0 + 350.0 * g.uniform();
        const double ra = kREarth + 20000.0 + 20000.0 * g.uniform();
        el.a = 0.5 * (rp + ra);
        el.e = (ra - rp) / (ra + rp);
        el.inc = 65.0 * g.uniform() * kDeg;
    }
    el.raan = 2.0 * kPi * g.uniform();
    el.argp = 2.0 * kPi * g.uniform();
    el.M = 2.0 * kPi * g.uniform();
    // Collision radius: log-normal, median 0.5 m, sigma_ln 1.2, clipped to [0.05, 15] m.
    double r = std::exp(std::log(0.5) + 1.2 * g.normal());
    radius_m = r < 0.05 ? 0.05 : (r > 15.0 ? 15.0 : r);
    return kind;
}

}  // namespace
}  // namespace ks


extern "C" {

int ks_generate_population(uint64_t seed, int64_t n_base, int64_t n_total, int n_parents, double frag_age_max_s,
                           double* states, double* size_m, uint8_t* alive) {
    using namespace ks;
    if (n_base < 0 || n_total < n_base || !states || !size_m || !alive || frag_age_max_s < 0.0) return KS_ERR_ARG;
    const int64_t n_frag = n_total - n_base;
    if (n_frag > 0 && (n_parents <= 0 || n_base == 0)) return KS_ERR_ARG;
    std::vector<uint8_t> kind(static_cast<size_t>(n_base));
    for (int64_t i = 0; i < n_base; ++i) {
        Rng g{seed, static_cast<uint64_t>(i)};
        Elements el;
        double radius = 0.0;
        kind[i] = static_cast<uint8_t>(draw_base(g, el, radius));
        elements_to_state(el, states + 6 * i);
        size_m[i] = 2.0 * radius;
        alive[i] = 1;
    }
    if (n_frag == 0) return KS_OK;
    // Parents: distinct LEO objects of the base catalogue.
    std::vector<int64_t> parents;
    std::vector<uint8_t> taken(static_cast<size_t>(n_base), 0);
    Rng pick{seed, 0xfeedf00dull};
    int64_t leo = 0;
    for (int64_t i = 0; i < n_base; ++i) leo += kind[i] == LEO;
    if (leo < n_parents) return KS_ERR_ARG;
    while (static_cast<int>(parents.size()) < n_parents) {
        const int64_t j = static_cast<int64_t>(pick.uniform() * static_cast<double>(n_base));
        if (j >= n_base || taken[j] || kind[j] != LEO) continue;
        taken[j] = 1;
        parents.push_back(j);
    }
    const double alpha1 = -1.6 + 1.0;  // radius power law exponent + 1
    const double rlo = std::pow(0.05, alpha1), rhi = std::pow(0.5, alpha1);
    for (int c = 0; c < n_parents; ++c) {
        const int64_t f0 = n_frag * c / n_parents, f1 = n_frag * (c + 1) / n_parents;
        Rng cg{seed, 0x100000000ull + static_cast<uint64_t>(c)};
        const double age = frag_age_max_s * cg.uniform();
        const double* ps = states + 6 * parents[c];
        // Release point: the parent's epoch state carried back by the cloud's age.
        double rel[6];
        if (!kepler_propagate(ps, -age, rel))
            for (int q = 0; q < 6; ++q) rel[q] = ps[q];
        for (int64_t f = f0; f < f1; ++f) {
            const int64_t i = n_base + f;
            Rng g{seed, 0x200000000ull + static_cast<uint64_t>(f)};
            double s[6];
            for (int attempt = 0;; ++attempt) {
                // Isotropic direction, log-normal magnitude (median 50 m/s, sigma_ln 0.8).
                const double z = 2.0 * g.uniform() - 1.0, phi = 2.0 * kPi * g.uniform();
                const double rho = std::sqrt(1.0 - z * z);
                const double dv = std::exp(std::log(0.05) + 0.8 * g.normal());
                double s0[6] = {rel[0], rel[1], rel[2], rel[3] + dv * rho * std::cos(phi),
                                rel[4] + dv * rho * std::sin(phi), rel[5] + dv * z};
                bool ok = kepler_propagate(s0, age, s);
                if (ok) {
                    const double r = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
                    ok = r > kREarth + 100.0;
                }
                if (ok || attempt >= 16) {
                    if (!ok) for (int q = 0; q < 6; ++q) s[q] = rel[q];
                    break;
                }
            }
            for (int q = 0; q < 6; ++q) states[6 * i + q] = s[q];
            const double r = std::pow(rlo + g.uniform() * (rhi - rlo), 1.0 / alpha1);
            size_m[i] = 2.0 * r;
            alive[i] = 1;
        }
    }
    return KS_OK;
}

}  // extern "C"
