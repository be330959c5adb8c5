// NASA Standard Breakup Model on the device, with counter-based random numbers.
//
// The host SBM (ks_breakup.cpp) reproduces the reference's Mersenne-Twister
// draws one after another, so its fragments equal the reference's bit for bit
// but must be drawn serially on the host. This device form draws every random
// number from a Philox counter that names it - (event, candidate fragment,
// draw) under the run's seed - so every fragment of every event can be drawn
// in parallel, in any order, and the result is still a pure function of the
// seed and the events. Its fragments follow the same laws as the reference's
// (src/core/breakup.cpp:192-338) but are different draws: parity with the
// reference is statistical (tests/test_gpu_sbm_device.py).
//
// The laws, from the published model (Johnson, Krisko, Liou, Anz-Meador, "NASA's
// new breakup model of EVOLVE 4.0", Adv. Space Res. 28(9), 2001), with the
// reference's choices where the model leaves one:
//   number      N(>L) = 0.1 M^0.75 L^-1.71 (collision), M the mass involved;
//               the count above L_c is a Poisson draw of that mean (capped)
//   size        L on [L_c, L_parent] by the inverse of the truncated power law
//   area/mass   chi = log10(A/m): above 11 cm a two-normal mixture, below 8 cm
//               one normal, in between one or the other with a probability
//               linear in L; means, deviations and weights piecewise linear in
//               log10 L (spacecraft fragments)
//   area        A = 0.540424 L^2; mass m = A / 10^chi
//   Delta-v     log10(dv [m/s]) ~ N(0.9 chi + 2.9, 0.4), at most the impact speed,
//               isotropic direction
//   mass        a parent contributes fragments while their masses fit its
//               budget (in candidate order; a candidate that does not fit is
//               skipped, later smaller ones may still fit)
//   escape      fragments with non-negative orbital energy leave and are counted
#pragma once

#include <cstdint>

#include "ks_exact.cuh"

namespace ks {

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplications and a
// key schedule by the Weyl constants, on a 128-bit counter under a 64-bit key.
// ---------------------------------------------------------------------------
constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

__host__ __device__ inline uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c.x;
        const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += kPhiloxW0;
        k.y += kPhiloxW1;
    }
    return c;
}

// Uniform in (0, 1), never 0 or 1 (logarithms stay finite): 32 random bits
// at the centre of their 2^-32 interval.
__host__ __device__ inline double u01(uint32_t x) { return (static_cast<double>(x) + 0.5) * 2.3283064365386963e-10; }

// The named draws of one fragment candidate: 12 uniforms from three Philox
// blocks of the counter (candidate, event, block, stream tag).
enum : int {
    kDrawSide = 0, kDrawSize, kDrawBridge, kDrawMixture, kDrawChiA, kDrawChiB, kDrawDvA, kDrawDvB, kDrawCosT,
    kDrawPhi, kDrawCount
};
constexpr uint32_t kStreamFragment = 0x46524147u;  // counter tag of fragment draws
constexpr uint32_t kStreamEvent = 0x45564e54u;     // counter tag of an event's own draws

struct CandidateDraws {
    double u[12];
};

__host__ __device__ inline CandidateDraws candidate_draws(uint64_t seed, uint32_t event, uint32_t cand) {
    CandidateDraws d;
    const uint2 key = make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    for (uint32_t b = 0; b < 3; ++b) {
        const uint4 r = philox4x32_10(make_uint4(cand, event, b, kStreamFragment), key);
        d.u[4 * b + 0] = u01(r.x);
        d.u[4 * b + 1] = u01(r.y);
        d.u[4 * b + 2] = u01(r.z);
        d.u[4 * b + 3] = u01(r.w);
    }
    return d;
}

// Standard normal from two uniforms (Box-Muller, cosine branch).
__host__ __device__ inline double normal_of(double ua, double ub) {
    return sqrt(-2.0 * log(ua)) * cos(6.283185307179586 * ub);
}

// Sequential uniforms of an event (its Poisson draw): block j of the event's
// own counter.
struct EventStream {
    uint64_t seed;
    uint32_t event;
    uint32_t block = 0;
    int used = 4;
    uint4 cur{};
    __host__ __device__ double next() {
        if (used == 4) {
            const uint2 key = make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
            cur = philox4x32_10(make_uint4(block++, event, 0xFFFFFFFFu, kStreamEvent), key);
            used = 0;
        }
        const uint32_t x = used == 0 ? cur.x : used == 1 ? cur.y : used == 2 ? cur.z : cur.w;
        ++used;
        return u01(x);
    }
};

// Poisson variate of mean `mean`: multiplication of uniforms below 10, the
// transformed rejection with squeeze of Hormann ("The transformed rejection
// method for generating Poisson random variables", Insurance: Mathematics and
// Economics 12, 1993) above. Exact in distribution; bounded loops (a
// rejection loop that has not accepted after 4096 tries returns the mode).
__host__ __device__ inline long long poisson_draw(EventStream& g, double mean) {
    if (!(mean > 0.0)) return 0;
    if (mean < 10.0) {
        const double stop = exp(-mean);
        long long k = 0;
        double p = g.next();
        while (p > stop && k < 1000) {
            ++k;
            p *= g.next();
        }
        return k;
    }
    const double s = sqrt(mean), lg = log(mean);
    const double b = 0.931 + 2.53 * s;
    const double a = -0.059 + 0.02483 * b;
    const double ainv = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int tries = 0; tries < 4096; ++tries) {
        const double u = g.next() - 0.5;
        const double v = g.next();
        const double us = 0.5 - fabs(u);
        const double k = floor((2.0 * a / us + b) * u + mean + 0.43);
        if (us >= 0.07 && v <= vr) return static_cast<long long>(k);
        if (k < 0.0 || (us < 0.013 && v > us)) continue;
        if (log(v * ainv / (a / (us * us) + b)) <= -mean + k * lg - lgamma(k + 1.0)) return static_cast<long long>(k);
    }
    return static_cast<long long>(floor(mean));
}

// Piecewise-linear profile: y0 up to x0, y1 from x1, linear in between.
__host__ __device__ inline double profile(double x, double x0, double y0, double x1, double y1) {
    return x <= x0 ? y0 : x >= x1 ? y1 : y0 + (y1 - y0) * ((x - x0) / (x1 - x0));
}

// chi = log10(A/m) of a fragment of size L = 10^lam (spacecraft breakup).
__host__ __device__ inline double sample_chi(double lam, const CandidateDraws& d) {
    const double L = exp10(lam);
    const double z = normal_of(d.u[kDrawChiA], d.u[kDrawChiB]);
    bool large = L >= 0.11;
    if (!large && L > 0.08) large = d.u[kDrawBridge] < (L - 0.08) / 0.03;
    if (!large) {
        const double mu = profile(lam, -1.75, -0.3, -1.25, -1.0);
        const double sd = lam <= -3.5 ? 0.2 : 0.2 + 0.1333 * (lam + 3.5);
        return mu + sd * z;
    }
    const double alpha = profile(lam, -1.95, 0.0, 0.55, 1.0);
    if (d.u[kDrawMixture] < alpha) {
        const double mu1 = profile(lam, -1.1, -0.6, 0.0, -0.95);
        const double s1 = profile(lam, -1.3, 0.1, -0.3, 0.3);
        return mu1 + s1 * z;
    }
    const double mu2 = profile(lam, -0.7, -1.2, -0.1, -2.0);
    const double s2 = profile(lam, -0.5, 0.5, -0.3, 0.3);
    return mu2 + s2 * z;
}

constexpr double kSbmExponent = 1.71;
constexpr double kSbmAreaCoeff = 0.540424;
constexpr long long kSbmMaxFragments = 200000;  // per event
constexpr double kSbmFallbackMassKg = 100.0;    // objects of unknown mass

// One parent of an event as the fragment draws need it.
struct DevParent {
    double s[6];      // state at the event time
    double size_m;    // characteristic size (upper bound of its fragments)
    double budget;    // mass it may give to fragments (kg)
};

// Size, area-to-mass and mass of candidate `d` (side already chosen): false if
// its parent is not larger than L_c (nothing it sheds is followed).
__host__ __device__ inline bool candidate_mass(const DevParent& p, double lc, const CandidateDraws& d, double& L,
                                               double& chi, double& m) {
    if (!(p.size_m > lc)) return false;
    const double r = pow(p.size_m / lc, -kSbmExponent);
    L = lc * pow(1.0 - d.u[kDrawSize] * (1.0 - r), -1.0 / kSbmExponent);
    chi = sample_chi(log10(L), d);
    m = kSbmAreaCoeff * L * L / exp10(chi);
    return true;
}

// Birth state of candidate `d` (parent state + Delta-v), true if bound to the Earth.
__host__ __device__ inline bool candidate_birth(const DevParent& p, double chi, double vrel_km_s,
                                                const CandidateDraws& d, double mu_earth, double out[6]) {
    double dv_ms = exp10(0.9 * chi + 2.9 + 0.4 * normal_of(d.u[kDrawDvA], d.u[kDrawDvB]));
    dv_ms = fmin(dv_ms, vrel_km_s * 1000.0);
    const double cz = 2.0 * d.u[kDrawCosT] - 1.0;
    const double phi = 6.283185307179586 * d.u[kDrawPhi];
    const double sz = sqrt(fmax(0.0, 1.0 - cz * cz));
    const double dv = dv_ms * 1e-3;
    out[0] = p.s[0];
    out[1] = p.s[1];
    out[2] = p.s[2];
    out[3] = p.s[3] + dv * sz * cos(phi);
    out[4] = p.s[4] + dv * sz * sin(phi);
    out[5] = p.s[5] + dv * cz;
    const double v2 = out[3] * out[3] + out[4] * out[4] + out[5] * out[5];
    const double r = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    return 0.5 * v2 - mu_earth / r < 0.0;
}

}  // namespace ks
