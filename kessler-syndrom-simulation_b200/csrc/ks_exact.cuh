// Exact FP64 device arithmetic for the plain (bit-identical) path.
//
// Every operation is an explicit round-to-nearest intrinsic, so the compiler
// can neither contract a multiply and an add into an FMA nor reorder anything.
// Each function keeps the operation order of the reference expression it
// restates; the reference builds its CPU path without FMA contraction and its
// CUDA path with --fmad=false for the same reason (src/core/collision_filter.hpp:3-9,
// CMakeLists.txt:76-78).
#pragma once

#include <cstdint>

#include "ks_types.h"

namespace ks {

__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }

// dot(a, a) = (x*x + y*y) + z*z (src/core/orbital.hpp:45)
__device__ __forceinline__ double xdot3(double x, double y, double z) {
    return xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z));
}

// acceleration(r, rm) (src/core/orbital.cpp:91-105). The moon-only factor
// MU_MOON / |rm|^3 is identical for every object and arrives precomputed.
__device__ __forceinline__ void accel_exact(const ForceConsts& fc, double rx, double ry, double rz,
                                            const MoonStage& m, double& ax, double& ay, double& az) {
    const double r2 = xdot3(rx, ry, rz);
    const double rn = xsqrt(r2);
    const double c = xdiv(fc.neg_mu_earth, xmul(r2, rn));
    ax = xmul(rx, c);
    ay = xmul(ry, c);
    az = xmul(rz, c);
    const double k = xdiv(fc.k_j2, xmul(xmul(r2, r2), rn));
    const double z2 = xdiv(xmul(xmul(5.0, rz), rz), r2);
    const double zm1 = xsub(z2, 1.0), zm3 = xsub(z2, 3.0);
    ax = xadd(ax, xmul(xmul(k, rx), zm1));
    ay = xadd(ay, xmul(xmul(k, ry), zm1));
    az = xadd(az, xmul(xmul(k, rz), zm3));
    const double dx = xsub(m.mx, rx), dy = xsub(m.my, ry), dz = xsub(m.mz, rz);
    const double dn = xsqrt(xdot3(dx, dy, dz));
    const double sd = xdiv(fc.mu_moon, xmul(xmul(dn, dn), dn));
    ax = xsub(xadd(ax, xmul(dx, sd)), m.ix);
    ay = xsub(xadd(ay, xmul(dy, sd)), m.iy);
    az = xsub(xadd(az, xmul(dz, sd)), m.iz);
}

// rk4(s, dt, rm0, rm1, rm2) (src/core/orbital.cpp:107-118). s is updated in place.
// The stage derivatives are folded into `acc` as they come, which keeps the
// reference's summation order ((k1 + 2 k2) + 2 k3) + k4 with fewer live registers.
__device__ __forceinline__ void rk4_exact(const ForceConsts& fc, double dt, const MoonStage& m0,
                                          const MoonStage& m1, const MoonStage& m2, double s[6]) {
    const double h2 = xdiv(dt, 2.0);
    double k[6], acc[6], y[3];
    k[0] = s[3]; k[1] = s[4]; k[2] = s[5];
    accel_exact(fc, s[0], s[1], s[2], m0, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = k[q];

    for (int q = 0; q < 3; ++q) y[q] = xadd(s[q], xmul(k[q], h2));
    for (int q = 0; q < 3; ++q) k[q] = xadd(s[3 + q], xmul(k[3 + q], h2));
    accel_exact(fc, y[0], y[1], y[2], m1, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = xadd(acc[q], xmul(k[q], 2.0));

    for (int q = 0; q < 3; ++q) y[q] = xadd(s[q], xmul(k[q], h2));
    for (int q = 0; q < 3; ++q) k[q] = xadd(s[3 + q], xmul(k[3 + q], h2));
    accel_exact(fc, y[0], y[1], y[2], m1, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = xadd(acc[q], xmul(k[q], 2.0));

    for (int q = 0; q < 3; ++q) y[q] = xadd(s[q], xmul(k[q], dt));
    for (int q = 0; q < 3; ++q) k[q] = xadd(s[3 + q], xmul(k[3 + q], dt));
    accel_exact(fc, y[0], y[1], y[2], m2, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = xadd(acc[q], k[q]);

    const double h6 = xdiv(dt, 6.0);
    for (int q = 0; q < 6; ++q) s[q] = xadd(s[q], xmul(acc[q], h6));
}

enum : int { FILTER_REJECT = 0, FILTER_REFINE = 1, FILTER_CO_ORBITING = 2 };

// filter_pair (src/core/collision_filter.hpp:37-66). dr, dv = state(j) - state(i)
// at the start of the step. The decision is unchanged when both dr and dv are
// negated (every product pairs two negated factors and rounding to nearest is
// sign-symmetric), so callers may subtract in either order.
__device__ __forceinline__ int filter_pair_exact(double rx, double ry, double rz, double vx, double vy,
                                                 double vz, double dt, double threshold_km, double vmin2) {
    const double dv2 = xdot3(vx, vy, vz);
    const double rv = xadd(xadd(xmul(rx, vx), xmul(ry, vy)), xmul(rz, vz));
    double ts = dv2 > 0 ? xdiv(-rv, dv2) : 0.0;
    if (ts < 0.0) ts = 0.0;
    if (ts > dt) ts = dt;
    const double px = xadd(rx, xmul(vx, ts)), py = xadd(ry, xmul(vy, ts)), pz = xadd(rz, xmul(vz, ts));
    const double gate =
        xadd(xadd(threshold_km, xmul(xmul(xmul(xmul(kGravityGradient, xsqrt(dv2)), dt), dt), dt)), 1e-3);
    if (xsqrt(xdot3(px, py, pz)) > gate) return FILTER_REJECT;
    if (dv2 < vmin2) return FILTER_CO_ORBITING;
    if (rv >= 0.0 && dv2 > xmul(kGravityGradient, xdot3(rx, ry, rz))) return FILTER_REJECT;
    return FILTER_REFINE;
}

// Cheap conservative test in front of filter_pair_exact: returns true only if
// filter_pair_exact would certainly return FILTER_REJECT because the closest
// approach of the linear relative motion stays beyond the distance gate.
//   gate_hi2 >= (threshold + G * vrel_max * dt^3 + 1e-3)^2, vrel_max >= |dv|.
// No division and no square root; margins cover the rounding of both sides.
__device__ __forceinline__ bool certainly_far(double r2, double dv2, double rv, double gate_hi2) {
    if (rv >= 0.0) return r2 > gate_hi2;             // closest point is the start: p = dr
    const double cross2 = r2 * dv2 - rv * rv;        // |dr x dv|^2 = min distance^2 * |dv|^2
    return cross2 > gate_hi2 * dv2 + 1e-12 * (r2 * dv2);
}

// Cubic Hermite of the relative motion over s in [0, 1]
// (src/core/collision.cpp:77-90); m = relative velocity * dt.
struct Hermite {
    double p0[3], m0[3], p1[3], m1[3];

    __device__ __forceinline__ void pos(double s, double out[3]) const {
        const double s2 = xmul(s, s), s3 = xmul(s2, s);
        const double c0 = xadd(xsub(xmul(2.0, s3), xmul(3.0, s2)), 1.0);
        const double c1 = xadd(xsub(s3, xmul(2.0, s2)), s);
        const double c2 = xadd(xmul(-2.0, s3), xmul(3.0, s2));
        const double c3 = xsub(s3, s2);
        for (int q = 0; q < 3; ++q)
            out[q] = xadd(xadd(xadd(xmul(p0[q], c0), xmul(m0[q], c1)), xmul(p1[q], c2)), xmul(m1[q], c3));
    }
    __device__ __forceinline__ void vel(double s, double out[3]) const {
        const double s2 = xmul(s, s);
        const double c0 = xsub(xmul(6.0, s2), xmul(6.0, s));
        const double c1 = xadd(xsub(xmul(3.0, s2), xmul(4.0, s)), 1.0);
        const double c2 = xadd(xmul(-6.0, s2), xmul(6.0, s));
        const double c3 = xsub(xmul(3.0, s2), xmul(2.0, s));
        for (int q = 0; q < 3; ++q)
            out[q] = xadd(xadd(xadd(xmul(p0[q], c0), xmul(m0[q], c1)), xmul(p1[q], c2)), xmul(m1[q], c3));
    }
    __device__ __forceinline__ double f(double s) const {
        double p[3];
        pos(s, p);
        return xdot3(p[0], p[1], p[2]);
    }
};

// closest_approach: 60 golden-section iterations on |p(s)|^2 (src/core/collision.cpp:94-105).
__device__ __forceinline__ double closest_approach_exact(const Hermite& h) {
    const double g = 0.6180339887498949;
    double a = 0.0, b = 1.0;
    double c = xsub(b, xmul(g, xsub(b, a))), d = xadd(a, xmul(g, xsub(b, a)));
    double fc = h.f(c), fd = h.f(d);
    // Branch-free form of the reference's loop (the same operations on every
    // lane, one evaluation of f per iteration): keep [a, d] with a new point
    // b - g (b - a) when f(c) < f(d), else [c, b] with a new point a + g (b - a).
    for (int it = 0; it < 60; ++it) {
        const bool left = fc < fd;
        const double na = left ? a : c, nb = left ? d : b;
        const double step = xmul(g, xsub(nb, na));
        const double x = left ? xsub(nb, step) : xadd(na, step);
        const double fx = h.f(x);
        const double nc = left ? x : d, nd = left ? c : x;
        const double nfc = left ? fx : fd, nfd = left ? fc : fx;
        a = na; b = nb; c = nc; d = nd; fc = nfc; fd = nfd;
    }
    return xmul(0.5, xadd(a, b));
}

}  // namespace ks
