// Split-precision device arithmetic.
//
// Propagation keeps the state, the RK4 combination and the central term
// -mu r / |r|^3 in FP64 (their stability needs it: the central term is ~1e4
// times the J2 term and is integrated over 8 640 steps a day), and evaluates
// the J2 and lunar perturbations in FP32. Contraction into FMA is allowed.
#pragma once

#include "ks_types.h"

namespace ks {

// Per-stage lunar position and indirect term, in FP32.
struct MoonStageF {
    float mx, my, mz;
    float ix, iy, iz;
};

__device__ __forceinline__ MoonStageF to_f32(const MoonStage& m) {
    return MoonStageF{static_cast<float>(m.mx), static_cast<float>(m.my), static_cast<float>(m.mz),
                      static_cast<float>(m.ix), static_cast<float>(m.iy), static_cast<float>(m.iz)};
}

struct SplitConsts {
    double mu_earth;
    float k_j2;      // 1.5 J2 MU_EARTH R_EARTH^2
    float mu_moon;
};

// acceleration(r, rm) of src/core/orbital.cpp:91-105 in split precision.
__device__ __forceinline__ void accel_split(const SplitConsts& sc, double rx, double ry, double rz,
                                            const MoonStageF& m, double& ax, double& ay, double& az) {
    const double r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const double ir = rsqrt(r2);
    const double c = -sc.mu_earth * (ir * ir * ir);
    const float fx = static_cast<float>(rx), fy = static_cast<float>(ry), fz = static_cast<float>(rz);
    const float fir = static_cast<float>(ir);
    // J2: (1.5 J2 mu Re^2 / r^4) * u * (5 uz^2 - {1, 1, 3}), u = r / |r|
    const float ux = fx * fir, uy = fy * fir, uz = fz * fir;
    const float fir2 = fir * fir;
    const float kj = sc.k_j2 * (fir2 * fir2);
    const float z2 = 5.0f * uz * uz;
    float px = kj * ux * (z2 - 1.0f);
    float py = kj * uy * (z2 - 1.0f);
    float pz = kj * uz * (z2 - 3.0f);
    // Moon: direct term minus the indirect term of the geocentric frame.
    const float dx = m.mx - fx, dy = m.my - fy, dz = m.mz - fz;
    const float id = rsqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
    const float sd = sc.mu_moon * (id * id * id);
    px += fmaf(dx, sd, -m.ix);
    py += fmaf(dy, sd, -m.iy);
    pz += fmaf(dz, sd, -m.iz);
    ax = fma(c, rx, static_cast<double>(px));
    ay = fma(c, ry, static_cast<double>(py));
    az = fma(c, rz, static_cast<double>(pz));
}

// rk4 (src/core/orbital.cpp:107-118) with split-precision accelerations.
__device__ __forceinline__ void rk4_split(const SplitConsts& sc, double dt, const MoonStageF& m0,
                                          const MoonStageF& m1, const MoonStageF& m2, double s[6]) {
    const double h2 = 0.5 * dt;
    double k[6], acc[6], y[3];
    k[0] = s[3]; k[1] = s[4]; k[2] = s[5];
    accel_split(sc, s[0], s[1], s[2], m0, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = k[q];
    for (int q = 0; q < 3; ++q) y[q] = fma(k[q], h2, s[q]);
    for (int q = 0; q < 3; ++q) k[q] = fma(k[3 + q], h2, s[3 + q]);
    accel_split(sc, y[0], y[1], y[2], m1, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = fma(k[q], 2.0, acc[q]);
    for (int q = 0; q < 3; ++q) y[q] = fma(k[q], h2, s[q]);
    for (int q = 0; q < 3; ++q) k[q] = fma(k[3 + q], h2, s[3 + q]);
    accel_split(sc, y[0], y[1], y[2], m1, k[3], k[4], k[5]);
    for (int q = 0; q < 6; ++q) acc[q] = fma(k[q], 2.0, acc[q]);
    for (int q = 0; q < 3; ++q) y[q] = fma(k[q], dt, s[q]);
    for (int q = 0; q < 3; ++q) k[q] = fma(k[3 + q], dt, s[3 + q]);
    accel_split(sc, y[0], y[1], y[2], m2, k[3], k[4], k[5]);
    const double h6 = dt / 6.0;
    for (int q = 0; q < 6; ++q) s[q] = fma(acc[q] + k[q], h6, s[q]);
}

// Conservative FP32 distance gate on recentred coordinates: 1 if the pair may
// pass filter_pair's distance gate. Inputs carry absolute errors of at most
// e_r (positions) and e_v (velocities), f32_pos_err and f32_vel_err: the true
// relative motion stays within e = e_r + e_v dt of the computed one over the
// step, so the gate widens by e, and the 1e-5 P term covers the FP32 rounding
// of P - m^2 (P = |dr|^2 |dv|^2).
constexpr float kF32PosErrKm = 5e-4f;   // floor of e_r
constexpr float kF32VelErrKmS = 5e-6f;  // floor of e_v

// e_r for records of a grid with cell edge `cell` km. A row record is its
// position relative to its cell's corner, in [0, cell], rounded to FP32
// (<= 2^-24 cell per component); a column record from a neighbour cell is also
// moved by an FP32 copy of the edge (<= 2^-24 cell) and rounded again within
// 2 cell (<= 2^-23 cell). Per component of dr: <= 2^-24 (1 + 1 + 2 + 1) cell
// < 3e-7 cell; over the three components < 5.2e-7 cell.
__host__ __device__ inline double f32_pos_err(double cell) { return fmax(static_cast<double>(kF32PosErrKm), 6e-7 * cell); }

// e_v when no record is faster than vmax km/s: velocities rounded to FP32
// (<= 2^-24 |v| per component each), so dv errs by < 1.2e-7 vmax per
// component, < 2.1e-7 vmax over the three.
__host__ __device__ inline double f32_vel_err(double vmax) { return fmax(static_cast<double>(kF32VelErrKmS), 2.2e-7 * vmax); }

__device__ __forceinline__ unsigned gate_open_f32(float4 cp, float4 cv, float4 rp, float4 rv, float gate2) {
    const float rx = cp.x - rp.x, ry = cp.y - rp.y, rz = cp.z - rp.z;
    const float vx = cv.x - rv.x, vy = cv.y - rv.y, vz = cv.z - rv.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    const float dv2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
    const float m = fminf(fmaf(rx, vx, fmaf(ry, vy, rz * vz)), 0.0f);
    const float P = r2 * dv2;
    return fmaf(-m, m, P) <= fmaf(dv2, gate2, 1e-5f * P) ? 1u : 0u;
}

// gate_open_f32 for two rows at once with Blackwell's packed FP32 arithmetic
// (FFMA2 / FMUL2: two lanes of an f32x2 per instruction, each rounded exactly
// as the scalar instruction): the same operations in the same order as
// gate_open_f32, so each of the two decisions equals the scalar gate's bit
// for bit, with about half the instructions. rows: the two rows' six
// components interleaved, {px0, px1}, {py0, py1}, {pz0, pz1}, {vx0, vx1},
// {vy0, vy1}, {vz0, vz1}. Bit 0: first row, bit 1: second.
__device__ __forceinline__ unsigned gate_open_f32x2(const float4 cp, const float4 cv, const float2* rows,
                                                    const float2 gate2) {
    const float2 m1 = make_float2(-1.0f, -1.0f);
    // c - r, rounded once: fma(r, -1, c).
    const float2 rx = __ffma2_rn(rows[0], m1, make_float2(cp.x, cp.x));
    const float2 ry = __ffma2_rn(rows[1], m1, make_float2(cp.y, cp.y));
    const float2 rz = __ffma2_rn(rows[2], m1, make_float2(cp.z, cp.z));
    const float2 vx = __ffma2_rn(rows[3], m1, make_float2(cv.x, cv.x));
    const float2 vy = __ffma2_rn(rows[4], m1, make_float2(cv.y, cv.y));
    const float2 vz = __ffma2_rn(rows[5], m1, make_float2(cv.z, cv.z));
    const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
    const float2 dv2 = __ffma2_rn(vx, vx, __ffma2_rn(vy, vy, __fmul2_rn(vz, vz)));
    const float2 rv = __ffma2_rn(rx, vx, __ffma2_rn(ry, vy, __fmul2_rn(rz, vz)));
    const float2 m = make_float2(fminf(rv.x, 0.0f), fminf(rv.y, 0.0f));
    const float2 P = __fmul2_rn(r2, dv2);
    const float2 lhs = __ffma2_rn(make_float2(-m.x, -m.y), m, P);
    const float2 rhs = __ffma2_rn(dv2, gate2, __fmul2_rn(make_float2(1e-5f, 1e-5f), P));
    return (lhs.x <= rhs.x ? 1u : 0u) | (lhs.y <= rhs.y ? 2u : 0u);
}

}  // namespace ks
