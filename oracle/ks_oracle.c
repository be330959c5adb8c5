/*
 * ORACLE - test infrastructure only.
 *
 * A plain-C restatement of the reference's per-step hot path, used to check
 * the B200 engine. Only tests/, the smoke check and bench.py's CPU-baseline
 * leg may load it, and only as the checker: the product never calls it.
 *
 * Parity of this restatement is pinned two ways (tests/test_oracle_pin.py):
 *   - bit-for-bit against the reference itself, compiled from its own sources
 *     into oracle/_ref/libksref.so by oracle/Makefile, on seeded synthetic
 *     populations (states, conjunction lists and per-step counters);
 *   - against the reference README's published run on its shipped catalogue
 *     (tests/golden/ref_catalog_1h.json, produced by the reference build).
 *
 * Floating point: every expression keeps the reference's operation order and
 * is compiled without FMA contraction (-ffp-contract=off, no -march), the same
 * contract the reference states in src/core/collision_filter.hpp:3-9.
 *
 * All citations are paths inside the reference repository.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ks_records.h"

/* src/core/orbital.hpp:19-26 */
#define KSO_PI 3.14159265358979323846
#define KSO_DEG (KSO_PI / 180.0)
#define KSO_MU_EARTH 398600.4418
#define KSO_MU_MOON 4902.800066
#define KSO_R_EARTH 6378.137
#define KSO_J2 1.08262668e-3
/* src/core/collision_filter.hpp:26 */
#define KSO_GRAVITY_GRADIENT 2e-6
/* src/core/collision_filter.hpp:82-83 */
#define KSO_DR_ERR_KM 5e-4f
#define KSO_DV_ERR_KM_S 5e-6f
/* src/core/collision_filter.hpp:118-119 */
#define KSO_KEY_OFFSET (1LL << 20)

enum { KSO_REJECT = 0, KSO_REFINE = 1, KSO_CO_ORBITING = 2 };

static double kso_dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double kso_norm3(const double* a) { return sqrt(kso_dot3(a, a)); }

static double kso_wrap360(double d) { return fmod(fmod(d, 360.0) + 360.0, 360.0); }

/* Truncated lunar series of Meeus, Astronomical Algorithms ch. 47, with the
 * term selection and evaluation order of src/core/orbital.cpp:53-85. */
void kso_moon_position(double jd, double out[3]) {
    double T = (jd - 2451545.0) / 36525.0;
    double Lp = kso_wrap360(218.3164477 + 481267.88123421 * T);
    double D = kso_wrap360(297.8501921 + 445267.1114034 * T);
    double M = kso_wrap360(357.5291092 + 35999.0502909 * T);
    double Mp = kso_wrap360(134.9633964 + 477198.8675055 * T);
    double F = kso_wrap360(93.2720950 + 483202.0175233 * T);
    D *= KSO_DEG; M *= KSO_DEG; Mp *= KSO_DEG; F *= KSO_DEG;

    double lon = Lp + 6.288774 * sin(Mp) + 1.274027 * sin(2 * D - Mp)
               + 0.658314 * sin(2 * D) + 0.213618 * sin(2 * Mp)
               - 0.185116 * sin(M) - 0.114332 * sin(2 * F)
               + 0.058793 * sin(2 * D - 2 * Mp) + 0.057066 * sin(2 * D - M - Mp)
               + 0.053322 * sin(2 * D + Mp) + 0.045758 * sin(2 * D - M);
    double lat = 5.128122 * sin(F) + 0.280602 * sin(Mp + F)
               + 0.277693 * sin(Mp - F) + 0.173237 * sin(2 * D - F)
               + 0.055413 * sin(2 * D - Mp + F) + 0.046271 * sin(2 * D - Mp - F);
    double dist = 385000.56 - 20905.355 * cos(Mp) - 3699.111 * cos(2 * D - Mp)
                - 2955.968 * cos(2 * D) - 569.925 * cos(2 * Mp)
                + 48.888 * cos(M) - 3.149 * cos(2 * F)
                + 246.158 * cos(2 * D - 2 * Mp) - 152.138 * cos(2 * D - M - Mp)
                - 170.733 * cos(2 * D + Mp) - 204.586 * cos(2 * D - M);

    double l = lon * KSO_DEG, b = lat * KSO_DEG;
    double eps = (23.439291 - 0.0130042 * T) * KSO_DEG;
    double xe = dist * cos(b) * cos(l);
    double ye = dist * cos(b) * sin(l);
    double ze = dist * sin(b);
    out[0] = xe;
    out[1] = ye * cos(eps) - ze * sin(eps);
    out[2] = ye * sin(eps) + ze * cos(eps);
}

/* src/core/orbital.cpp:91-105: point mass + J2 + lunar direct minus indirect. */
void kso_acceleration(const double r[3], const double rm[3], double a[3]) {
    double r2 = kso_dot3(r, r), rn = sqrt(r2);
    double c = -KSO_MU_EARTH / (r2 * rn);
    a[0] = r[0] * c; a[1] = r[1] * c; a[2] = r[2] * c;

    double k = 1.5 * KSO_J2 * KSO_MU_EARTH * KSO_R_EARTH * KSO_R_EARTH / (r2 * r2 * rn);
    double z2 = 5.0 * r[2] * r[2] / r2;
    a[0] = a[0] + k * r[0] * (z2 - 1.0);
    a[1] = a[1] + k * r[1] * (z2 - 1.0);
    a[2] = a[2] + k * r[2] * (z2 - 3.0);

    double d[3] = {rm[0] - r[0], rm[1] - r[1], rm[2] - r[2]};
    double dn = kso_norm3(d), mn = kso_norm3(rm);
    double sd = KSO_MU_MOON / (dn * dn * dn);
    double sm = KSO_MU_MOON / (mn * mn * mn);
    for (int q = 0; q < 3; ++q) a[q] = a[q] + d[q] * sd - rm[q] * sm;
}

/* src/core/orbital.cpp:107-118: classic RK4, moon at start, middle (twice), end. */
void kso_rk4(const double s[6], double dt, const double m0[3], const double m1[3],
             const double m2[3], double out[6]) {
    double k1[6], k2[6], k3[6], k4[6], y[6];
    const double h2 = dt / 2;
    k1[0] = s[3]; k1[1] = s[4]; k1[2] = s[5];
    kso_acceleration(s, m0, k1 + 3);
    for (int q = 0; q < 6; ++q) y[q] = s[q] + k1[q] * h2;
    k2[0] = y[3]; k2[1] = y[4]; k2[2] = y[5];
    kso_acceleration(y, m1, k2 + 3);
    for (int q = 0; q < 6; ++q) y[q] = s[q] + k2[q] * h2;
    k3[0] = y[3]; k3[1] = y[4]; k3[2] = y[5];
    kso_acceleration(y, m1, k3 + 3);
    for (int q = 0; q < 6; ++q) y[q] = s[q] + k3[q] * dt;
    k4[0] = y[3]; k4[1] = y[4]; k4[2] = y[5];
    kso_acceleration(y, m2, k4 + 3);
    const double h6 = dt / 6;
    for (int q = 0; q < 6; ++q) out[q] = s[q] + (k1[q] + k2[q] * 2 + k3[q] * 2 + k4[q]) * h6;
}

/* src/core/collision_filter.hpp:37-66 */
int kso_filter_pair(double rx, double ry, double rz, double vx, double vy, double vz,
                    double dt, double threshold_km, double vmin2) {
    const double dv2 = vx * vx + vy * vy + vz * vz;
    const double rv = rx * vx + ry * vy + rz * vz;
    double ts = dv2 > 0 ? -rv / dv2 : 0.0;
    if (ts < 0.0) ts = 0.0;
    if (ts > dt) ts = dt;
    const double px = rx + vx * ts, py = ry + vy * ts, pz = rz + vz * ts;
    const double gate = threshold_km + KSO_GRAVITY_GRADIENT * sqrt(dv2) * dt * dt * dt + 1e-3;
    if (sqrt(px * px + py * py + pz * pz) > gate) return KSO_REJECT;
    if (dv2 < vmin2) return KSO_CO_ORBITING;
    if (rv >= 0.0 && dv2 > KSO_GRAVITY_GRADIENT * (rx * rx + ry * ry + rz * rz)) return KSO_REJECT;
    return KSO_REFINE;
}

/* src/core/collision_filter.hpp:85-114 (single-precision conservative gate). */
int kso_prefilter_keep(float rx, float ry, float rz, float vx, float vy, float vz,
                       float dt, float threshold_km, float vmin2) {
    const float dv2 = vx * vx + vy * vy + vz * vz;
    const float rv = rx * vx + ry * vy + rz * vz;
    const float r2 = rx * rx + ry * ry + rz * rz;
    const float dvn = sqrtf(dv2), rn = sqrtf(r2);
    float ts = dv2 > 0.0f ? -rv / dv2 : 0.0f;
    if (ts < 0.0f) ts = 0.0f;
    if (ts > dt) ts = dt;
    const float px = rx + vx * ts, py = ry + vy * ts, pz = rz + vz * ts;
    const float d = sqrtf(px * px + py * py + pz * pz);
    const float gate = threshold_km + (float)KSO_GRAVITY_GRADIENT * dvn * dt * dt * dt + 1e-3f;
    const float margin = 1e-5f * (rn + dvn * dt) + KSO_DR_ERR_KM + KSO_DV_ERR_KM_S * dt;
    if (d > gate + margin) return 0;
    const float rv_tol = 1e-5f * rn * dvn + KSO_DR_ERR_KM * dvn + KSO_DV_ERR_KM_S * rn;
    if (dv2 > 1.1f * vmin2 && rv > rv_tol && dv2 > 1.01f * (float)KSO_GRAVITY_GRADIENT * r2) return 0;
    return 1;
}

/* src/core/collision_filter.hpp:121-125 */
static unsigned long long kso_cell_key(long long ix, long long iy, long long iz) {
    return ((unsigned long long)(ix + KSO_KEY_OFFSET) << 42) |
           ((unsigned long long)(iy + KSO_KEY_OFFSET) << 21) |
           (unsigned long long)(iz + KSO_KEY_OFFSET);
}

/* src/core/collision_filter.hpp:127-132 */
static void kso_cell_coords(unsigned long long key, long long* ix, long long* iy, long long* iz) {
    const unsigned long long mask = (1ULL << 21) - 1;
    *ix = (long long)((key >> 42) & mask) - KSO_KEY_OFFSET;
    *iy = (long long)((key >> 21) & mask) - KSO_KEY_OFFSET;
    *iz = (long long)(key & mask) - KSO_KEY_OFFSET;
}

/* src/core/collision_filter.hpp:137-140 */
static const int KSO_FORWARD[13][3] = {{1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0},
                                       {1, 0, 1},   {1, 1, -1}, {1, 1, 0},  {1, 1, 1},  {0, 1, -1},
                                       {0, 1, 0},   {0, 1, 1},  {0, 0, 1}};

/* src/core/collision.cpp:339-356: cell edge from the largest start-of-step
 * speed among objects alive after the step. */
double kso_cell_size(long n, const double* before, const uint8_t* alive_after, double dt,
                     double threshold_km) {
    double vmax = 0.0;
    for (long i = 0; i < n; ++i) {
        if (!alive_after[i]) continue;
        double v = kso_norm3(before + 6 * i + 3);
        if (v > vmax) vmax = v;
    }
    const double vrel_max = 2.0 * vmax;
    double c = vrel_max * dt + threshold_km + KSO_GRAVITY_GRADIENT * vrel_max * dt * dt * dt;
    return c > 1.0 ? c : 1.0;
}

/* src/core/collision.cpp:77-90: cubic Hermite of the relative motion, s in [0, 1]. */
typedef struct { double p0[3], m0[3], p1[3], m1[3]; } kso_hermite;

static void kso_hermite_pos(const kso_hermite* h, double s, double out[3]) {
    double s2 = s * s, s3 = s2 * s;
    double c0 = 2 * s3 - 3 * s2 + 1, c1 = s3 - 2 * s2 + s, c2 = -2 * s3 + 3 * s2, c3 = s3 - s2;
    for (int q = 0; q < 3; ++q) out[q] = h->p0[q] * c0 + h->m0[q] * c1 + h->p1[q] * c2 + h->m1[q] * c3;
}

static void kso_hermite_vel(const kso_hermite* h, double s, double out[3]) {
    double s2 = s * s;
    double c0 = 6 * s2 - 6 * s, c1 = 3 * s2 - 4 * s + 1, c2 = -6 * s2 + 6 * s, c3 = 3 * s2 - 2 * s;
    for (int q = 0; q < 3; ++q) out[q] = h->p0[q] * c0 + h->m0[q] * c1 + h->p1[q] * c2 + h->m1[q] * c3;
}

static double kso_hermite_f(const kso_hermite* h, double s) {
    double p[3];
    kso_hermite_pos(h, s, p);
    return kso_dot3(p, p);
}

/* src/core/collision.cpp:94-105: 60 golden-section iterations on |p(s)|^2. */
static double kso_closest_approach(const kso_hermite* h) {
    const double g = 0.6180339887498949;
    double a = 0.0, b = 1.0;
    double c = b - g * (b - a), d = a + g * (b - a);
    double fc = kso_hermite_f(h, c), fd = kso_hermite_f(h, d);
    for (int it = 0; it < 60; ++it) {
        if (fc < fd) { b = d; d = c; fd = fc; c = b - g * (b - a); fc = kso_hermite_f(h, c); }
        else         { a = c; c = d; fc = fd; d = a + g * (b - a); fd = kso_hermite_f(h, d); }
    }
    return 0.5 * (a + b);
}

/* src/core/collision.cpp:283-287 */
static double kso_collision_radius_km(double size_m, double scale) { return 0.5 * size_m * 1e-3 * scale; }

/* src/core/collision.cpp:109-132 */
static int kso_refine_pair(const double* before, const double* after, const double* size_m, int i, int j,
                           double t0, double dt, double threshold_km, double radius_scale,
                           ks_conjunction* out) {
    const double *bi = before + 6 * (long)i, *bj = before + 6 * (long)j;
    const double *ai = after + 6 * (long)i, *aj = after + 6 * (long)j;
    kso_hermite h;
    for (int q = 0; q < 3; ++q) {
        h.p0[q] = bj[q] - bi[q];
        h.m0[q] = (bj[3 + q] - bi[3 + q]) * dt;
        h.p1[q] = aj[q] - ai[q];
        h.m1[q] = (aj[3 + q] - ai[3 + q]) * dt;
    }
    double s = kso_closest_approach(&h);
    if (s <= 1e-9 || s >= 1.0 - 1e-9) return 0;
    double p[3], v[3];
    kso_hermite_pos(&h, s, p);
    double miss = kso_norm3(p);
    if (miss > threshold_km) return 0;
    kso_hermite_vel(&h, s, v);
    out->i = i;
    out->j = j;
    out->t = t0 + s * dt;
    out->miss_km = miss;
    out->v_rel_km_s = kso_norm3(v) / dt;
    out->collision = miss < kso_collision_radius_km(size_m[i], radius_scale) +
                                kso_collision_radius_km(size_m[j], radius_scale);
    out->realisation = 0;
    return 1;
}

typedef struct { unsigned long long key; int idx; } kso_entry;
typedef struct { unsigned long long key; long begin, end; } kso_cell;

static int kso_entry_cmp(const void* a, const void* b) {
    const kso_entry *x = (const kso_entry*)a, *y = (const kso_entry*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* src/core/collision.cpp:743-747: order by (t, i, j). */
static int kso_conj_cmp(const void* a, const void* b) {
    const ks_conjunction *x = (const ks_conjunction*)a, *y = (const ks_conjunction*)b;
    if (x->t != y->t) return x->t < y->t ? -1 : 1;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    return (x->j > y->j) - (x->j < y->j);
}

static long kso_find_cell(const kso_cell* cells, long ncells, unsigned long long key) {
    long lo = 0, hi = ncells;
    while (lo < hi) {
        long mid = (lo + hi) / 2;
        if (cells[mid].key < key) lo = mid + 1; else hi = mid;
    }
    return (lo < ncells && cells[lo].key == key) ? lo : -1;
}

typedef struct {
    ks_conjunction* buf;
    long count, cap;
    long long candidates, refined, co_orbiting;
} kso_sink;

static void kso_visit(kso_sink* sk, int a, int b, const double* before, const double* after,
                      const double* size_m, double t0, double dt, double thr, double rscale, double vmin2) {
    sk->candidates++;
    const int i = a < b ? a : b, j = a < b ? b : a;
    const double *p = before + 6 * (long)i, *q = before + 6 * (long)j;
    int r = kso_filter_pair(q[0] - p[0], q[1] - p[1], q[2] - p[2], q[3] - p[3], q[4] - p[4], q[5] - p[5],
                            dt, thr, vmin2);
    if (r == KSO_CO_ORBITING) { sk->co_orbiting++; return; }
    if (r != KSO_REFINE) return;
    sk->refined++;
    ks_conjunction c;
    if (kso_refine_pair(before, after, size_m, i, j, t0, dt, thr, rscale, &c)) {
        if (sk->count >= sk->cap) {
            long ncap = sk->cap ? 2 * sk->cap : 64;
            ks_conjunction* nb = (ks_conjunction*)realloc(sk->buf, sizeof(ks_conjunction) * (size_t)ncap);
            if (!nb) return;
            sk->buf = nb;
            sk->cap = ncap;
        }
        sk->buf[sk->count++] = c;
    }
}

/* One screening pass (src/core/collision.cpp:360-563 then :739-748): grid of
 * start-of-step positions of the objects alive after the step, pairs inside
 * each cell and with its 13 forward neighbours, linear filter, Hermite
 * refinement, result sorted by (t, i, j). Grouping here is a plain sort;
 * the reference's hash/radix grouping yields the same cell set. */
long kso_screen(long n, const double* before, const double* after, const uint8_t* alive_after,
                const double* size_m, double t0, double dt, double threshold_km, double radius_scale,
                double min_encounter_speed_km_s, ks_conjunction* out, long cap, ks_step_stats* stats) {
    const double cell = kso_cell_size(n, before, alive_after, dt, threshold_km);
    kso_entry* e = (kso_entry*)malloc(sizeof(kso_entry) * (size_t)(n > 0 ? n : 1));
    long m = 0;
    for (long i = 0; i < n; ++i) {
        if (!alive_after[i]) continue;
        const double* r = before + 6 * i;
        e[m].key = kso_cell_key((long long)floor(r[0] / cell), (long long)floor(r[1] / cell),
                                (long long)floor(r[2] / cell));
        e[m].idx = (int)i;
        ++m;
    }
    qsort(e, (size_t)m, sizeof(kso_entry), kso_entry_cmp);
    kso_cell* cells = (kso_cell*)malloc(sizeof(kso_cell) * (size_t)(m > 0 ? m : 1));
    long nc = 0;
    for (long k = 0; k < m; ++k) {
        if (k == 0 || e[k].key != e[k - 1].key) {
            cells[nc].key = e[k].key;
            cells[nc].begin = k;
            ++nc;
        }
    }
    for (long c = 0; c < nc; ++c) cells[c].end = c + 1 < nc ? cells[c + 1].begin : m;

    const double vmin2 = min_encounter_speed_km_s * min_encounter_speed_km_s;
    kso_sink sk = {0};
    int max_cell = 0;
    for (long c = 0; c < nc; ++c) {
        const kso_cell* cc = &cells[c];
        int size = (int)(cc->end - cc->begin);
        if (size > max_cell) max_cell = size;
        for (long p = cc->begin; p < cc->end; ++p)
            for (long q = p + 1; q < cc->end; ++q)
                kso_visit(&sk, e[p].idx, e[q].idx, before, after, size_m, t0, dt, threshold_km,
                          radius_scale, vmin2);
        long long x, y, z;
        kso_cell_coords(cc->key, &x, &y, &z);
        for (int o = 0; o < 13; ++o) {
            long other = kso_find_cell(cells, nc, kso_cell_key(x + KSO_FORWARD[o][0], y + KSO_FORWARD[o][1],
                                                               z + KSO_FORWARD[o][2]));
            if (other < 0) continue;
            for (long p = cc->begin; p < cc->end; ++p)
                for (long q = cells[other].begin; q < cells[other].end; ++q)
                    kso_visit(&sk, e[p].idx, e[q].idx, before, after, size_m, t0, dt, threshold_km,
                              radius_scale, vmin2);
        }
    }
    qsort(sk.buf, (size_t)sk.count, sizeof(ks_conjunction), kso_conj_cmp);
    for (long k = 0; k < sk.count && k < cap; ++k) out[k] = sk.buf[k];
    if (stats) {
        stats->candidate_pairs = sk.candidates;
        stats->refined_pairs = sk.refined;
        stats->co_orbiting = sk.co_orbiting;
        stats->conjunctions = sk.count;
        stats->cell_km = cell;
        stats->max_cell_objects = max_cell;
        stats->alive = (int32_t)m;
    }
    long found = sk.count;
    free(sk.buf);
    free(cells);
    free(e);
    return found;
}

/* src/core/orbital.cpp:286-300: one step of every alive object; objects whose
 * new radius is below R_EARTH die. moon[0..2] = positions at t, t+dt/2, t+dt. */
void kso_step(long n, double* states, uint8_t* alive, double dt, const double moon[9]) {
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        if (!alive[i]) continue;
        double out[6];
        kso_rk4(states + 6 * i, dt, moon, moon + 3, moon + 6, out);
        memcpy(states + 6 * i, out, sizeof(out));
        if (kso_norm3(out) < KSO_R_EARTH) alive[i] = 0;
    }
}

/* Moon at the start, middle and end of the step starting at t
 * (src/core/orbital.cpp:287-289). */
void kso_step_moon(double epoch_jd, double t, double dt, double moon[9]) {
    kso_moon_position(epoch_jd + t / 86400.0, moon);
    kso_moon_position(epoch_jd + (t + dt / 2) / 86400.0, moon + 3);
    kso_moon_position(epoch_jd + (t + dt) / 86400.0, moon + 6);
}

/* The CLI step loop (src/main.cpp:346-407), screening optional, no breakup.
 * Same argument meaning as the reference harness's ksref_run. Returns the
 * number of conjunctions (written up to conj_cap). */
long kso_run(long n, double* states, uint8_t* alive, const double* size_m, double epoch_jd,
             double t_start, double dt, long steps, int screen, double threshold_km,
             double radius_scale, double min_encounter_speed_km_s,
             ks_conjunction* conj, long conj_cap, ks_step_stats* stats) {
    double* before = (double*)malloc(sizeof(double) * 6 * (size_t)(n > 0 ? n : 1));
    ks_conjunction* tmp = NULL;
    long tmp_cap = 0, total = 0;
    double t = t_start;
    for (long step = 0; step < steps; ++step) {
        if (screen) memcpy(before, states, sizeof(double) * 6 * (size_t)n);
        double moon[9];
        kso_step_moon(epoch_jd, t, dt, moon);
        const double t0 = t;
        kso_step(n, states, alive, dt, moon);
        t += dt;
        if (!screen) continue;
        ks_step_stats st;
        long nf = kso_screen(n, before, states, alive, size_m, t0, dt, threshold_km, radius_scale,
                             min_encounter_speed_km_s, tmp, tmp_cap, &st);
        if (nf > tmp_cap) {
            free(tmp);
            tmp_cap = nf * 2;
            tmp = (ks_conjunction*)malloc(sizeof(ks_conjunction) * (size_t)tmp_cap);
            nf = kso_screen(n, before, states, alive, size_m, t0, dt, threshold_km, radius_scale,
                            min_encounter_speed_km_s, tmp, tmp_cap, &st);
        }
        for (long k = 0; k < nf; ++k) {
            if (total < conj_cap) {
                conj[total] = tmp[k];
                conj[total].step = step;
            }
            ++total;
        }
        if (stats) {
            st.step = step;
            stats[step] = st;
        }
    }
    free(tmp);
    free(before);
    return total;
}
