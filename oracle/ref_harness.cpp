// Test-infrastructure harness around the UNMODIFIED reference sources.
//
// This file is part of the checker, not of the product. It is compiled together
// with the reference's own src/core/orbital.cpp and src/core/collision.cpp,
// read in place from the reference tree (see oracle/Makefile), into
// oracle/_ref/libksref.so. Only tests/, the smoke check and bench.py's CPU
// baseline leg load it.
//
// It drives the reference exactly the way its CLI step loop does
// (src/main.cpp:346-407): copy `before`, Screener::begin, Simulation::step,
// Screener::finish, collect conjunctions, and (ksref_run_breakup) hand them to
// Fragmentation::apply, with an optional forced impact (Fragmentation::impact)
// at the start of one step.
// Object sizes are set directly (Object::size_m) because the catalogue text
// format only carries radar-cross-section classes (src/core/orbital.cpp:162).

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "core/breakup.hpp"
#include "core/collision.hpp"
#include "core/collision_filter.hpp"
#include "core/orbital.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

#include "ks_records.h"

using namespace kessler;

namespace {

void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

}  // namespace

extern "C" {

int ksref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ksref_moon_position(double jd, double out[3]) {
    Vec3 m = moon_position(jd);
    out[0] = m.x; out[1] = m.y; out[2] = m.z;
}

void ksref_acceleration(const double r[3], const double rm[3], double out[3]) {
    Vec3 a = acceleration(Vec3{r[0], r[1], r[2]}, Vec3{rm[0], rm[1], rm[2]});
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
}

void ksref_rk4(const double s[6], double dt, const double m0[3], const double m1[3],
               const double m2[3], double out[6]) {
    State st{{s[0], s[1], s[2]}, {s[3], s[4], s[5]}};
    State o = rk4(st, dt, Vec3{m0[0], m0[1], m0[2]}, Vec3{m1[0], m1[1], m1[2]},
                  Vec3{m2[0], m2[1], m2[2]});
    out[0] = o.r.x; out[1] = o.r.y; out[2] = o.r.z;
    out[3] = o.v.x; out[4] = o.v.y; out[5] = o.v.z;
}

int ksref_filter_pair(double rx, double ry, double rz, double vx, double vy, double vz,
                      double dt, double threshold_km, double vmin2) {
    return filter_pair(rx, ry, rz, vx, vy, vz, dt, threshold_km, vmin2);
}

int ksref_prefilter_keep(float rx, float ry, float rz, float vx, float vy, float vz,
                         float dt, float threshold_km, float vmin2) {
    return prefilter_keep(rx, ry, rz, vx, vy, vz, dt, threshold_km, vmin2) ? 1 : 0;
}

double ksref_read_epoch_jd(const char* path) { return read_epoch_jd(path); }

// Loads a catalogue with the reference parser. Returns the number of objects
// (or -1); fills at most `cap` rows of states (AoS, 6 doubles), size_m and ids.
long ksref_load_catalog(const char* path, long cap, double* states, double* size_m, int* ids,
                        int* dropped) {
    std::vector<Object> objs = load_catalog(path, dropped);
    const long n = static_cast<long>(objs.size());
    for (long i = 0; i < n && i < cap; ++i) {
        const Object& o = objs[i];
        if (states) {
            double* s = states + 6 * i;
            s[0] = o.s.r.x; s[1] = o.s.r.y; s[2] = o.s.r.z;
            s[3] = o.s.v.x; s[4] = o.s.v.y; s[5] = o.s.v.z;
        }
        if (size_m) size_m[i] = o.size_m;
        if (ids) ids[i] = o.id;
    }
    return n;
}

// One Screener::screen call (CPU backend) on given before/after states.
// Returns the number of conjunctions (written up to `cap`), -1 on bad input.
long ksref_screen(long n, const double* before, const double* after, const uint8_t* alive_after,
                  const double* size_m, double t0, double dt, double threshold_km,
                  double radius_scale, double min_encounter_speed_km_s, int threads,
                  ks_conjunction* out, long cap, ks_step_stats* stats) {
    if (n < 0) return -1;
    set_threads(threads);
    std::vector<State> b(n);
    std::vector<Object> a(n);
    for (long i = 0; i < n; ++i) {
        const double* s = before + 6 * i;
        b[i] = State{{s[0], s[1], s[2]}, {s[3], s[4], s[5]}};
        const double* q = after + 6 * i;
        a[i].s = State{{q[0], q[1], q[2]}, {q[3], q[4], q[5]}};
        a[i].alive = alive_after[i] != 0;
        a[i].size_m = size_m[i];
    }
    ScreeningConfig cfg;
    cfg.threshold_km = threshold_km;
    cfg.radius_scale = radius_scale;
    cfg.min_encounter_speed_km_s = min_encounter_speed_km_s;
    ScreeningStats st;
    std::vector<Conjunction> found = screen_step(b, a, t0, dt, cfg, &st);
    const long nf = static_cast<long>(found.size());
    for (long k = 0; k < nf && k < cap; ++k) {
        const Conjunction& c = found[k];
        out[k] = ks_conjunction{c.i, c.j, 0, c.t, c.miss_km, c.v_rel_km_s, c.collision ? 1 : 0, 0};
    }
    if (stats) {
        long alive = 0;
        for (long i = 0; i < n; ++i) alive += alive_after[i] ? 1 : 0;
        *stats = ks_step_stats{0, st.candidate_pairs, st.refined_pairs, st.co_orbiting, nf,
                               st.cell_km, st.max_cell_objects, static_cast<int32_t>(alive)};
    }
    return nf;
}

namespace {

ks_breakup_event to_record(const BreakupEvent& ev, long step, long first_fragment) {
    ks_breakup_event r{};
    r.step = step;
    r.t = ev.t;
    r.id = ev.id;
    r.realisation = 0;
    r.target = ev.target;
    r.projectile = ev.projectile;
    r.catastrophic = ev.catastrophic ? 1 : 0;
    r.fragments = ev.fragments;
    r.escaped = ev.escaped;
    r.first_fragment = first_fragment;
    r.v_rel_km_s = ev.v_rel_km_s;
    r.energy_j_per_g = ev.energy_j_per_g;
    r.target_mass_kg = ev.target_mass_kg;
    r.projectile_mass_kg = ev.projectile_mass_kg;
    r.sbm_mass_kg = ev.sbm_mass_kg;
    r.expected_fragments = ev.expected_fragments;
    r.fragments_mass_kg = ev.fragments_mass_kg;
    r.position[0] = ev.position.x;
    r.position[1] = ev.position.y;
    r.position[2] = ev.position.z;
    return r;
}

}  // namespace

// Fragmentation::impact on a one-object simulation at time t. Writes up to cap
// fragments (birth states, sizes, masses, area-to-mass); returns the number of
// fragments created. target_after: [alive, mass_kg] of the target afterwards.
long ksref_impact(uint64_t seed, double lc_m, double catastrophic_j_per_g, const double* state, double mass_kg,
                  double size_m, double projectile_mass_kg, double v_rel_km_s, double epoch_jd, double t,
                  ks_breakup_event* event, double* frag_states, double* frag_size, double* frag_mass,
                  double* frag_a2m, long cap, double* target_after) {
    Simulation sim;
    sim.epoch_jd = epoch_jd;
    sim.t = t;
    Object o;
    o.s = State{{state[0], state[1], state[2]}, {state[3], state[4], state[5]}};
    o.mass_kg = mass_kg;
    o.size_m = size_m;
    sim.objects.push_back(o);
    BreakupConfig cfg;
    cfg.lc_m = lc_m;
    cfg.catastrophic_j_per_g = catastrophic_j_per_g;
    cfg.seed = seed;
    Fragmentation frag(cfg);
    const BreakupEvent ev = frag.impact(sim, 0, projectile_mass_kg, v_rel_km_s);
    *event = to_record(ev, 0, 1);
    const long m = static_cast<long>(sim.objects.size()) - 1;
    for (long k = 0; k < m && k < cap; ++k) {
        const Object& f = sim.objects[static_cast<size_t>(k + 1)];
        double* s = frag_states + 6 * k;
        s[0] = f.s.r.x; s[1] = f.s.r.y; s[2] = f.s.r.z;
        s[3] = f.s.v.x; s[4] = f.s.v.y; s[5] = f.s.v.z;
        frag_size[k] = f.size_m;
        frag_mass[k] = f.mass_kg;
        frag_a2m[k] = f.area_to_mass;
    }
    target_after[0] = sim.objects[0].alive ? 1.0 : 0.0;
    target_after[1] = sim.objects[0].mass_kg;
    return m;
}

// The CLI step loop with --breakup (src/main.cpp:343-407): screening every
// step, Fragmentation::apply on its conjunctions, and a forced impact on object
// impact_index (if >= 0) at the start of step impact_step.
//   in:  n objects (states n x 6, alive, size_m, mass_kg; 0 = unknown mass)
//   out: up to obj_cap objects (initial ones then fragments): states, alive,
//        size, mass, area-to-mass, originating event; conjunctions, events,
//        per-step counters (steps entries).
// counts: [objects, conjunctions, events]. Returns 0, or 1 if a capacity was
// too small (counts then hold the sizes needed).
int ksref_run_breakup(long n, const double* states, const uint8_t* alive, const double* size_m, const double* mass_kg,
                      double epoch_jd, double dt, long steps, double threshold_km, double radius_scale,
                      double min_encounter_speed_km_s, int threads, double lc_m, double catastrophic_j_per_g,
                      uint64_t seed, long impact_index, double impact_mass_kg, double impact_vrel_km_s,
                      long impact_step, long obj_cap, double* out_states, uint8_t* out_alive, double* out_size,
                      double* out_mass, double* out_a2m, int32_t* out_event, ks_conjunction* conj, long conj_cap,
                      ks_breakup_event* events, long ev_cap, ks_step_stats* stats, long* counts) {
    set_threads(threads);
    Simulation sim;
    sim.objects.resize(n);
    for (long i = 0; i < n; ++i) {
        const double* s = states + 6 * i;
        Object& o = sim.objects[i];
        o.id = static_cast<int>(i);
        o.s = State{{s[0], s[1], s[2]}, {s[3], s[4], s[5]}};
        o.alive = alive[i] != 0;
        o.size_m = size_m[i];
        o.mass_kg = mass_kg ? mass_kg[i] : 0.0;
    }
    sim.epoch_jd = epoch_jd;
    sim.dt = dt;
    ScreeningConfig cfg;
    cfg.threshold_km = threshold_km;
    cfg.radius_scale = radius_scale;
    cfg.min_encounter_speed_km_s = min_encounter_speed_km_s;
    Screener screener(cfg);
    BreakupConfig bcfg;
    bcfg.lc_m = lc_m;
    bcfg.catastrophic_j_per_g = catastrophic_j_per_g;
    bcfg.seed = seed;
    Fragmentation frag(bcfg);
    std::vector<State> before;
    std::vector<ks_breakup_event> evs;
    long n_conj = 0, next_first = n;
    auto record = [&](const BreakupEvent& ev, long step) {
        evs.push_back(to_record(ev, step, next_first));
        next_first += ev.fragments;
    };
    for (long step = 0; step < steps; ++step) {
        if (impact_index >= 0 && step == impact_step)
            record(frag.impact(sim, static_cast<int>(impact_index), impact_mass_kg, impact_vrel_km_s), step);
        const int nobj = static_cast<int>(sim.objects.size());
        before.resize(nobj);
        for (int i = 0; i < nobj; ++i) before[i] = sim.objects[i].s;
        screener.begin(before, sim.objects, sim.dt);
        const double t0 = sim.t;
        sim.step();
        ScreeningStats st;
        std::vector<Conjunction> found = screener.finish(before, sim.objects, t0, sim.dt, &st);
        for (const Conjunction& c : found) {
            if (n_conj < conj_cap)
                conj[n_conj] = ks_conjunction{c.i, c.j, step, c.t, c.miss_km, c.v_rel_km_s, c.collision ? 1 : 0, 0};
            ++n_conj;
        }
        if (stats) {
            long alive_n = 0;
            for (const Object& o : sim.objects) alive_n += o.alive ? 1 : 0;
            stats[step] = ks_step_stats{step, st.candidate_pairs, st.refined_pairs, st.co_orbiting,
                                        static_cast<int64_t>(found.size()), st.cell_km, st.max_cell_objects,
                                        static_cast<int32_t>(alive_n)};
        }
        for (const BreakupEvent& ev : frag.apply(sim, before, t0, sim.dt, found)) record(ev, step);
    }
    const long m = static_cast<long>(sim.objects.size());
    counts[0] = m;
    counts[1] = n_conj;
    counts[2] = static_cast<long>(evs.size());
    if (m > obj_cap || n_conj > conj_cap || counts[2] > ev_cap) return 1;
    for (long i = 0; i < m; ++i) {
        const Object& o = sim.objects[static_cast<size_t>(i)];
        double* s = out_states + 6 * i;
        s[0] = o.s.r.x; s[1] = o.s.r.y; s[2] = o.s.r.z;
        s[3] = o.s.v.x; s[4] = o.s.v.y; s[5] = o.s.v.z;
        out_alive[i] = o.alive ? 1 : 0;
        out_size[i] = o.size_m;
        out_mass[i] = o.mass_kg;
        out_a2m[i] = o.area_to_mass;
        out_event[i] = o.event;
    }
    std::copy(evs.begin(), evs.end(), events);
    return 0;
}

// The CLI step loop (src/main.cpp:346-407), screening optional, no breakup.
//   states  : in/out, n x 6 doubles (kessler::State layout)
//   alive   : in/out
//   timings : [propagation_s, screening_s, grid_s, pairs_s, wall_s] (optional)
// Returns the total number of conjunctions found (written up to conj_cap), or -1.
long ksref_run(long n, double* states, uint8_t* alive, const double* size_m, double epoch_jd,
               double t_start, double dt, long steps, int screen, double threshold_km,
               double radius_scale, double min_encounter_speed_km_s, int threads,
               ks_conjunction* conj, long conj_cap, ks_step_stats* stats, double* timings) {
    if (n < 0 || steps < 0) return -1;
    set_threads(threads);
    using clock = std::chrono::steady_clock;
    Simulation sim;
    sim.objects.resize(n);
    for (long i = 0; i < n; ++i) {
        const double* s = states + 6 * i;
        Object& o = sim.objects[i];
        o.id = static_cast<int>(i);
        o.s = State{{s[0], s[1], s[2]}, {s[3], s[4], s[5]}};
        o.alive = alive[i] != 0;
        o.size_m = size_m ? size_m[i] : 0.8;
    }
    sim.epoch_jd = epoch_jd;
    sim.t = t_start;
    sim.dt = dt;

    ScreeningConfig cfg;
    cfg.threshold_km = threshold_km;
    cfg.radius_scale = radius_scale;
    cfg.min_encounter_speed_km_s = min_encounter_speed_km_s;
    Screener screener(cfg);
    std::vector<State> before;
    long total = 0;
    double t_prop = 0, t_screen = 0, t_grid = 0, t_pairs = 0;
    const auto w0 = clock::now();
    for (long step = 0; step < steps; ++step) {
        if (screen) {
            const int nobj = static_cast<int>(sim.objects.size());
            before.resize(nobj);
            #pragma omp parallel for schedule(static)
            for (int i = 0; i < nobj; ++i) before[i] = sim.objects[i].s;
            screener.begin(before, sim.objects, sim.dt);
        }
        const double t0 = sim.t;
        const auto c0 = clock::now();
        sim.step();
        const auto c1 = clock::now();
        t_prop += std::chrono::duration<double>(c1 - c0).count();
        if (screen) {
            ScreeningStats st;
            std::vector<Conjunction> found = screener.finish(before, sim.objects, t0, sim.dt, &st);
            t_screen += std::chrono::duration<double>(clock::now() - c1).count();
            t_grid += st.grid_s;
            t_pairs += st.pairs_s;
            for (const Conjunction& c : found) {
                if (total < conj_cap)
                    conj[total] = ks_conjunction{c.i, c.j, step, c.t, c.miss_km, c.v_rel_km_s,
                                                 c.collision ? 1 : 0, 0};
                ++total;
            }
            if (stats) {
                long alive_n = 0;
                for (const Object& o : sim.objects) alive_n += o.alive ? 1 : 0;
                stats[step] = ks_step_stats{step, st.candidate_pairs, st.refined_pairs,
                                            st.co_orbiting, static_cast<int64_t>(found.size()),
                                            st.cell_km, st.max_cell_objects,
                                            static_cast<int32_t>(alive_n)};
            }
        }
    }
    const double wall = std::chrono::duration<double>(clock::now() - w0).count();
    for (long i = 0; i < n; ++i) {
        const Object& o = sim.objects[i];
        double* s = states + 6 * i;
        s[0] = o.s.r.x; s[1] = o.s.r.y; s[2] = o.s.r.z;
        s[3] = o.s.v.x; s[4] = o.s.v.y; s[5] = o.s.v.z;
        alive[i] = o.alive ? 1 : 0;
    }
    if (timings) {
        timings[0] = t_prop; timings[1] = t_screen; timings[2] = t_grid; timings[3] = t_pairs;
        timings[4] = wall;
    }
    return total;
}

}  // extern "C"
