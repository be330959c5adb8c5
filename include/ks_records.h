/*
 * Plain-C record layouts shared by the B200 engine, its C-ABI callers and the
 * CPU checkers. No C++ or CUDA types appear here.
 *
 * Units follow the reference: kilometres, seconds, km/s, Earth-centred
 * inertial frame (src/core/orbital.hpp:4-5).
 */
#ifndef KS_RECORDS_H
#define KS_RECORDS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One close approach found inside a step.
 * Mirrors kessler::Conjunction (src/core/collision.hpp:39-45) and adds the
 * step index so that a multi-step run can be returned as one flat list. */
typedef struct ks_conjunction {
    int32_t i;            /* index into the population, i < j (whole batch for a batched population) */
    int32_t j;
    int64_t step;         /* global step index whose interval (t0, t0+dt) holds the TCA */
    double t;             /* time of closest approach, seconds since epoch */
    double miss_km;       /* distance at TCA */
    double v_rel_km_s;    /* relative speed at TCA */
    int32_t collision;    /* 1 if miss_km < R_i + R_j */
    int32_t realisation;  /* realisation both objects belong to (0 for a single population) */
} ks_conjunction;         /* 48 bytes */

/* Per-step screening counters.
 * Mirrors the counting fields of kessler::ScreeningStats
 * (src/core/collision.hpp:47-62); timings are reported separately. */
typedef struct ks_step_stats {
    int64_t step;              /* global step index */
    int64_t candidate_pairs;   /* pairs produced by the grid (own cell + 13 forward cells) */
    int64_t refined_pairs;     /* pairs the linear filter sent to the Hermite refinement */
    int64_t co_orbiting;       /* pairs under the distance gate but slower than the minimum encounter speed */
    int64_t conjunctions;      /* conjunctions reported for this step */
    double cell_km;            /* grid cell edge used for this step */
    int32_t max_cell_objects;  /* population of the fullest cell */
    int32_t alive;             /* objects alive after the step */
} ks_step_stats;               /* 56 bytes */

/* One fragmentation (collision or forced impact).
 * Mirrors kessler::BreakupEvent (src/core/breakup.hpp:81-98); names are left
 * to the caller (a fragment is "FRAG <id>-<k>" for the k-th fragment of event
 * <id>, a forced impact's projectile "PROJECTILE"). */
typedef struct ks_breakup_event {
    int64_t step;                /* step whose interval holds the event (the next step for a forced impact) */
    double t;                    /* seconds since epoch */
    int32_t id;                  /* event number within its realisation, from 0 */
    int32_t realisation;
    int64_t target, projectile;  /* object indices; -1 for a forced impact's fictitious projectile */
    int32_t catastrophic;
    int32_t fragments;           /* fragments added: objects first_fragment .. first_fragment + fragments - 1 */
    int32_t escaped;             /* fragments on hyperbolic trajectories, dropped */
    int32_t pad;
    int64_t first_fragment;
    double v_rel_km_s;
    double energy_j_per_g;
    double target_mass_kg, projectile_mass_kg;
    double sbm_mass_kg;          /* M of the number law */
    double expected_fragments;   /* N(> L_c) of the law */
    double fragments_mass_kg;
    double position[3];          /* target position at the event, km */
} ks_breakup_event;              /* 144 bytes */

#ifdef __cplusplus
}
#endif

#endif /* KS_RECORDS_H */
