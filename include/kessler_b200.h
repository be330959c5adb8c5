/*
 * kessler_b200 - C ABI of the B200 engine for the per-step hot path of
 * Kessler_Sim: RK4 propagation (point-mass Earth + J2 + Moon) followed by
 * hash-grid conjunction screening (linear pair filter + Hermite TCA refinement).
 *
 * Plain C: pointers, sizes and status codes only. One context owns one CUDA
 * stream on one device and the device-resident population. A context is not
 * re-entrant: drive it from one host thread.
 *
 * Each entry point names the reference interface it replaces (paths inside the
 * reference repository). Units are km, s, km/s in the ECI frame of the input.
 * States are passed in the reference's kessler::State layout: 6 doubles per
 * object, {rx, ry, rz, vx, vy, vz} (src/core/orbital.hpp:51).
 */
#ifndef KESSLER_B200_H
#define KESSLER_B200_H

#include <stddef.h>
#include <stdint.h>

#include "ks_records.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ks_ctx ks_ctx;

/* Status codes. The reference reports failures as bool + message and then
 * falls back to the CPU for good (src/core/collision.cpp:706-714); this ABI
 * returns a status and keeps the message for ks_last_error, with no fallback. */
enum {
    KS_OK = 0,
    KS_ERR_ARG = 1,        /* bad argument (null pointer, negative size, ...) */
    KS_ERR_CUDA = 2,       /* a CUDA call failed; see ks_last_error */
    KS_ERR_NO_DEVICE = 3,  /* no usable CUDA device */
    KS_ERR_STATE = 4,      /* call out of order (e.g. ks_run before ks_set_population) */
    KS_ERR_OVERFLOW = 5,   /* a device buffer stayed too small after retries */
    KS_ERR_RANGE = 6,      /* input outside the supported domain (grid keys, sizes) */
    KS_ERR_TIMEOUT = 7     /* a bounded device-side wait gave up */
};

/* Precision of the propagation and of the pair screening. */
enum {
    KS_PRECISION_FP64 = 0,  /* plain form: every operation in FP64, in the reference's order,
                               no FMA contraction; bit-identical to the reference CPU path */
    KS_PRECISION_SPLIT = 1  /* FP64 state, central term and relative positions; FP32 J2 and
                               lunar terms and FP32 recentred pair gate (FP64 re-check) */
};

/* --- lifecycle: replaces gpu::create / gpu::destroy (src/core/collision_gpu.hpp:47-48)
 *     and the device side of Screener::set_gpu (src/core/collision.hpp:93). */
int ks_create(int device, ks_ctx** out);
void ks_destroy(ks_ctx* ctx);
const char* ks_last_error(const ks_ctx* ctx);
const char* ks_device_name(const ks_ctx* ctx);
/* cudaStream_t of the context, for callers that time or order work around it. */
void* ks_stream(ks_ctx* ctx);

/* --- population: the device becomes the owner of Simulation::objects' states
 *     (src/core/orbital.hpp:145; Object::s, alive, size_m at :71-78).
 *     states: n x 6 doubles; size_m: n doubles (characteristic size L, metres;
 *     collision radius = L/2, src/core/collision.cpp:283-287); alive: n bytes or NULL (all alive). */
int ks_set_population(ks_ctx* ctx, int64_t n, const double* states, const double* size_m,
                      const uint8_t* alive);
/* A batch of independent realisations (Monte Carlo runs) resident together:
 * realisation r owns objects offsets[r] .. offsets[r+1]-1 of the arrays
 * (offsets has realisations + 1 entries, offsets[0] = 0, at most 65535
 * realisations). Every kernel of a step covers all realisations; objects of
 * different realisations never share a cell, so each realisation's
 * conjunctions are those of a run on its objects alone. Conjunction indices
 * are batch-wide, with the realisation in ks_conjunction.realisation; step
 * counters are sums over realisations. Replaces one Simulation per
 * realisation (src/core/orbital.hpp:144-163). */
int ks_set_population_batch(ks_ctx* ctx, int32_t realisations, const int64_t* offsets, const double* states,
                            const double* size_m, const uint8_t* alive);
int ks_get_population(ks_ctx* ctx, int64_t n, double* states, uint8_t* alive);
int64_t ks_population_size(const ks_ctx* ctx);

/* --- clock: Simulation::{epoch_jd, t, dt} (src/core/orbital.hpp:146-148). */
int ks_set_clock(ks_ctx* ctx, double epoch_jd, double t, double dt);
int ks_get_clock(const ks_ctx* ctx, double* t, int64_t* steps_done);

/* --- screening configuration: ScreeningConfig (src/core/collision.hpp:26-37);
 *     enabled=0 runs propagation only (the CLI without --screen, src/main.cpp:352). */
int ks_set_screening(ks_ctx* ctx, int enabled, double threshold_km, double radius_scale,
                     double min_encounter_speed_km_s);
int ks_set_precision(ks_ctx* ctx, int precision);
/* Steps captured per CUDA graph (0 = launch kernels directly, no graph). */
int ks_set_steps_per_graph(ks_ctx* ctx, int steps_per_graph);
/* Per-phase CUDA-event timing of every step (adds event records to each step). */
int ks_set_profiling(ks_ctx* ctx, int enabled);
/* Upper bounds (0 = none) on the survivor-pair and conjunction buffers, which
 * otherwise grow on demand (the reference grows its pair list the same way,
 * src/core/collision_gpu.cu:424-437). A step that needs more replays, then
 * fails with KS_ERR_OVERFLOW. */
int ks_set_buffer_limits(ks_ctx* ctx, int64_t survivor_pairs, int64_t conjunctions);
/* Writes `bytes` of scratch before every step (0 = off), so that each step
 * starts with a cold L2; for measurements. */
int ks_set_l2_flush(ks_ctx* ctx, int64_t bytes);

/* Launch-shape knobs (no counterpart in the reference): "pair_variant" (FP64
 * precision's pair kernel: 0 FP64 gate, two columns per lane; 1 FP64 gate, one
 * column per lane; 2, the default, the split kernel's FP32 gate on
 * cell-relative records; every variant decides with the exact FP64 filter),
 * "pair_blocks_per_sm" (0 = default: 4 for the split kernel; 5 compiles it for
 * 48 registers),
 * "subcell_bits" (0..3: Morton order of objects inside a cell; default 1), "box_min_rows"
 * (split pair kernel: skip tiles whose row and column blocks are provably
 * apart, for tiles of at least this many rows; default 4; 0 = off), "cell_scale_permille"
 * (1000..4000: grid cell edge = the reference's edge x value/1000),
 * "prop_block" (32..128, threads per block of the propagation kernels),
 * "item_col_blocks" (1..64, column blocks of 32 per pair-kernel work item),
 * "pack_keys" (1: the radix sort carries the object index in the low bits of
 * its keys where they leave room, the default; 0: a separate index array),
 * "pair_gate_x2" (1, the default: the FP32 pair gate evaluates two rows per
 * instruction with packed f32x2 arithmetic, decisions identical to the scalar
 * gate's; 0: one row at a time),
 * "pair_stage2" (second FP32 stage of the pair kernel, on the pairs the gate
 * flags: 0 row by row over the warp's flagged rows, 1 the default, one pair
 * per lane from a queue when the flags are sparse, 2 always queued),
 * "prop_min_blocks" (4..6, default 4: resident 128-thread blocks per SM the
 * FP64 propagation kernel is compiled for; more blocks, fewer registers each),
 * "sort_rank_ballot" (radix-sort ranking within a warp: 0, the default, by
 * the hardware match instruction; 1 by eight ballots, one per digit bit),
 * "sort_fused" (1, the default: the object sort and the cell build run as one
 * cooperative launch of one 1024-thread block per SM, grid barriers between
 * their phases, wherever the keys fit its registers (up to 12 288 per SM) and
 * the keys carry the object index; 0: the separate radix passes and cell
 * kernels),
 * "sort_digit_bits" (8, the default: the fused sort takes 8-bit digits; 11:
 * 11-bit digits where that saves a pass and their counters fit, three passes
 * for the four 8-bit ones of 32 key bits),
 * "hash_slots_per_cell" (0..64, default 0: the fused cell build keeps its
 * cell table as (key, cell) words in buckets of four, 4 slots per cell, where
 * the cell keys take at most 40 bits, else the whole hash; n: (key, cell)
 * pairs over the power of two of at least n slots per cell of the step),
 * "lookback_polls" (0..2^30, default 2^22: polls a radix-sort tile makes of a
 * predecessor's unpublished digit counts, or a block of the fused sort makes of
 * a grid barrier, before it gives up; a wait that runs out fails the run with
 * KS_ERR_TIMEOUT and leaves the simulation where the failed chunk of steps
 * began, with no records from it).
 * Conjunctions, refined and co-orbiting counts and states never change;
 * candidate_pairs and cell_km change with the cell edge. */
int ks_set_tuning(ks_ctx* ctx, const char* key, int64_t value);

/* Configuration chosen by ks_autotune. */
typedef struct ks_tuning_choice {
    int32_t steps_per_graph;
    int32_t pair_variant, pair_blocks_per_sm, subcell_bits, box_min_rows;
    int32_t cell_scale_permille;
    int32_t prop_block;
    int32_t item_col_blocks;
    int32_t trials;              /* configurations timed */
    double ms_per_step_start;    /* device time per step of the starting configuration */
    double ms_per_step_best;     /* ... and of the chosen one */
} ks_tuning_choice;

/* Autotuner (no counterpart in the reference, whose OpenMP loop has no launch
 * shape to choose): times short runs of the resident population from a
 * snapshot under candidate steps-per-graph, pair-kernel shapes (variant and
 * resident blocks per SM), sub-cell order, box pruning, grid cell edge and
 * propagation block size, by coordinate descent, and keeps the fastest. Each
 * trial runs at least trial_steps steps (and two graphs). The population,
 * clock, conjunctions and counters are restored afterwards, so the
 * simulation's results are those of an untuned run; only speed changes. */
int ks_autotune(ks_ctx* ctx, int32_t trial_steps, ks_tuning_choice* out);

/* --- run: Simulation::advance (src/core/orbital.hpp:154) with, per step, the
 *     CLI's Screener::begin / Simulation::step / Screener::finish sequence
 *     (src/main.cpp:352-373). Conjunctions and per-step counters accumulate in
 *     the context until taken. */
int ks_run(ks_ctx* ctx, int64_t steps);

/* Captures, instantiates and uploads the graphs that the next ks_run calls
 * launch for chunks of steps_per_graph steps (both step parities), sized as
 * those calls would size them, without running a step, so that a timed run
 * does not pay for their capture. A later change of population size, tuning
 * or buffer sizes captures again where it must. No-op without graphs or with
 * fragmentation on the device. */
int ks_prepare_run(ks_ctx* ctx);

/* Conjunctions found since the last take, ordered by (t, i, j) as Screener::finish
 * orders them (src/core/collision.cpp:743-747). With out == NULL only *count is
 * set (number available). Otherwise up to cap records are moved out. */
int ks_take_conjunctions(ks_ctx* ctx, ks_conjunction* out, int64_t cap, int64_t* count);
/* Zero-copy form of ks_take_conjunctions (no counterpart in the reference,
 * whose records are already host vectors): *first points at the oldest
 * *count records not yet taken, in the same (t, i, j) order, inside the
 * engine's host memory (the pinned buffer the device copied the last chunk's
 * records into, or a holder of older ones), and those records count as taken.
 * Call it until *count is 0 to get every record. The memory stays valid until
 * the next call on ctx that runs steps, sets the population or takes records
 * again; read or copy the records before that. */
int ks_take_conjunctions_view(ks_ctx* ctx, const ks_conjunction** first, int64_t* count);
int ks_take_step_stats(ks_ctx* ctx, ks_step_stats* out, int64_t cap, int64_t* count);

/* --- fragmentation: Fragmentation (src/core/breakup.hpp:100-153), the CLI's
 *     --breakup / --impact (src/main.cpp:28-36, 343-346, 401-407).
 * With on != 0, every collision a step reports is fragmented by the NASA
 * Standard Breakup Model before the next step, as the reference's loop does
 * after Screener::finish: parents destroyed (or the target eroded below the
 * catastrophic threshold), fragments appended after the population and carried
 * to the end of the step. A run of steps ends its chunk at each step that holds
 * a collision. Fragments and events equal the reference's for the same seed
 * (same draws, same arithmetic). lc_m: smallest fragment followed;
 * catastrophic_j_per_g: specific-energy threshold; realisation r of a batch
 * draws from its own stream seeded seed + r. BreakupConfig (breakup.hpp:75-79). */
int ks_set_breakup(ks_ctx* ctx, int on, double lc_m, double catastrophic_j_per_g, uint64_t seed);
/* Where fragmentation runs when ks_set_breakup is on (no counterpart in the
 * reference, which fragments on the host after each step, src/main.cpp:401-407).
 * KS_BREAKUP_HOST (the default): the reference's own draws on the host,
 * fragments identical to the reference's; a chunk of steps ends at each step
 * that holds a collision. KS_BREAKUP_DEVICE: the NASA SBM on the device inside
 * every step, its random numbers drawn from Philox counters named by (seed +
 * realisation, event, fragment, draw); the laws are the reference's, the draws
 * are not, so fragments agree with the reference's in distribution, not one by
 * one. Chunks then run through collisions. The population may grow to
 * max_objects objects, the memory budget allocated when the population is
 * set; fragments that would pass it fail the run with KS_ERR_OVERFLOW, as does
 * a step with more than 16384 collisions (or more than 2048 whose parents collide earlier in the same step). Call before ks_set_population(_batch).
 * ks_autotune, ks_save/load_population, ks_screen and ks_propagate are not
 * available in this mode (KS_ERR_STATE). */
enum { KS_BREAKUP_HOST = 0, KS_BREAKUP_DEVICE = 1 };
int ks_set_breakup_mode(ks_ctx* ctx, int mode, int64_t max_objects);
/* Masses (kg) of the population's objects, 0 = unknown (fragmentation then
 * uses 100 kg): the output of assign_masses (src/core/breakup.cpp:104-111). */
int ks_set_masses(ks_ctx* ctx, int64_t n, const double* mass_kg);
/* Forced impact of a fictitious projectile on object `target`, now:
 * Fragmentation::impact (src/core/breakup.cpp:340-360). */
int ks_impact(ks_ctx* ctx, int64_t target, double projectile_mass_kg, double v_rel_km_s);
/* One forced impact on a lone object, on the host, no context or device: the
 * SBM with a fresh stream seeded `seed` (Fragmentation::impact on a one-object
 * Simulation at time t). Writes up to cap fragments at their birth state
 * (6 doubles each) with size, mass and area-to-mass; target_after receives the
 * target's [alive, mass_kg] afterwards. Returns the number of fragments, or -1. */
int64_t ks_sbm_impact(uint64_t seed, double lc_m, double catastrophic_j_per_g, const double* state,
                      double target_mass_kg, double target_size_m, double projectile_mass_kg, double v_rel_km_s,
                      double t, ks_breakup_event* event, double* frag_states, double* frag_size, double* frag_mass,
                      double* frag_area_to_mass, int64_t cap, double* target_after);
/* Population file (no counterpart in the reference, whose catalogue format
 * carries neither sizes, masses nor fragment provenance, and whose snapshots,
 * src/core/orbital.cpp:190-197, keep only states at 9 digits): writes the
 * resident population bit for bit - states, alive flags, sizes, masses,
 * area-to-mass ratios, originating events, realisations - with the clock and
 * the fragmentation configuration and random streams, so that
 * ks_load_population resumes the run exactly (same states, conjunctions and
 * fragments as an uninterrupted run). Conjunctions, counters and breakup
 * events not yet taken are not saved. Little-endian binary: a "KSPOPv1"
 * header, then the per-object arrays, then the random streams. */
int ks_save_population(ks_ctx* ctx, const char* path);
int ks_load_population(ks_ctx* ctx, const char* path);
/* Fragmentation events since the last take, in the order they happened
 * (same conventions as ks_take_conjunctions). */
int ks_take_breakups(ks_ctx* ctx, ks_breakup_event* out, int64_t cap, int64_t* count);
/* Per-object properties (any pointer may be NULL): size (m), mass (kg, 0 =
 * unknown), area-to-mass ratio (m^2/kg, fragments only), originating event
 * (-1 for the initial population) and realisation. n = ks_population_size. */
int ks_get_objects(ks_ctx* ctx, int64_t n, double* size_m, double* mass_kg, double* area_to_mass, int32_t* event,
                   int32_t* realisation);

/* --- one-shot screening on host states: replaces Screener::screen and screen_step
 *     (src/core/collision.hpp:100-102, 124-128). before/after: n x 6 doubles,
 *     alive_after: n bytes, size_m: n doubles. Results sorted by (t, i, j), step = 0.
 *     Uses the context's device buffers: a resident population is discarded. */
int ks_screen(ks_ctx* ctx, int64_t n, const double* before, const double* after,
              const uint8_t* alive_after, const double* size_m, double t0, double dt,
              ks_conjunction* out, int64_t cap, int64_t* count, ks_step_stats* stats);

/* --- allocation-free one-shot screening. No counterpart in the reference: it
 *     exists for callers that must not allocate GPU memory at call time, such as
 *     an application whose device memory is already handed to its own pool, or
 *     a time-critical loop that cannot afford cudaMalloc / cudaFree, which
 *     synchronise the device. Same inputs and outputs as ks_screen (thresholds
 *     passed explicitly, no context). It always screens in FP64 precision with
 *     the default launch shapes, so its records and counters equal those of
 *     ks_screen on a context left in FP64 precision with default tuning. Its
 *     device buffers are carved from one fixed array in the library's device
 *     image (about 9.3 MB, held by every GPU that loads the library until
 *     exit). Limits: n <= 16384 objects, <= 131072 pairs sent to refinement,
 *     <= 32768 conjunctions; beyond them it returns KS_ERR_RANGE /
 *     KS_ERR_OVERFLOW and writes no records. *count receives the number of
 *     conjunctions found, also when cap or the fixed conjunction capacity is
 *     too small for them, and 0 on every other error. stream is a
 *     cudaStream_t or NULL; the call waits for its own work on it before
 *     returning. error (optional, error_len bytes) receives a message.
 *     The first call on each device looks up the array's device address, so
 *     make that first call before any stream capture. Calls share the array:
 *     calls that overlap on the GPU (other threads, other streams) race. */
int ks_screen_noalloc(int64_t n, const double* before, const double* after, const uint8_t* alive_after,
                      const double* size_m, double t0, double dt, double threshold_km, double radius_scale,
                      double min_encounter_speed_km_s, ks_conjunction* out, int64_t cap, int64_t* count,
                      ks_step_stats* stats, void* stream, char* error, int64_t error_len);

/* --- one-shot propagation on host states: `steps` calls of Simulation::step
 *     without screening (src/core/orbital.cpp:286-300) starting at time t.
 *     states/alive are updated in place. A resident population is discarded. */
int ks_propagate(ks_ctx* ctx, int64_t n, double* states, uint8_t* alive, double epoch_jd,
                 double t, double dt, int64_t steps);

/* --- timing of the last ks_run when profiling is on (milliseconds summed over steps). */
typedef struct ks_timing {
    double propagate_ms;   /* fused RK4 + cell-key kernel */
    double sort_ms;        /* key fix-up + radix sort */
    double cells_ms;       /* cell ranges, hash, neighbour table, sorted gather */
    double pairs_ms;       /* pair enumeration + filter */
    double refine_ms;      /* per-pair TCA refinement */
    double total_ms;       /* device time of all steps */
    int64_t steps;
    int64_t object_steps;  /* sum over steps of alive objects propagated */
    int64_t sort_passes;   /* 8-bit radix passes per step */
    int64_t candidate_pairs;     /* summed over steps */
    int64_t exact_filter_pairs;  /* candidates that needed the full FP64 filter_pair */
    int64_t refined_pairs;       /* pairs refined (Hermite TCA) */
    double chunk_ms;       /* device work of the chunks outside their steps: set-up, checkpoint,
                              ordering of the chunk's conjunction records, replays (L2 flushes excluded) */
    int64_t sort_cells_fused;  /* 1: the last steps sorted and built the cells in one cooperative launch
                                  (sort_ms then holds both, cells_ms is 0); 0: separate kernels */
    /* Host wall time of the run's chunks (fragmentation on the host), always
     * measured: in all, before the first launch of each chunk (parameters,
     * buffer sizing, graph capture), in the launch calls, waiting for the
     * device; the rest is record copies beyond those a chunk brings back,
     * ordering of ties, counters, replays and fragmentation. */
    double host_chunk_ms;
    double host_prep_ms;
    double host_launch_ms;
    double host_sync_ms;
} ks_timing;
int ks_get_timing(const ks_ctx* ctx, ks_timing* out);

/* --- host utilities (no device work) --- */

/* Lunar position (Meeus ch. 47 truncated series), ECI km: the function the
 * reference evaluates three times per step (src/core/orbital.cpp:53-85, 287-289). */
void ks_moon_position(double jd, double out[3]);

/* Seeded synthetic population (Keplerian elements -> Cartesian FP64 ECI).
 * n_base objects of the mixed catalogue (75% LEO, 6% MEO, 6% GEO, 13% GTO/HEO),
 * then n_total - n_base fragments spread around n_parents random LEO base objects.
 * frag_age_max_s: fragments are released up to this long before the epoch
 * (0 = all released at the epoch, at their parent's position).
 * Writes states (n_total x 6), size_m (n_total) and alive (n_total). */
int ks_generate_population(uint64_t seed, int64_t n_base, int64_t n_total, int n_parents,
                           double frag_age_max_s, double* states, double* size_m, uint8_t* alive);

/* FP64 issue rate of this device, measured by a dependent-chain microbenchmark:
 * add/mul instructions per second (no FMA) and FMA instructions per second. */
int ks_measure_fp64(ks_ctx* ctx, double* addmul_per_s, double* fma_per_s);
/* The same for FP32 (add/mul without contraction, and FMA). */
int ks_measure_fp32(ks_ctx* ctx, double* addmul_per_s, double* fma_per_s);
/* Packed FP32 (Blackwell FFMA2, two FMAs per lane and instruction): FMA
 * operations per second, each lane of an f32x2 counted once. */
int ks_measure_fp32x2(ks_ctx* ctx, double* fma_ops_per_s);

#ifdef __cplusplus
}
#endif

#endif /* KESSLER_B200_H */
