// Internal interface between the host engine (ks_engine.cu) and the kernels
// (ks_kernels.cu). Not part of the public C ABI.
//
// Device data layout (one context, capacity `cap` objects):
//   state[2]     two FP64 buffers of cap states, 6 contiguous doubles each
//                {rx, ry, rz, vx, vy, vz} (the reference's State), ping-ponged
//                each step (start-of-step -> end-of-step)
//   alive[2]     one byte per object per buffer
//   size_m       characteristic size L (m); collision radius = L/2
//   keys/idx     cell keys (u64) and object indices (i32), two buffers each for the radix sort
//   cells        begin offsets, keys, column-list lengths, 13 forward neighbours per cell
//   hash         open-addressing table cell key -> cell index
//   sorted       start-of-step states gathered in cell order (AoS, 6 doubles per entry)
//   items        pair work list: (cell, row block, first column block, column blocks);
//                a cell's columns are its own objects then its 13 forward
//                neighbours' objects, in blocks of 32
//   survivors    pairs sent to refinement (int2, i < j)
//   conj         conjunction records of the current chunk of steps
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ks_exact.cuh"
#include "ks_records.h"

namespace ks {

// A collision the refinement found, listed for the device SBM.
struct CollisionRec {
    int i, j;
    double t;
};

// Per-step inputs computed on the host.
struct StepParams {
    double t0;         // start of the step, seconds since epoch (Simulation::t)
    int64_t step;      // global index of the step in the run
    MoonStage m[3];    // moon at t0, t0 + dt/2, t0 + dt (src/core/orbital.cpp:287-289)
};

// Grid actually used for one step: cell edge and the compact key layout.
// Cell coordinates (floor(r / cell)) are shifted by lo and packed as
// cx << (wy + wz) | cy << wz | cz; below them, 3 * sub bits order the objects
// of a cell by the Morton code of their 2^sub x 2^sub x 2^sub sub-cell (any
// order inside a cell gives the same pairs); bit `bits` marks objects outside
// the grid.
struct GridParams {
    double cell;
    double inv_cell;     // 1 / cell, correctly rounded (cell_key's fast quotient)
    long long lo[3];
    long long span[3];   // hi - lo per axis
    int w[3];
    int rbits;           // realisation index bits, above the cell coordinates (batches)
    int sub;             // sub-cell bits per axis
    int bits;            // rbits + wx + wy + wz + 3 * sub
};

enum : int {
    FLAG_SURVIVOR_OVERFLOW = 1,
    FLAG_CONJ_OVERFLOW = 2,
    FLAG_SORT_BITS = 4,      // more key bits than the sort passes launched cover
    FLAG_KEY_RANGE = 8,      // a key fell outside its grid bounds
    FLAG_ITEMS_OVERFLOW = 16,  // pair work list longer than its buffer
    FLAG_TIMEOUT = 32,       // a bounded device-side wait gave up
    FLAG_KEYS_REBUILT = 64,  // k_fix_keys rebuilt the keys: their digit histogram is recounted
    FLAG_PACK_WIDTH = 128,   // cell key + dead flag + object index do not fit 64 bits: sort unpacked
    FLAG_CONJ_LARGE = 256,   // more records than the one-block ordering takes: ordered by the multi-block sort
    FLAG_COLL_OVERFLOW = 512,   // device SBM: more collisions in one step than its event buffer holds
    FLAG_POP_BUDGET = 1024,     // device SBM: fragments would pass the population's capacity
    FLAG_HALTED = 2048,         // device SBM: an earlier step of the chunk was left void; this step does nothing
    FLAG_CONJ_TIES = 4096,      // records sharing an ordering key in a run longer than the device orders: the host orders
};


// Per-step control block, device resident.
struct Ctrl {
    // Speculation inputs, written by the previous step: largest speed and
    // position bounds over the objects alive at the start of this step.
    unsigned long long spec_vmax;      // bits of a non-negative double
    unsigned long long bb_min[3];      // order-preserving encodings of doubles
    unsigned long long bb_max[3];
    // Results of this step.
    unsigned long long vmax_true;      // largest start speed over objects alive after the step
    unsigned long long candidates;
    unsigned long long co_orbiting;
    unsigned long long refined;
    unsigned long long conj;
    unsigned long long object_steps;   // objects propagated (alive at start)
    unsigned long long exact_evals;    // candidates that needed the full filter
    int n_alive;                       // alive after the step
    int n_cells;
    unsigned int n_items;              // pair work items
    unsigned int item_ticket;          // next pair work item to hand out
    int max_cell;
    int flags;
    unsigned int n_coll;               // collisions of this step listed for the device SBM
    GridParams grid;
};

// Pair work items of a step.
inline int64_t items_total(const Ctrl& c) { return static_cast<int64_t>(c.n_items); }

struct ChunkCtrl {
    int halt_step;                     // device SBM: first step of the chunk left void (-1: none); later steps did nothing
    int n_live;                        // device SBM: population size at the chunk's end
    unsigned int events;               // device SBM: breakup records of the chunk
    unsigned long long conj_count;     // records appended in this chunk
    int flags;
    int sort_n;                        // records ordered by the chunk's conjunction sort
};

struct DeviceBuffers {
    int64_t cap = 0;
    double* state[2] = {nullptr, nullptr};
    uint8_t* alive[2] = {nullptr, nullptr};
    double* size_m = nullptr;
    uint16_t* real_id = nullptr;           // realisation of each object (batches), else null
    double* ckpt_state = nullptr;
    uint8_t* ckpt_alive = nullptr;
    unsigned long long* keys[2] = {nullptr, nullptr};
    int* idx[2] = {nullptr, nullptr};
    unsigned int* sort_hist = nullptr;     // 8 passes x 256 digits (global offsets); in a context, a second
                                           // 8 x 256 for keys k_fix_keys rebuilt
    unsigned int* sort_status = nullptr;   // look-back words: passes x tiles x 256
    int64_t sort_status_len = 0;
    unsigned int* sort_ctr = nullptr;      // tile tickets, one per pass
    int* block_counts = nullptr;           // cell heads per tile
    unsigned int* fused = nullptr;         // k_sort_cells: barrier, digit totals, per-block counts and starts
    int fused_grid = 0;                    // blocks the fused scratch is sized for
    int* cell_begin = nullptr;             // cap + 1
    unsigned long long* cell_key = nullptr;
    int* nbr = nullptr;                    // 13 per cell
    int* cell_len = nullptr;               // per cell: length of its column list
    int2* col_tab = nullptr;               // per cell: its column list's segments for the pair kernel (16 int2)
    unsigned int* item_part = nullptr;     // heavy, then light cells' work items per chunk of 256 cells, then offsets
    int4* items = nullptr;
    int64_t items_cap = 0;
    unsigned long long* hash_keys = nullptr;
    int* hash_vals = nullptr;
    int64_t hash_cap = 0;                  // power of two
    double* sorted = nullptr;              // 6 per sorted entry
    float4* sorted32 = nullptr;            // FP32 records: cell-relative position, velocity, in cell order
    float4* rec32 = nullptr;               // the same records in object order, written with the keys
    int* sorted_orig = nullptr;
    int2* survivors = nullptr;
    int64_t surv_cap = 0;
    ks_conjunction* conj = nullptr;
    int64_t conj_cap = 0;
    // Ordering of a chunk's conjunction records on the device (radix sort on a
    // 32-bit key monotone in t, record index in the low bits): keys ping-pong, look-back status,
    // digit histograms, tile tickets, and the records in order.
    unsigned long long* conj_keys[2] = {nullptr, nullptr};
    unsigned int* conj_status = nullptr;
    unsigned int* conj_hist = nullptr;
    unsigned int* conj_ctr = nullptr;
    ks_conjunction* conj_sorted = nullptr;
    Ctrl* ctrl = nullptr;                  // max_chunk + 1 entries
    int ctrl_len = 0;
    ChunkCtrl* chunk = nullptr;
    StepParams* params = nullptr;          // max_chunk entries
    // Fragmentation on the device (NASA SBM, counter-based draws): the
    // population grows inside a chunk up to `cap` objects.
    int* n_live = nullptr;                 // current population size
    double* mass_kg = nullptr;             // per object (0 = unknown)
    double* a2m = nullptr;                 // area-to-mass ratio (m^2/kg), fragments
    int32_t* event_of = nullptr;           // originating event (-1: initial population)
    struct CollisionRec* coll = nullptr;   // this step's collisions (refinement output)
    int coll_cap = 0;
    struct SbmEventWork* sbm_work = nullptr;  // coll_cap events of a step
    ks_breakup_event* sbm_events = nullptr;   // the chunk's breakup records
    int64_t sbm_events_cap = 0;
    int* sbm_next_event = nullptr;         // next event number per realisation
    int* sbm_order = nullptr;              // a step's collisions in (t, i, j) order (coll_cap)
    int* sbm_first = nullptr;              // per object: its first event of the step (cap)
    int* sbm_pending = nullptr;            // a step's events whose parents met an earlier event
    int* sbm_misc = nullptr;               // [0]: how many of those
};

// Launch-shape knobs (set through ks_set_tuning; 0 = default).
struct Tuning {
    int pair_variant = 2;         // FP64 gate: 0 two columns per lane, 1 one; 2: FP32 gate on cell-relative records
    int pair_blocks_per_sm = 0;   // resident blocks of the pair kernel
    int subcell_bits = 1;         // Morton order inside cells, bits per axis (0..3)
    int box_min_rows = 4;         // split pairs: block-box pruning for tiles with at least this many rows (0: off)
    double cell_scale = 1.0;      // cell edge = reference edge x this (>= 1; changes only candidate counts)
    int prop_block = 128;         // threads per block of the propagation kernels (32..128, multiple of 32)
    int item_col_blocks = 16;     // column blocks of 32 per pair work item (1..64)
    int lookback_polls = 1 << 22; // polls of a radix-sort look-back before it gives up (FLAG_TIMEOUT)
    int pair_gate_x2 = 1;         // FP32 pair gate on two rows per instruction (packed f32x2)
    int pair_stage2 = 1;          // second FP32 stage: 0 row by row, 1 compacted when sparse, 2 always compacted
    int sort_rank_ballot = 0;     // radix ranking by eight ballots instead of the hardware match
    int prop_min_blocks = 4;      // FP64 propagation: resident 128-thread blocks per SM it is compiled for (4..6)
    int sort_fused = 1;           // object sort and cell build in one cooperative launch (k_sort_cells) where it fits
    int sort_digit_bits = 8;      // fused sort: 8-bit digits; 11: 11-bit digits where they save a pass and fit
    int hash_slots_per_cell = 0;  // fused cell build: 0 packed buckets (4 slots a cell) where keys fit, else the whole
                                  // table; n: (key, cell) pairs over n slots a cell (rounded to a power of two)
};

// Time from a fragmentation event to the end of its step and the lunar stages
// of that sub-step (dt = 0: the event closes the step).
struct FragSpan {
    double dt;
    MoonStage m[3];
};

// Everything a step's kernels need, by value.
struct StepArgs {
    Tuning tune;
    ForceConsts fc;
    double dt;
    double threshold_km;
    double vmin2;
    double radius_scale;
    double gate_hi2;           // unused by the propagation kernel
    int n;                     // population size (objects, alive or not)
    int rbits;                 // realisation bits of the keys (0: one population)
    const uint16_t* real_id;   // realisation of each object, or null
    int screening;             // 0: propagation only
    int precision;             // KS_PRECISION_FP64 or KS_PRECISION_SPLIT
    int sort_passes;
    const StepParams* sp;      // this step's inputs
    Ctrl* ctrl;                // this step's control block
    Ctrl* ctrl_next;           // next step's control block (speculation outputs)
    int src;                   // state buffer holding the start of the step (0 or 1)
    unsigned int* hist;        // radix digit histogram the propagation fills with the keys it emits, or null
    float4* rec32;             // FP32 record of each object, written with its key (object order)
    int pack_bits;             // > 0: sort keys carry the object index in their low pack_bits bits
    // Fragmentation on the device (null / 0 otherwise): the live population
    // size (kernels bound their loops by it; n above is then the capacity the
    // grids are sized for), and the chunk control whose halt_step voids the
    // rest of the chunk.
    const int* n_live;
    ChunkCtrl* chunk;
    int step_in_chunk;
    int steps_in_chunk;
    CollisionRec* coll;        // device SBM: collisions of the step, for fragmentation (null: not listed)
    int coll_cap;
};

// A step whose results are void does nothing past that point:
//  - a radix pass whose look-back gave up (FLAG_TIMEOUT) leaves the step's
//    keys unordered and partly stale, and packed keys carry object indices:
//    every kernel of the step that consumes them returns at once, so that no
//    index read from such a key is ever used;
//  - with fragmentation on the device, a step after one left void (FLAG_HALTED,
//    set by launch_step_gate) runs nothing at all, and the next chunk starts
//    again at the void step.
// The host discards the void steps.
__device__ __forceinline__ bool step_void(const Ctrl* c) { return (c->flags & (FLAG_TIMEOUT | FLAG_HALTED)) != 0; }

// Population size a kernel works on: the live count when the population can
// grow inside a chunk, else the fixed n.
__device__ __forceinline__ int live_n(const StepArgs& a) { return a.n_live ? *a.n_live : a.n; }


// One event of the device SBM, passed between its kernels.
struct SbmEventWork {
    double s[2][6];        // target, projectile: states at the event time
    double size_m[2];      // characteristic sizes (upper bounds of their fragments)
    double budget[2];      // mass each gives to fragments (kg)
    double mass[2];        // masses before the event (kg)
    double vrel;           // km/s
    double t;              // event time, seconds since epoch
    double rem;            // rest of the step after the event (s)
    double expected;       // N(> L_c) of the number law
    long long n_cand;      // candidates drawn (Poisson count, capped)
    int target, projectile;  // object indices (-1: a forced impact's projectile)
    int realisation;
    int id;                // event number within its realisation
    int catastrophic;
    int kept;              // fragments kept (within budget, bound to the Earth)
    int escaped;
    int offset;            // first of its fragments after the population's end
    double kept_mass;
    int record;            // index of its breakup record in the chunk
};

// Device SBM parameters.
struct SbmArgs {
    double lc_m;
    double catastrophic_j_per_g;
    unsigned long long seed;
    int cap;               // population capacity (memory budget)
    int realisations;      // realisations of the batch (event numbers are per realisation)
};

// Kernel launchers (ks_kernels.cu). All enqueue on `stream` and never synchronise.
// checkpoint: also save the carried speculation into its checkpoint slot (replays restore it).
void launch_chunk_init(const DeviceBuffers& b, int k_steps, cudaStream_t stream, bool checkpoint = false);
void launch_seed_ctrl(const DeviceBuffers& b, int n, int src, Ctrl* target, int use_alive_src,
                      cudaStream_t stream);
void launch_propagate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
void launch_screen_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
// Fragments born inside a step: rows [first, first + count) advanced over
// their events' remaining time (spans[row_span[k]]), then their alive flags set.
void launch_advance_spans(const ForceConsts& fc, const FragSpan* spans, const int* row_span, int64_t first,
                          int count, double* state, uint8_t* alive, cudaStream_t stream);
// rows[12 q ..] = the 6 start-of-step then 6 end-of-step doubles of object idx[q].
void launch_gather_rows(const double* before, const double* after, const int64_t* idx, int count, double* rows,
                        cudaStream_t stream);
// alive[idx[q]] = 0.
void launch_clear_alive(uint8_t* alive, const int64_t* idx, int count, cudaStream_t stream);
void launch_fix_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
void launch_sort(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
bool f32_records(const StepArgs& a);
void launch_cells(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
// Fused sort + cell build: blocks per launch on the current device (0: not
// available), scratch words for that grid, whether a step takes the fused path.
int fused_grid();
int64_t fused_scratch_words(int grid);
bool sort_cells_fused(const DeviceBuffers& b, const StepArgs& a);
void launch_sort_cells(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
void launch_pairs(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
// Orders the chunk's conjunction records by TCA into conj_sorted (records
// whose TCAs share a 32-bit key keep their append order; the host finishes
// the (t, i, j) order). t_start: device address of the chunk's first step
// start time; span_s: the chunk's duration.
// Records ordered by one block in shared memory (chunks expected to hold few).
constexpr int kConjSmall = 16384;
void launch_conj_sort(const DeviceBuffers& b, ChunkCtrl* chunk, const double* t_start, double span_s, bool small,
                      cudaStream_t stream);
void launch_refine(const DeviceBuffers& b, const StepArgs& a, ks_conjunction* conj_out, int64_t conj_cap,
                   ChunkCtrl* chunk, cudaStream_t stream);

// Device SBM (ks_sbm.cu). After a step's refinement: voids the rest of the
// chunk if the step's buffers overflowed, then fragments the step's
// collisions in (t, i, j) order and appends the fragments, carried to the
// step's end, after the live population.
void launch_step_gate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream);
void launch_sbm_step(const DeviceBuffers& b, const StepArgs& a, const SbmArgs& s, cudaStream_t stream);
// Fragments `count` events already in b.sbm_work (forced impacts, no step):
// number draws, budgets, fragments appended at the end of state/alive.
void launch_sbm_prepared(const DeviceBuffers& b, const SbmArgs& s, const ForceConsts& fc, int count, int64_t step,
                         double* state, uint8_t* alive, Ctrl* spec, ChunkCtrl* chunk, cudaStream_t stream);
// Collisions one step can fragment on the device (a step with more fails the run).
constexpr int kSbmStepEvents = 16384;
// Sets the kernels' launch attributes (dynamic shared memory); once per device.
cudaError_t sbm_init_attributes();
// Index of the key/idx buffer holding the sorted result after `passes` passes.
inline int sorted_buffer(int passes) { return passes & 1; }

int sm_count();
cudaError_t measure_fp64(double* addmul_per_s, double* fma_per_s, cudaStream_t stream);
cudaError_t measure_fp32(double* addmul_per_s, double* fma_per_s, cudaStream_t stream);
cudaError_t measure_fp32x2(double* fma_ops_per_s, cudaStream_t stream);

}  // namespace ks
