// Host side of the B200 engine: the C ABI declared in include/kessler_b200.h.
//
// The device owns the population for the whole run. ks_run advances it in
// chunks of K steps; a chunk is one CUDA graph (or K direct launches):
//   chunk_init, then per step: propagate, fix_keys, sort, cells, pairs, refine.
// The only per-chunk host work is uploading the K rows of lunar positions,
// reading back K control blocks and the chunk's conjunction records, and
// ordering those records by (t, i, j). Variable-size outputs live in
// fixed-capacity buffers; an overflow flag makes the host grow the buffer,
// restore the chunk's checkpoint and replay the chunk, so results never
// depend on capacities (the reference retries its pair list the same way,
// src/core/collision_gpu.cu:424-437).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <atomic>
#include <chrono>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "kessler_b200.h"
#include "ks_breakup.h"
#include "ks_engine.h"
#include "ks_host.h"

using ks::Ctrl;
using ks::StepArgs;
using ks::StepParams;

namespace {

constexpr int kPhases = 7;  // event slots per step: 0..5 the phases, 6 before the step's L2 flush
constexpr int kMaxReplays = 6;
constexpr int64_t kSbmChunkEvents = 65536;  // breakup records one chunk holds (device fragmentation)

}  // namespace

struct ks_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string name, err;
    ks::DeviceBuffers b;
    int64_t n = 0;
    double epoch_jd = ks::kDefaultEpochJd;
    double t = 0.0, dt = 10.0;
    int64_t steps_done = 0;
    int screening = 1;
    double thr = 5.0, rscale = 1.0, vmin = 0.01;
    int precision = KS_PRECISION_FP64;
    int steps_per_graph = 32;
    int profiling = 0;
    int cur = 0;
    int sort_passes = 8;
    bool has_pop = false;
    int max_chunk = 0;
    StepParams* h_params = nullptr;
    Ctrl* h_ctrl = nullptr;
    ks::ChunkCtrl* h_chunk = nullptr;
    ks_conjunction* h_conj = nullptr;
    int64_t h_conj_cap = 0;
    std::vector<ks_conjunction> conj_out;
    std::vector<ks_conjunction> conj_view;  // older records handed out by the last zero-copy take
    // The last chunk's ordered records, still in h_conj[pend_begin, pend_end):
    // newer than conj_out, moved into it before anything reuses h_conj, so
    // that a caller taking records after every step copies them only once.
    int64_t pend_begin = 0, pend_end = 0;
    std::vector<ks_step_stats> stats_out;
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> ev;
    cudaEvent_t ev_chunk[2] = {nullptr, nullptr};  // around a chunk's device work (profiling)
    ks_timing timing{};
    ks::Tuning tune;
    bool ckpt_states = false;  // the checkpoint holds states (chunks of more than one step)
    int chunk_hint = 0;        // steps of the last chunk that ended early at a collision (0: none)
    void* frag_scratch = nullptr;  // device staging of fragmentation work (parent rows, spans)
    size_t frag_scratch_bytes = 0;
    bool pack_keys = true;     // object index packed below the cell key in the sort keys
    int64_t max_step_conj = 0; // most conjunction records of one step so far (record buffer sizing)
    bool conj_small = false;   // chunks order their records in one block (few expected)
    int64_t chunk_spec = 0;    // records a chunk copies back with its control blocks
    int64_t graph_spec[2] = {0, 0};  // the same, as captured in graph_exec[]
    int64_t graph_n[2] = {-1, -1};   // population size graph_exec[] was captured for
    bool allow_pack = true;    // tuning: packing allowed where the keys leave room
    int realisations = 1;
    int rbits = 0;
    std::vector<int64_t> offsets;  // realisation offsets (batches)
    void* l2_flush = nullptr;
    int64_t l2_flush_bytes = 0;

    // Fragmentation on the device (ks_set_breakup_mode KS_BREAKUP_DEVICE):
    // the population grows inside chunks up to dev_cap objects; no replays,
    // a chunk whose step was left void restarts at that step.
    bool dev_sbm = false;
    int64_t dev_cap = 0;
    ks_breakup_event* h_sbm_events = nullptr;  // pinned copy of a chunk's breakup records
    int dev_stalls = 0;                        // chunks in a row that ended void at their first step

    // Fragmentation (NASA SBM) on the host, between steps. Per-object
    // properties the device does not need are mirrored here, built on first
    // use; one random stream and event counter per realisation.
    struct Breakup {
        bool on = false;
        ks::SbmParams params;
        uint64_t seed = 1;
        std::vector<ks::SbmRng> rng;
        std::vector<int32_t> next_event;
        std::vector<double> size_m, mass_kg, area_to_mass;
        std::vector<int32_t> event;
        std::vector<uint16_t> rid;
        bool mirrors = false;
        std::vector<ks_breakup_event> out;
    } bk;
};

namespace {

int fail(ks_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define KS_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(ctx, KS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

void drop_graphs(ks_ctx* ctx) {
    for (auto& g : ctx->graph_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

void free_objects(ks_ctx* ctx) {
    ks::DeviceBuffers& b = ctx->b;
    for (int k = 0; k < 2; ++k) { dfree(b.state[k]); dfree(b.alive[k]); dfree(b.keys[k]); dfree(b.idx[k]); }
    dfree(b.size_m); dfree(b.real_id); dfree(b.ckpt_state); dfree(b.ckpt_alive); dfree(b.block_counts);
    dfree(b.sort_hist); dfree(b.sort_status); dfree(b.sort_ctr);
    dfree(b.cell_begin); dfree(b.cell_key); dfree(b.nbr); dfree(b.cell_len); dfree(b.col_tab); dfree(b.item_part); dfree(b.hash_keys); dfree(b.hash_vals);
    dfree(b.sorted); dfree(b.sorted32); dfree(b.rec32); dfree(b.sorted_orig); dfree(b.fused);
    b.fused_grid = 0;
    dfree(b.n_live); dfree(b.mass_kg); dfree(b.a2m); dfree(b.event_of); dfree(b.coll); dfree(b.sbm_work);
    dfree(b.sbm_events); dfree(b.sbm_next_event); dfree(b.sbm_order); dfree(b.sbm_first); dfree(b.sbm_pending);
    dfree(b.sbm_misc);
    if (ctx->h_sbm_events) cudaFreeHost(ctx->h_sbm_events);
    ctx->h_sbm_events = nullptr;
    b.coll_cap = 0;
    b.sbm_events_cap = 0;
    b.cap = 0;
    b.hash_cap = 0;
    b.sort_status_len = 0;
}

int ensure_objects(ks_ctx* ctx, int64_t n) {
    // With fragmentation on the device the arrays are sized once for the
    // population's budget: fragments are appended inside the chunks' graphs.
    const int64_t want = ctx->dev_sbm ? std::max(n, ctx->dev_cap) : n;
    if (want <= ctx->b.cap && (!ctx->dev_sbm || ctx->b.n_live)) return KS_OK;
    if (want > (int64_t(1) << 30)) return fail(ctx, KS_ERR_RANGE, "population larger than 2^30 objects");
    drop_graphs(ctx);
    free_objects(ctx);
    ks::DeviceBuffers& b = ctx->b;
    const int64_t cap = std::max<int64_t>(want, 1024);
    for (int k = 0; k < 2; ++k) {
        KS_CUDA(cudaMalloc(&b.state[k], sizeof(double) * 6 * cap));
        KS_CUDA(cudaMalloc(&b.alive[k], cap));
        KS_CUDA(cudaMalloc(&b.keys[k], sizeof(unsigned long long) * cap));
        KS_CUDA(cudaMalloc(&b.idx[k], sizeof(int) * cap));
    }
    KS_CUDA(cudaMalloc(&b.size_m, sizeof(double) * cap));
    KS_CUDA(cudaMalloc(&b.real_id, sizeof(uint16_t) * cap));
    KS_CUDA(cudaMalloc(&b.ckpt_state, sizeof(double) * 6 * cap));
    KS_CUDA(cudaMalloc(&b.ckpt_alive, cap));
    b.sort_status_len = 8 * 256 * ((cap + 2047) / 2048);
    KS_CUDA(cudaMalloc(&b.sort_hist, sizeof(unsigned int) * 2 * 8 * 256));  // propagation's counts, then k_fix_keys's
    KS_CUDA(cudaMalloc(&b.sort_status, sizeof(unsigned int) * b.sort_status_len));
    KS_CUDA(cudaMalloc(&b.sort_ctr, sizeof(unsigned int) * 8));
    KS_CUDA(cudaMalloc(&b.block_counts, sizeof(int) * ((cap + 1023) / 1024 + 1)));
    KS_CUDA(cudaMalloc(&b.cell_begin, sizeof(int) * (cap + 1)));
    KS_CUDA(cudaMalloc(&b.cell_key, sizeof(unsigned long long) * cap));
    KS_CUDA(cudaMalloc(&b.nbr, sizeof(int) * 13 * cap));
    KS_CUDA(cudaMalloc(&b.cell_len, sizeof(int) * cap));
    KS_CUDA(cudaMalloc(&b.col_tab, sizeof(int2) * 16 * cap));
    KS_CUDA(cudaMalloc(&b.item_part, sizeof(unsigned int) * 2 * ((cap + 255) / 256 + 1)));
    int64_t h = 16;
    while (h < 2 * cap) h <<= 1;
    b.hash_cap = h;
    KS_CUDA(cudaMalloc(&b.hash_keys, sizeof(unsigned long long) * h));
    KS_CUDA(cudaMalloc(&b.hash_vals, sizeof(int) * h));
    KS_CUDA(cudaMalloc(&b.sorted, sizeof(double) * 6 * cap));
    KS_CUDA(cudaMalloc(&b.sorted32, sizeof(float4) * 2 * cap));
    KS_CUDA(cudaMalloc(&b.rec32, sizeof(float4) * 2 * cap));
    KS_CUDA(cudaMalloc(&b.sorted_orig, sizeof(int) * cap));
    // Scratch of the fused sort + cell build, sized for this device's grid
    // (looked up here, outside any stream capture).
    if (const int fg = ks::fused_grid()) {
        KS_CUDA(cudaMalloc(&b.fused, sizeof(unsigned int) * ks::fused_scratch_words(fg)));
        b.fused_grid = fg;
    }
    // Every path leaves the cell-key hash empty after a step; it starts so.
    KS_CUDA(cudaMemset(b.hash_keys, 0xFF, sizeof(unsigned long long) * h));
    if (ctx->dev_sbm) {
        KS_CUDA(cudaMalloc(&b.n_live, sizeof(int)));
        KS_CUDA(cudaMalloc(&b.mass_kg, sizeof(double) * cap));
        KS_CUDA(cudaMalloc(&b.a2m, sizeof(double) * cap));
        KS_CUDA(cudaMalloc(&b.event_of, sizeof(int32_t) * cap));
        b.coll_cap = ks::kSbmStepEvents;
        KS_CUDA(cudaMalloc(&b.coll, sizeof(ks::CollisionRec) * b.coll_cap));
        KS_CUDA(cudaMalloc(&b.sbm_work, sizeof(ks::SbmEventWork) * b.coll_cap));
        b.sbm_events_cap = kSbmChunkEvents;
        KS_CUDA(cudaMalloc(&b.sbm_events, sizeof(ks_breakup_event) * b.sbm_events_cap));
        KS_CUDA(cudaHostAlloc(&ctx->h_sbm_events, sizeof(ks_breakup_event) * b.sbm_events_cap, cudaHostAllocDefault));
        KS_CUDA(cudaMalloc(&b.sbm_next_event, sizeof(int) * 65536));
        KS_CUDA(cudaMalloc(&b.sbm_order, sizeof(int) * b.coll_cap));
        KS_CUDA(cudaMalloc(&b.sbm_first, sizeof(int) * cap));
        KS_CUDA(cudaMemset(b.sbm_first, 0x7F, sizeof(int) * cap));  // "no event yet"
        KS_CUDA(cudaMalloc(&b.sbm_pending, sizeof(int) * 2048));
        KS_CUDA(cudaMalloc(&b.sbm_misc, sizeof(int) * 4));
    }
    b.cap = cap;
    return KS_OK;
}

int ensure_survivors(ks_ctx* ctx, int64_t want) {
    if (want <= ctx->b.surv_cap) return KS_OK;
    drop_graphs(ctx);
    dfree(ctx->b.survivors);
    ctx->b.surv_cap = 0;
    KS_CUDA(cudaMalloc(&ctx->b.survivors, sizeof(int2) * want));
    ctx->b.surv_cap = want;
    return KS_OK;
}

int ensure_items(ks_ctx* ctx, int64_t want) {
    if (want <= ctx->b.items_cap) return KS_OK;
    drop_graphs(ctx);
    dfree(ctx->b.items);
    ctx->b.items_cap = 0;
    KS_CUDA(cudaMalloc(&ctx->b.items, sizeof(int4) * want));
    ctx->b.items_cap = want;
    return KS_OK;
}

void free_conj(ks_ctx* ctx) {
    ks::DeviceBuffers& b = ctx->b;
    dfree(b.conj);
    for (int k = 0; k < 2; ++k) dfree(b.conj_keys[k]);
    dfree(b.conj_status); dfree(b.conj_hist); dfree(b.conj_ctr); dfree(b.conj_sorted);
    b.conj_cap = 0;
}

// Moves the pending records of the last chunk behind conj_out.
void stash_pending(ks_ctx* ctx) {
    if (ctx->pend_end > ctx->pend_begin)
        ctx->conj_out.insert(ctx->conj_out.end(), ctx->h_conj + ctx->pend_begin, ctx->h_conj + ctx->pend_end);
    ctx->pend_begin = ctx->pend_end = 0;
}

// Forgets every record not yet taken.
void clear_records(ks_ctx* ctx) {
    ctx->conj_out.clear();
    ctx->pend_begin = ctx->pend_end = 0;
}

int ensure_conj(ks_ctx* ctx, int64_t want) {
    if (want > ctx->b.conj_cap || want > ctx->h_conj_cap) {
        if (want > (int64_t(1) << 30)) return fail(ctx, KS_ERR_RANGE, "more than 2^30 conjunctions in one chunk");
        // Room to grow: callers ask for a margin over the largest count so far,
        // which rises a little at a time; regrowing (and capturing the graphs
        // again) at each rise cost milliseconds per chunk.
        want = std::min<int64_t>(want + want / 2, int64_t(1) << 30);
    }
    if (want > ctx->b.conj_cap) {
        drop_graphs(ctx);
        free_conj(ctx);
        ks::DeviceBuffers& b = ctx->b;
        const int64_t tiles = (want + 2047) / 2048;
        KS_CUDA(cudaMalloc(&b.conj, sizeof(ks_conjunction) * want));
        KS_CUDA(cudaMalloc(&b.conj_sorted, sizeof(ks_conjunction) * want));
        for (int k = 0; k < 2; ++k) KS_CUDA(cudaMalloc(&b.conj_keys[k], sizeof(unsigned long long) * want));
        KS_CUDA(cudaMalloc(&b.conj_status, sizeof(unsigned int) * 256 * 4 * tiles));
        KS_CUDA(cudaMalloc(&b.conj_hist, sizeof(unsigned int) * 8 * 256));
        KS_CUDA(cudaMalloc(&b.conj_ctr, sizeof(unsigned int) * 8));
        b.conj_cap = want;
    }
    if (want > ctx->h_conj_cap) {
        stash_pending(ctx);
        drop_graphs(ctx);  // graphs copy records into h_conj
        if (ctx->h_conj) cudaFreeHost(ctx->h_conj);
        ctx->h_conj = nullptr;
        ctx->h_conj_cap = 0;
        KS_CUDA(cudaHostAlloc(&ctx->h_conj, sizeof(ks_conjunction) * want, cudaHostAllocDefault));
        ctx->h_conj_cap = want;
    }
    return KS_OK;
}

// Control blocks: max_chunk step slots, then the carry slot and its checkpoint.
int ensure_chunk(ks_ctx* ctx, int k) {
    if (k <= ctx->max_chunk) return KS_OK;
    drop_graphs(ctx);
    ks::DeviceBuffers& b = ctx->b;
    // Keep the carried speculation across the reallocation.
    Ctrl carry{};
    const bool keep = b.ctrl != nullptr;
    if (keep) KS_CUDA(cudaMemcpy(&carry, b.ctrl + b.ctrl_len - 2, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    dfree(b.ctrl);
    dfree(b.params);
    if (ctx->h_params) cudaFreeHost(ctx->h_params);
    if (ctx->h_ctrl) cudaFreeHost(ctx->h_ctrl);
    ctx->h_params = nullptr;
    ctx->h_ctrl = nullptr;
    b.ctrl_len = k + 2;
    KS_CUDA(cudaMalloc(&b.ctrl, sizeof(Ctrl) * b.ctrl_len));
    KS_CUDA(cudaMemset(b.ctrl, 0, sizeof(Ctrl) * b.ctrl_len));
    KS_CUDA(cudaMalloc(&b.params, sizeof(StepParams) * k));
    KS_CUDA(cudaHostAlloc(&ctx->h_params, sizeof(StepParams) * k, cudaHostAllocDefault));
    KS_CUDA(cudaHostAlloc(&ctx->h_ctrl, sizeof(Ctrl) * b.ctrl_len, cudaHostAllocDefault));
    if (keep) KS_CUDA(cudaMemcpy(b.ctrl + b.ctrl_len - 2, &carry, sizeof(Ctrl), cudaMemcpyHostToDevice));
    for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
    ctx->ev.assign(static_cast<size_t>(k) * kPhases, nullptr);
    for (auto& e : ctx->ev) KS_CUDA(cudaEventCreate(&e));
    for (cudaEvent_t& e : ctx->ev_chunk)
        if (!e) KS_CUDA(cudaEventCreate(&e));
    ctx->max_chunk = k;
    return KS_OK;
}

Ctrl* carry_slot(ks_ctx* ctx) { return ctx->b.ctrl + ctx->b.ctrl_len - 2; }
Ctrl* carry_ckpt_slot(ks_ctx* ctx) { return ctx->b.ctrl + ctx->b.ctrl_len - 1; }

ks::ForceConsts force_consts() {
    ks::ForceConsts fc;
    fc.neg_mu_earth = -ks::kMuEarth;
    fc.k_j2 = ks::j2_numerator();
    fc.mu_moon = ks::kMuMoon;
    fc.r_earth = ks::kREarth;
    return fc;
}

int passes_for_bits(int bits) { return std::max(1, (bits + 1 + 7) / 8); }

// Host estimate of the key width from a seeded control block. Only sizes the
// number of radix passes; the device checks it and the chunk is replayed with
// more passes if the estimate was short.
int estimate_bits(const Ctrl& c, double dt, double thr, int sub, int rbits, double scale) {
    const double vmax = [&] { double v; std::memcpy(&v, &c.spec_vmax, 8); return v; }();
    auto dec = [](unsigned long long u) {
        unsigned long long b = (u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
        double d;
        std::memcpy(&d, &b, 8);
        return d;
    };
    const double vrel = 2.0 * vmax;
    double cell = vrel * dt + thr + ks::kGravityGradient * vrel * dt * dt * dt;
    if (cell < 1.0) cell = 1.0;
    if (scale > 1.0) cell *= scale;
    int bits = rbits;
    for (int a = 0; a < 3; ++a) {
        const double mn = dec(c.bb_min[a]), mx = dec(c.bb_max[a]);
        if (!(mn <= mx)) continue;
        const long long span = static_cast<long long>(std::floor(mx / cell)) - static_cast<long long>(std::floor(mn / cell));
        int w = 0;
        while (w < 63 && (span >> w) > 0) ++w;
        bits += w;
    }
    return bits + 3 * sub;
}

void fill_params(ks_ctx* ctx, int k_steps, double t_start, int64_t step0, double* t_end) {
    double t = t_start;
    for (int k = 0; k < k_steps; ++k) {
        StepParams& sp = ctx->h_params[k];
        sp.t0 = t;
        sp.step = step0 + k;
        ks::moon_stages(ctx->epoch_jd, t, ctx->dt, sp.m);
        t += ctx->dt;  // Simulation::step (src/core/orbital.cpp:299)
    }
    *t_end = t;
}

// Bits that hold every object index 0 .. n-1 (at least 1).
int index_bits(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

StepArgs step_args(ks_ctx* ctx, int k, int k_steps, int src) {
    StepArgs a{};
    a.tune = ctx->tune;
    a.fc = force_consts();
    a.dt = ctx->dt;
    a.threshold_km = ctx->thr;
    a.vmin2 = ctx->vmin * ctx->vmin;
    a.radius_scale = ctx->rscale;
    a.n = static_cast<int>(ctx->n);
    a.rbits = ctx->rbits;
    a.real_id = ctx->rbits > 0 ? ctx->b.real_id : nullptr;
    a.screening = ctx->screening;
    a.precision = ctx->precision;
    a.sort_passes = ctx->sort_passes;
    a.sp = ctx->b.params + k;
    a.ctrl = ctx->b.ctrl + k;
    a.ctrl_next = (k == k_steps - 1) ? carry_slot(ctx) : ctx->b.ctrl + k + 1;
    a.src = src;
    a.hist = ctx->screening ? ctx->b.sort_hist : nullptr;  // the propagation counts the sort's digits
    a.rec32 = ctx->b.rec32;
    a.pack_bits = ctx->pack_keys ? index_bits(ctx->n) : 0;
    if (ctx->dev_sbm) {
        // Grids sized for the capacity, loops bounded by the live count; the
        // packed object index must hold every index the population can reach.
        a.n = static_cast<int>(ctx->b.cap);
        a.n_live = ctx->b.n_live;
        a.chunk = ctx->b.chunk;
        a.step_in_chunk = k;
        a.steps_in_chunk = k_steps;
        a.coll = ctx->bk.on ? ctx->b.coll : nullptr;
        a.coll_cap = ctx->b.coll_cap;
        a.pack_bits = ctx->pack_keys ? index_bits(ctx->b.cap) : 0;
    }
    // The fused sort counts its own digits: the propagation need not.
    if (a.hist && ks::sort_cells_fused(ctx->b, a)) a.hist = nullptr;
    return a;
}

// Which cell build the steps take: 0 separate kernels, 1 the fused launch.
int fused_form(ks_ctx* ctx) {
    return ctx->screening && ks::sort_cells_fused(ctx->b, step_args(ctx, 0, 1, 0)) ? 1 : 0;
}

ks::SbmArgs sbm_args(const ks_ctx* ctx) {
    ks::SbmArgs s{};
    s.lc_m = ctx->bk.params.lc_m;
    s.catastrophic_j_per_g = ctx->bk.params.catastrophic_j_per_g;
    s.seed = ctx->bk.seed;
    s.cap = static_cast<int>(ctx->b.cap);
    s.realisations = ctx->realisations;
    return s;
}

void record(ks_ctx* ctx, int k, int phase, bool capturing) {
    if (!ctx->profiling) return;
    cudaEvent_t e = ctx->ev[static_cast<size_t>(k) * kPhases + phase];
    if (capturing) cudaEventRecordWithFlags(e, ctx->stream, cudaEventRecordExternal);
    else cudaEventRecord(e, ctx->stream);
}

// End of a chunk's device work, before its results are copied back.
void record_chunk_end(ks_ctx* ctx, bool capturing) {
    if (!ctx->profiling) return;
    if (capturing) cudaEventRecordWithFlags(ctx->ev_chunk[1], ctx->stream, cudaEventRecordExternal);
    else cudaEventRecord(ctx->ev_chunk[1], ctx->stream);
}

// A chunk in stream order: its step parameters up (from h_params), set-up
// (with the checkpoint of the carried speculation), the steps, the ordering
// of its records, and its control blocks and first chunk_spec records back to
// the host, so that running it takes one launch and one synchronisation.
void enqueue_chunk(ks_ctx* ctx, int k_steps, int src0, bool capturing) {
    cudaStream_t s = ctx->stream;
    cudaMemcpyAsync(ctx->b.params, ctx->h_params, sizeof(StepParams) * k_steps, cudaMemcpyHostToDevice, s);
    ks::launch_chunk_init(ctx->b, k_steps, s, true);
    int src = src0;
    for (int k = 0; k < k_steps; ++k) {
        const StepArgs a = step_args(ctx, k, k_steps, src);
        record(ctx, k, 6, capturing);
        if (ctx->l2_flush_bytes > 0) cudaMemsetAsync(ctx->l2_flush, k & 0xFF, ctx->l2_flush_bytes, s);
        record(ctx, k, 0, capturing);
        if (a.hist) cudaMemsetAsync(a.hist, 0, sizeof(unsigned int) * 2 * 8 * 256, s);
        ks::launch_propagate(ctx->b, a, s);
        record(ctx, k, 1, capturing);
        if (ctx->screening) {
            ks::launch_fix_keys(ctx->b, a, s);
            if (ks::sort_cells_fused(ctx->b, a)) {
                ks::launch_sort_cells(ctx->b, a, s);  // sort and cells in one launch: timed as the sort
                record(ctx, k, 2, capturing);
                record(ctx, k, 3, capturing);
            } else {
                ks::launch_sort(ctx->b, a, s);
                record(ctx, k, 2, capturing);
                ks::launch_cells(ctx->b, a, s);
                record(ctx, k, 3, capturing);
            }
            ks::launch_pairs(ctx->b, a, s);
            record(ctx, k, 4, capturing);
            ks::launch_refine(ctx->b, a, ctx->b.conj, ctx->b.conj_cap, ctx->b.chunk, s);
            if (ctx->dev_sbm) {
                ks::launch_step_gate(ctx->b, a, s);
                if (ctx->bk.on) ks::launch_sbm_step(ctx->b, a, sbm_args(ctx), s);
            }
            record(ctx, k, 5, capturing);
        }
        src ^= 1;
    }
    if (ctx->dev_sbm)
        cudaMemcpyAsync(&ctx->b.chunk->n_live, ctx->b.n_live, sizeof(int), cudaMemcpyDeviceToDevice, s);
    if (ctx->screening)
        ks::launch_conj_sort(ctx->b, ctx->b.chunk, &ctx->b.params[0].t0, k_steps * ctx->dt, ctx->conj_small, s);
    record_chunk_end(ctx, capturing);
    cudaMemcpyAsync(ctx->h_ctrl, ctx->b.ctrl, sizeof(Ctrl) * k_steps, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ctx->h_chunk, ctx->b.chunk, sizeof(ks::ChunkCtrl), cudaMemcpyDeviceToHost, s);
    if (ctx->chunk_spec > 0)
        cudaMemcpyAsync(ctx->h_conj, ctx->b.conj_sorted, sizeof(ks_conjunction) * ctx->chunk_spec,
                        cudaMemcpyDeviceToHost, s);
}

// Captures and instantiates the chunk's graph if it does not exist yet.
int ensure_graph(ks_ctx* ctx, int k_steps) {
    const bool use_graph = ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph;
    if (!use_graph) return KS_OK;
    cudaGraphExec_t& exec = ctx->graph_exec[ctx->cur];
    // The population size is in the kernels' arguments (with fragmentation on
    // the host; on the device they hold the capacity): a graph captured for
    // another size, as after fragments were appended, is captured again.
    if (exec && !ctx->dev_sbm && ctx->graph_n[ctx->cur] != ctx->n) drop_graphs(ctx);
    if (!exec) {
        cudaGraph_t g = nullptr;
        KS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_chunk(ctx, k_steps, ctx->cur, true);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
        if (le != cudaSuccess) return fail(ctx, KS_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(le));
        if (ee != cudaSuccess) return fail(ctx, KS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            exec = nullptr;
            return fail(ctx, KS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        // Uploaded now rather than by its first launch.
        KS_CUDA(cudaGraphUpload(exec, ctx->stream));
        ctx->graph_spec[ctx->cur] = ctx->chunk_spec;
        ctx->graph_n[ctx->cur] = ctx->n;
    }
    return KS_OK;
}

int launch_chunk(ks_ctx* ctx, int k_steps) {
    const bool use_graph = ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph;
    if (!use_graph) {
        enqueue_chunk(ctx, k_steps, ctx->cur, false);
        KS_CUDA(cudaGetLastError());
        return KS_OK;
    }
    const int rc = ensure_graph(ctx, k_steps);
    if (rc) return rc;
    KS_CUDA(cudaGraphLaunch(ctx->graph_exec[ctx->cur], ctx->stream));
    return KS_OK;
}

// Start-of-chunk checkpoint for replays. A one-step chunk never overwrites
// its input states (steps ping-pong between two buffers), so its states need
// none; the carried control block is saved by the chunk's own set-up kernel.
int save_checkpoint(ks_ctx* ctx, int k_steps) {
    ks::DeviceBuffers& b = ctx->b;
    ctx->ckpt_states = k_steps > 1;
    if (ctx->ckpt_states) {
        KS_CUDA(cudaMemcpyAsync(b.ckpt_state, b.state[ctx->cur], sizeof(double) * 6 * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.ckpt_alive, b.alive[ctx->cur], ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return KS_OK;
}

int restore_checkpoint(ks_ctx* ctx) {
    ks::DeviceBuffers& b = ctx->b;
    if (ctx->ckpt_states) {
        KS_CUDA(cudaMemcpyAsync(b.state[ctx->cur], b.ckpt_state, sizeof(double) * 6 * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.alive[ctx->cur], b.ckpt_alive, ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    KS_CUDA(cudaMemcpyAsync(carry_slot(ctx), carry_ckpt_slot(ctx), sizeof(Ctrl), cudaMemcpyDeviceToDevice, ctx->stream));
    return KS_OK;
}

bool conj_less(const ks_conjunction& a, const ks_conjunction& b) {
    if (a.t != b.t) return a.t < b.t;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
}

using HostClock = std::chrono::steady_clock;
double host_ms(HostClock::time_point a, HostClock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// (t, i, j) order of records the device already ordered by a key monotone in
// t: only records that shared a key can be out of order, so an insertion
// pass is linear in practice.
template <typename It>
void finish_order(It first, It last) {
    for (It it = first; it != last; ++it) {
        if (it == first || !conj_less(*it, *(it - 1))) continue;
        const ks_conjunction v = *it;
        It j = it;
        do {
            *j = *(j - 1);
            --j;
        } while (j != first && conj_less(v, *(j - 1)));
        *j = v;
    }
}

void accumulate_timing(ks_ctx* ctx, int k_steps) {
    if (!ctx->profiling) return;
    auto el = [&](int k, int p0, int p1) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[static_cast<size_t>(k) * kPhases + p0], ctx->ev[static_cast<size_t>(k) * kPhases + p1]);
        return static_cast<double>(ms);
    };
    double steps_ms = 0.0, flush_ms = 0.0;
    for (int k = 0; k < k_steps; ++k) {
        ctx->timing.propagate_ms += el(k, 0, 1);
        const double step_ms = ctx->screening ? el(k, 0, 5) : el(k, 0, 1);
        if (ctx->screening) {
            ctx->timing.sort_ms += el(k, 1, 2);
            ctx->timing.cells_ms += el(k, 2, 3);
            ctx->timing.pairs_ms += el(k, 3, 4);
            ctx->timing.refine_ms += el(k, 4, 5);
        }
        ctx->timing.total_ms += step_ms;
        steps_ms += step_ms;
        flush_ms += el(k, 6, 0);
    }
    // The chunk's work outside its steps: set-up, checkpoint, ordering of its
    // records (and any replay); the L2 flushes are left out.
    float chunk = 0.f;
    cudaEventElapsedTime(&chunk, ctx->ev_chunk[0], ctx->ev_chunk[1]);
    ctx->timing.chunk_ms += std::max(0.0, static_cast<double>(chunk) - steps_ms - flush_ms);
}

int apply_collisions(ks_ctx* ctx, int64_t step, double t0, const std::vector<ks_conjunction>& hits);

// Runs one chunk of k_steps; replays it after growing whatever overflowed.
// With fragmentation on, a chunk ends at the first step that holds a
// collision (the chunk is replayed up to that step), and the collisions are
// fragmented before the next step, as the reference's loop does after each
// step (src/main.cpp:401-407).
// Sizes the chunk's record buffer and its ordering, and which records come
// back with the control blocks (shared by both chunk loops).
int plan_records(ks_ctx* ctx, int k_steps) {
    int rc = KS_OK;
    // Room for the chunk's records at the largest per-step count seen so far,
    // so that a longer chunk does not overflow and replay; sized for a whole
    // graph's chunk even when this one is shorter (a run's first chunks end
    // early while the counts are learnt), so that the first full chunk does
    // not grow the buffers (pinned host memory included) again.
    if (ctx->screening && ctx->max_step_conj > 0) {
        const int64_t span = std::max<int64_t>(k_steps, ctx->steps_per_graph);
        const int64_t want = std::min<int64_t>(ctx->max_step_conj * span * 5 / 4 + 256, int64_t(1) << 30);
        if (want > ctx->b.conj_cap && (rc = ensure_conj(ctx, want))) return rc;
    }
    // One-block ordering of the records where the chunk should hold few.
    const bool small = ctx->screening && ctx->max_step_conj > 0 &&
                       ctx->max_step_conj * k_steps * 5 / 4 + 256 <= ks::kConjSmall;
    if (small != ctx->conj_small) {
        ctx->conj_small = small;
        drop_graphs(ctx);
    }
    // Records copied back with the control blocks, up to the expected count,
    // so that a chunk with no more than that needs one host round trip.
    const int64_t spec = ctx->screening ? std::min<int64_t>(ctx->max_step_conj * k_steps * 5 / 4 + 256, ctx->b.conj_cap) : 0;
    ctx->chunk_spec = ctx->max_step_conj > 0 && spec <= (int64_t(1) << 16) ? spec : 0;
    const bool use_graph = ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph;
    if (use_graph && ctx->graph_exec[ctx->cur] && ctx->graph_spec[ctx->cur] < ctx->chunk_spec) drop_graphs(ctx);
    return KS_OK;
}

// One chunk with fragmentation on the device. The population grows inside the
// chunk's graph; nothing is replayed: a step whose buffers overflowed (or whose
// sort gave up) is left void together with the rest of the chunk, its
// predecessors' results are kept, the buffers grow, and the next chunk starts
// at the void step from the states the chunk left (a void step never writes
// its start-of-step buffer).
int run_chunk_dev(ks_ctx* ctx, int k_steps) {
    const HostClock::time_point h0 = HostClock::now();
    stash_pending(ctx);
    int rc = ensure_chunk(ctx, k_steps);
    if (rc) return rc;
    double t_end = 0.0;
    fill_params(ctx, k_steps, ctx->t, ctx->steps_done, &t_end);
    if ((rc = plan_records(ctx, k_steps))) return rc;
    if ((rc = ensure_graph(ctx, k_steps))) return rc;
    if (ctx->profiling) KS_CUDA(cudaEventRecord(ctx->ev_chunk[0], ctx->stream));
    const HostClock::time_point hl = HostClock::now();
    ctx->timing.host_prep_ms += host_ms(h0, hl);
    rc = launch_chunk(ctx, k_steps);
    if (rc) return rc;
    const HostClock::time_point hs = HostClock::now();
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->timing.host_launch_ms += host_ms(hl, hs);
    ctx->timing.host_sync_ms += host_ms(hs, HostClock::now());
    const ks::ChunkCtrl ch = *ctx->h_chunk;
    if (ch.flags & ks::FLAG_POP_BUDGET)
        return fail(ctx, KS_ERR_OVERFLOW, "fragments would pass the population budget of " +
                                              std::to_string(ctx->b.cap) + " objects (ks_set_breakup_mode)");
    const int h = ch.halt_step;
    const int done = h < 0 ? k_steps : h;
    const int64_t last_step = ctx->steps_done + done;  // records of steps before this one are complete
    // Limits met inside a step's fragmentation (after its gate) leave that
    // step's fragmentation incomplete: the run fails rather than go on.
    for (int k = 0; k < done; ++k)
        if (ctx->h_ctrl[k].flags & ks::FLAG_COLL_OVERFLOW)
            return fail(ctx, KS_ERR_OVERFLOW, "more than 2048 collisions in one step with a parent that collided earlier "
                                              "in the step, or more breakup records in one chunk than " +
                                              std::to_string(ctx->b.sbm_events_cap));
    // Conjunction records, ordered on the device; those of the void step are dropped.
    int64_t have = (ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph) ? ctx->graph_spec[ctx->cur]
                                                                                : ctx->chunk_spec;
    int64_t nc = std::min<int64_t>(static_cast<int64_t>(ch.conj_count), ctx->b.conj_cap);
    if (ch.flags & ks::FLAG_CONJ_LARGE) {
        ks::launch_conj_sort(ctx->b, ctx->b.chunk, &ctx->b.params[0].t0, k_steps * ctx->dt, false, ctx->stream);
        KS_CUDA(cudaMemcpyAsync(ctx->h_chunk, ctx->b.chunk, sizeof(ks::ChunkCtrl), cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->h_chunk->flags & ks::FLAG_TIMEOUT) return fail(ctx, KS_ERR_TIMEOUT, "radix sort look-back or grid barrier wait gave up");
        have = 0;
    }
    if (nc > have) {
        KS_CUDA(cudaMemcpyAsync(ctx->h_conj + have, ctx->b.conj_sorted + have, sizeof(ks_conjunction) * (nc - have),
                                cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    // Without a void step every record is kept: no pass over them.
    int64_t kept = h < 0 ? nc : 0;
    if (h >= 0)
        for (int64_t q = 0; q < nc; ++q)
            if (ctx->h_conj[q].step < last_step) ctx->h_conj[kept++] = ctx->h_conj[q];
    if (kept > 0) {
        if (ctx->h_chunk->flags & ks::FLAG_CONJ_TIES) finish_order(ctx->h_conj, ctx->h_conj + kept);
        ctx->pend_begin = 0;
        ctx->pend_end = kept;
    }
    // Breakup records of the kept steps (the void step fragmented nothing).
    if (ch.events > 0) {
        const int64_t ne = std::min<int64_t>(ch.events, ctx->b.sbm_events_cap);
        KS_CUDA(cudaMemcpyAsync(ctx->h_sbm_events, ctx->b.sbm_events, sizeof(ks_breakup_event) * ne,
                                cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->bk.out.insert(ctx->bk.out.end(), ctx->h_sbm_events, ctx->h_sbm_events + ne);
    }
    for (int k = 0; k < done; ++k) {
        const Ctrl& c = ctx->h_ctrl[k];
        ks_step_stats st{};
        st.step = ctx->steps_done + k;
        st.candidate_pairs = static_cast<int64_t>(c.candidates);
        st.refined_pairs = static_cast<int64_t>(c.refined);
        st.co_orbiting = static_cast<int64_t>(c.co_orbiting);
        st.conjunctions = static_cast<int64_t>(c.conj);
        st.cell_km = ctx->screening ? c.grid.cell : 0.0;
        st.max_cell_objects = c.max_cell;
        st.alive = c.n_alive;
        ctx->stats_out.push_back(st);
        ctx->max_step_conj = std::max(ctx->max_step_conj, static_cast<int64_t>(c.conj));
        ctx->timing.object_steps += static_cast<int64_t>(c.object_steps);
        ctx->timing.candidate_pairs += static_cast<int64_t>(c.candidates);
        ctx->timing.exact_filter_pairs += static_cast<int64_t>(c.exact_evals);
        ctx->timing.refined_pairs += static_cast<int64_t>(c.refined);
    }
    accumulate_timing(ctx, done);
    ctx->timing.steps += done;
    ctx->timing.sort_passes = ctx->sort_passes;
    ctx->timing.sort_cells_fused = fused_form(ctx);
    ctx->steps_done += done;
    ctx->t = done == k_steps ? t_end : ctx->h_params[done].t0;
    if (done & 1) ctx->cur ^= 1;
    ctx->n = ch.n_live;
    if (h < 0) {
        ctx->dev_stalls = 0;
        return KS_OK;
    }
    // The void step restarts the next chunk: its speculation becomes the carry.
    KS_CUDA(cudaMemcpyAsync(carry_slot(ctx), ctx->b.ctrl + h, sizeof(Ctrl), cudaMemcpyDeviceToDevice, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->dev_stalls = done == 0 ? ctx->dev_stalls + 1 : 0;
    if (ctx->dev_stalls > kMaxReplays) return fail(ctx, KS_ERR_OVERFLOW, "device buffers still overflowing after regrowth");
    const Ctrl& c = ctx->h_ctrl[h];
    const int flags = c.flags | (ch.flags & ks::FLAG_CONJ_OVERFLOW);
    if (flags & ks::FLAG_TIMEOUT) return fail(ctx, KS_ERR_TIMEOUT, "radix sort look-back or grid barrier wait gave up");
    if (flags & ks::FLAG_KEY_RANGE) return fail(ctx, KS_ERR_RANGE, "cell key outside its grid bounds or wider than 63 bits");
    if (flags & ks::FLAG_COLL_OVERFLOW)
        return fail(ctx, KS_ERR_OVERFLOW, "more than " + std::to_string(ks::kSbmStepEvents) +
                                              " collisions in one step");
    if (flags & ks::FLAG_PACK_WIDTH) {
        ctx->pack_keys = false;
        drop_graphs(ctx);
    }
    if (flags & ks::FLAG_SORT_BITS) {
        ctx->sort_passes = std::max(ctx->sort_passes, passes_for_bits(c.grid.bits));
        drop_graphs(ctx);
    }
    if (c.refined > static_cast<unsigned long long>(ctx->b.surv_cap) &&
        (rc = ensure_survivors(ctx, static_cast<int64_t>(c.refined) * 2)))
        return rc;
    if (ks::items_total(c) > ctx->b.items_cap && (rc = ensure_items(ctx, ks::items_total(c) * 3 / 2 + 1024))) return rc;
    if ((ch.flags & ks::FLAG_CONJ_OVERFLOW) && (rc = ensure_conj(ctx, static_cast<int64_t>(ch.conj_count) * 2 + 1024)))
        return rc;
    return KS_OK;
}

// Buffer sizes and graph shape of a chunk of k_steps steps with fragmentation
// on the host: the plan of plan_records.
int plan_chunk(ks_ctx* ctx, int k_steps) { return plan_records(ctx, k_steps); }

int run_chunk(ks_ctx* ctx, int k_steps) {
    if (ctx->dev_sbm) return run_chunk_dev(ctx, k_steps);
    const HostClock::time_point h0 = HostClock::now();
    stash_pending(ctx);  // this chunk's records land in h_conj
    int rc = ensure_chunk(ctx, k_steps);
    if (rc) return rc;
    double t_end = 0.0;
    fill_params(ctx, k_steps, ctx->t, ctx->steps_done, &t_end);  // uploaded by the chunk itself
    if ((rc = plan_chunk(ctx, k_steps))) return rc;
    const bool use_graph = ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph;
    // A new graph is built before the chunk's start is recorded, so that the
    // chunk's device time holds no wait for the host.
    if ((rc = ensure_graph(ctx, k_steps))) return rc;
    if (ctx->profiling) KS_CUDA(cudaEventRecord(ctx->ev_chunk[0], ctx->stream));
    if (ctx->screening) {
        rc = save_checkpoint(ctx, k_steps);
        if (rc) return rc;
    }
    int64_t have = 0;  // leading records of this chunk's run already in h_conj
    for (int attempt = 0;; ++attempt) {
        const HostClock::time_point hl = HostClock::now();
        if (attempt == 0) ctx->timing.host_prep_ms += host_ms(h0, hl);
        rc = launch_chunk(ctx, k_steps);
        if (rc) return rc;
        const HostClock::time_point hs = HostClock::now();
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->timing.host_launch_ms += host_ms(hl, hs);
        ctx->timing.host_sync_ms += host_ms(hs, HostClock::now());
        have = use_graph ? ctx->graph_spec[ctx->cur] : ctx->chunk_spec;
        int flags = ctx->h_chunk->flags;
        unsigned long long max_refined = 0;
        int max_bits = 0;
        int64_t max_items = 0;
        for (int k = 0; k < k_steps; ++k) {
            flags |= ctx->h_ctrl[k].flags;
            max_refined = std::max(max_refined, ctx->h_ctrl[k].refined);
            max_bits = std::max(max_bits, ctx->h_ctrl[k].grid.bits);
            max_items = std::max(max_items, ks::items_total(ctx->h_ctrl[k]));
        }
        const bool surv_over = max_refined > static_cast<unsigned long long>(ctx->b.surv_cap);
        const bool items_over = max_items > ctx->b.items_cap;
        if (flags & ks::FLAG_KEY_RANGE) return fail(ctx, KS_ERR_RANGE, "cell key outside its grid bounds or wider than 63 bits");
        if (flags & ks::FLAG_TIMEOUT) {
            // The chunk's results are void: put the simulation back at the
            // chunk's start, so that the caller may simply run it again.
            if (ctx->screening) restore_checkpoint(ctx);
            return fail(ctx, KS_ERR_TIMEOUT, "radix sort look-back or grid barrier wait gave up");
        }
        if (!(flags & (ks::FLAG_CONJ_OVERFLOW | ks::FLAG_SORT_BITS | ks::FLAG_PACK_WIDTH)) && !surv_over && !items_over)
            break;
        if (attempt >= kMaxReplays) return fail(ctx, KS_ERR_OVERFLOW, "device buffers still overflowing after replays");
        if (flags & ks::FLAG_PACK_WIDTH) {
            ctx->pack_keys = false;  // keys too wide to carry the object index: sort it separately
            drop_graphs(ctx);
        }
        if (flags & ks::FLAG_SORT_BITS) {
            ctx->sort_passes = std::max(ctx->sort_passes, passes_for_bits(max_bits));
            drop_graphs(ctx);
        }
        if (surv_over && (rc = ensure_survivors(ctx, static_cast<int64_t>(max_refined) * 2))) return rc;
        if (items_over && (rc = ensure_items(ctx, max_items * 3 / 2 + 1024))) return rc;
        if ((flags & ks::FLAG_CONJ_OVERFLOW) &&
            (rc = ensure_conj(ctx, static_cast<int64_t>(ctx->h_chunk->conj_count) * 2)))
            return rc;
        rc = restore_checkpoint(ctx);
        if (rc) return rc;
        continue;
    }
    int64_t nc = 0;
    bool was_cut = false;
    for (int cut = 0;; ++cut) {
        nc = static_cast<int64_t>(ctx->h_chunk->conj_count);
        if (ctx->h_chunk->flags & ks::FLAG_CONJ_LARGE) {
            // More records than the one-block ordering takes: the multi-block sort.
            ks::launch_conj_sort(ctx->b, ctx->b.chunk, &ctx->b.params[0].t0, k_steps * ctx->dt, false, ctx->stream);
            KS_CUDA(cudaMemcpyAsync(ctx->h_chunk, ctx->b.chunk, sizeof(ks::ChunkCtrl), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            KS_CUDA(cudaStreamSynchronize(ctx->stream));
            if (ctx->h_chunk->flags & ks::FLAG_TIMEOUT) return fail(ctx, KS_ERR_TIMEOUT, "radix sort look-back or grid barrier wait gave up");
            have = 0;
        }
        if (nc > have) {
            // Records already ordered by TCA on the device (conj_sorted).
            KS_CUDA(cudaMemcpyAsync(ctx->h_conj + have, ctx->b.conj_sorted + have, sizeof(ks_conjunction) * (nc - have),
                                    cudaMemcpyDeviceToHost, ctx->stream));
            KS_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        if (!ctx->bk.on || nc == 0) break;
        int64_t first_hit = -1;
        for (int64_t q = 0; q < nc; ++q)
            if (ctx->h_conj[q].collision && (first_hit < 0 || ctx->h_conj[q].step < first_hit)) first_hit = ctx->h_conj[q].step;
        if (first_hit < 0 || first_hit - ctx->steps_done >= k_steps - 1) break;
        if (cut > 0) return fail(ctx, KS_ERR_STATE, "replay to the first collision step did not end there");
        // Replay the chunk up to the step of the first collision (same inputs, same results).
        k_steps = static_cast<int>(first_hit - ctx->steps_done) + 1;
        was_cut = true;
        fill_params(ctx, k_steps, ctx->t, ctx->steps_done, &t_end);
        rc = restore_checkpoint(ctx);
        if (rc) return rc;
        rc = launch_chunk(ctx, k_steps);
        if (rc) return rc;
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        have = ctx->steps_per_graph > 0 && k_steps == ctx->steps_per_graph ? ctx->graph_spec[ctx->cur] : ctx->chunk_spec;
        if (ctx->h_chunk->flags & (ks::FLAG_CONJ_OVERFLOW | ks::FLAG_TIMEOUT | ks::FLAG_KEY_RANGE))
            return fail(ctx, KS_ERR_STATE, "replay to the first collision step overflowed");
    }
    std::vector<ks_conjunction> hits;
    const double t_last = ctx->h_params[k_steps - 1].t0;
    if (nc > 0) {
        // The device ordered the records by (t, i, j), ties of its key included,
        // unless a run of ties was longer than it takes.
        if (ctx->h_chunk->flags & ks::FLAG_CONJ_TIES) finish_order(ctx->h_conj, ctx->h_conj + nc);
        ctx->pend_begin = 0;
        ctx->pend_end = nc;
        if (ctx->bk.on)
            for (int64_t q = 0; q < nc; ++q)
                if (ctx->h_conj[q].collision) hits.push_back(ctx->h_conj[q]);
    }
    for (int k = 0; k < k_steps; ++k) {
        const Ctrl& c = ctx->h_ctrl[k];
        ks_step_stats st{};
        st.step = ctx->steps_done + k;
        st.candidate_pairs = static_cast<int64_t>(c.candidates);
        st.refined_pairs = static_cast<int64_t>(c.refined);
        st.co_orbiting = static_cast<int64_t>(c.co_orbiting);
        st.conjunctions = static_cast<int64_t>(c.conj);
        st.cell_km = ctx->screening ? c.grid.cell : 0.0;
        st.max_cell_objects = c.max_cell;
        st.alive = c.n_alive;
        ctx->stats_out.push_back(st);
        ctx->max_step_conj = std::max(ctx->max_step_conj, static_cast<int64_t>(c.conj));
        ctx->timing.object_steps += static_cast<int64_t>(c.object_steps);
        ctx->timing.candidate_pairs += static_cast<int64_t>(c.candidates);
        ctx->timing.exact_filter_pairs += static_cast<int64_t>(c.exact_evals);
        ctx->timing.refined_pairs += static_cast<int64_t>(c.refined);
    }
    accumulate_timing(ctx, k_steps);
    ctx->timing.steps += k_steps;
    ctx->timing.sort_passes = ctx->sort_passes;
    ctx->timing.sort_cells_fused = fused_form(ctx);
    ctx->steps_done += k_steps;
    ctx->t = t_end;
    if (k_steps & 1) ctx->cur ^= 1;
    // Chunk length after collisions: as long as the one that ended early, then
    // doubling back while chunks run through.
    if (was_cut) ctx->chunk_hint = k_steps;
    else if (ctx->chunk_hint > 0) ctx->chunk_hint = 2 * ctx->chunk_hint >= ctx->max_chunk ? 0 : 2 * ctx->chunk_hint;
    if (!hits.empty()) return apply_collisions(ctx, ctx->steps_done - 1, t_last, hits);
    return KS_OK;
}

int seed_speculation(ks_ctx* ctx) {
    ks::launch_seed_ctrl(ctx->b, static_cast<int>(ctx->n), ctx->cur, carry_slot(ctx), 1, ctx->stream);
    Ctrl c{};
    KS_CUDA(cudaMemcpyAsync(&c, carry_slot(ctx), sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    const int bits = estimate_bits(c, ctx->dt, ctx->thr, ctx->tune.subcell_bits, ctx->rbits, ctx->tune.cell_scale);
    const int passes = passes_for_bits(bits);
    // Keys, dead flag and object index in 64 bits, with 2 bits to spare for the estimate.
    const int64_t indices = ctx->dev_sbm ? ctx->b.cap : ctx->n;  // fragments take indices up to the capacity
    const bool pack = ctx->allow_pack && bits + 1 + index_bits(indices) + 2 <= 64;
    // The chunk graphs hold both in their kernels' arguments: rebuilt only if they change.
    if (passes != ctx->sort_passes || pack != ctx->pack_keys) drop_graphs(ctx);
    ctx->sort_passes = passes;
    ctx->pack_keys = pack;
    return KS_OK;
}

// Device fragmentation: live count, masses (unknown), area-to-mass ratios,
// provenance and event counters of a freshly uploaded population.
int init_device_fragmentation(ks_ctx* ctx, bool single_population) {
    if (!ctx->dev_sbm) return KS_OK;
    ks::DeviceBuffers& b = ctx->b;
    const int n = static_cast<int>(ctx->n);
    KS_CUDA(cudaMemcpyAsync(b.n_live, &n, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    KS_CUDA(cudaMemsetAsync(b.mass_kg, 0, sizeof(double) * b.cap, ctx->stream));
    KS_CUDA(cudaMemsetAsync(b.a2m, 0, sizeof(double) * b.cap, ctx->stream));
    KS_CUDA(cudaMemsetAsync(b.event_of, 0xFF, sizeof(int32_t) * b.cap, ctx->stream));
    KS_CUDA(cudaMemsetAsync(b.sbm_next_event, 0, sizeof(int) * 65536, ctx->stream));
    if (single_population) KS_CUDA(cudaMemsetAsync(b.real_id, 0, sizeof(uint16_t) * b.cap, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->dev_stalls = 0;
    return KS_OK;
}

int upload_population(ks_ctx* ctx, int64_t n, const double* states, const double* size_m, const uint8_t* alive,
                      int buf) {
    ks::DeviceBuffers& b = ctx->b;
    if (n > 0) {
        KS_CUDA(cudaMemcpyAsync(b.state[buf], states, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, ctx->stream));
        if (alive) KS_CUDA(cudaMemcpyAsync(b.alive[buf], alive, n, cudaMemcpyHostToDevice, ctx->stream));
        else KS_CUDA(cudaMemsetAsync(b.alive[buf], 1, n, ctx->stream));
        if (size_m) KS_CUDA(cudaMemcpyAsync(b.size_m, size_m, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    }
    KS_CUDA(cudaGetLastError());
    return KS_OK;
}

// ---------------------------------------------------------------------------
// Fragmentation between steps (NASA SBM on the host, fragments' sub-step on
// the device)
// ---------------------------------------------------------------------------

void reset_breakup_run(ks_ctx* ctx) {
    ctx->chunk_hint = 0;
    ks_ctx::Breakup& k = ctx->bk;
    k.rng.clear();
    k.next_event.clear();
    k.out.clear();
    k.mirrors = false;
    k.size_m.clear();
    k.mass_kg.clear();
    k.area_to_mass.clear();
    k.event.clear();
    k.rid.clear();
}

// Host copies of the per-object properties fragmentation reads.
int ensure_mirrors(ks_ctx* ctx) {
    ks_ctx::Breakup& k = ctx->bk;
    if (k.mirrors) return KS_OK;
    const size_t n = static_cast<size_t>(ctx->n);
    k.size_m.assign(n, 0.0);
    k.mass_kg.assign(n, 0.0);
    k.area_to_mass.assign(n, 0.0);
    k.event.assign(n, -1);
    k.rid.assign(n, 0);
    if (n > 0) {
        KS_CUDA(cudaMemcpyAsync(k.size_m.data(), ctx->b.size_m, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        if (ctx->rbits > 0)
            KS_CUDA(cudaMemcpyAsync(k.rid.data(), ctx->b.real_id, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    k.mirrors = true;
    return KS_OK;
}

// One random stream per realisation, seeded seed + realisation.
void ensure_streams(ks_ctx* ctx) {
    ks_ctx::Breakup& k = ctx->bk;
    while (static_cast<int>(k.rng.size()) < ctx->realisations) {
        k.rng.emplace_back(k.seed + static_cast<uint64_t>(k.rng.size()));
        k.next_event.push_back(0);
    }
}

// Grows the object arrays to hold `want` objects, keeping the current states,
// alive flags, sizes and realisation ids.
int grow_objects(ks_ctx* ctx, int64_t want) {
    ks::DeviceBuffers& b = ctx->b;
    if (want <= b.cap) return KS_OK;
    const int64_t n = ctx->n;
    const int64_t cap = std::max<int64_t>(want, b.cap + b.cap / 2 + 1024);
    double *st = nullptr, *sz = nullptr;
    uint8_t* al = nullptr;
    uint16_t* rid = nullptr;
    if (n > 0) {
        KS_CUDA(cudaMalloc(&st, sizeof(double) * 6 * n));
        KS_CUDA(cudaMalloc(&sz, sizeof(double) * n));
        KS_CUDA(cudaMalloc(&al, n));
        KS_CUDA(cudaMalloc(&rid, sizeof(uint16_t) * n));
        KS_CUDA(cudaMemcpyAsync(st, b.state[ctx->cur], sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(sz, b.size_m, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(al, b.alive[ctx->cur], n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(rid, b.real_id, sizeof(uint16_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    int rc = ensure_objects(ctx, cap);
    if (!rc && n > 0) {
        KS_CUDA(cudaMemcpyAsync(b.state[ctx->cur], st, sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.size_m, sz, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.alive[ctx->cur], al, n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.real_id, rid, sizeof(uint16_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    dfree(st);
    dfree(sz);
    dfree(al);
    dfree(rid);
    return rc;
}

struct NewFragments {
    std::vector<ks::SbmFragment> rows;
    std::vector<uint16_t> rid;
    std::vector<int32_t> event;
    struct Span {
        int64_t first;
        int count;
        double remaining_s;  // time from the event to the end of its step
        double jd0;          // Julian date of the event
    };
    std::vector<Span> spans;
    std::vector<int64_t> killed;
};

int ensure_frag_scratch(ks_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->frag_scratch_bytes) return KS_OK;
    if (ctx->frag_scratch) cudaFree(ctx->frag_scratch);
    ctx->frag_scratch = nullptr;
    ctx->frag_scratch_bytes = 0;
    const size_t want = std::max(bytes, size_t(1) << 20);
    KS_CUDA(cudaMalloc(&ctx->frag_scratch, want));
    ctx->frag_scratch_bytes = want;
    return KS_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Appends the fragments after the population, carries those born inside a
// step to its end (one device launch for all events), and removes the
// destroyed parents.
int commit_fragments(ks_ctx* ctx, const NewFragments& nf) {
    ks::DeviceBuffers& b = ctx->b;
    const int64_t n0 = ctx->n;
    const int64_t m = static_cast<int64_t>(nf.rows.size());
    int rc = grow_objects(ctx, n0 + m);
    if (rc) return rc;
    const size_t ns = nf.spans.size(), nk = nf.killed.size();
    const size_t bytes = align256(sizeof(ks::FragSpan) * std::max<size_t>(ns, 1)) +
                         align256(sizeof(int) * std::max<int64_t>(m, 1)) + align256(sizeof(int64_t) * std::max<size_t>(nk, 1));
    rc = ensure_frag_scratch(ctx, bytes);
    if (rc) return rc;
    char* base = static_cast<char*>(ctx->frag_scratch);
    ks::FragSpan* d_spans = reinterpret_cast<ks::FragSpan*>(base);
    int* d_row_span = reinterpret_cast<int*>(base + align256(sizeof(ks::FragSpan) * std::max<size_t>(ns, 1)));
    int64_t* d_killed = reinterpret_cast<int64_t*>(reinterpret_cast<char*>(d_row_span) +
                                                   align256(sizeof(int) * std::max<int64_t>(m, 1)));
    if (m > 0) {
        std::vector<double> st(static_cast<size_t>(6 * m)), sz(static_cast<size_t>(m));
        for (int64_t q = 0; q < m; ++q) {
            const ks::SbmFragment& f = nf.rows[static_cast<size_t>(q)];
            std::copy(f.s, f.s + 6, &st[static_cast<size_t>(6 * q)]);
            sz[static_cast<size_t>(q)] = f.size_m;
        }
        std::vector<ks::FragSpan> spans(ns);
        std::vector<int> row_span(static_cast<size_t>(m), 0);
        for (size_t k = 0; k < ns; ++k) {
            const NewFragments::Span& sp = nf.spans[k];
            spans[k].dt = sp.remaining_s > 0 ? sp.remaining_s : 0.0;
            if (sp.remaining_s > 0 && sp.count > 0) ks::moon_stages_from(sp.jd0, sp.remaining_s, spans[k].m);
            for (int q = 0; q < sp.count; ++q) row_span[static_cast<size_t>(sp.first - n0 + q)] = static_cast<int>(k);
        }
        KS_CUDA(cudaMemcpyAsync(b.state[ctx->cur] + 6 * n0, st.data(), sizeof(double) * 6 * m, cudaMemcpyHostToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.size_m + n0, sz.data(), sizeof(double) * m, cudaMemcpyHostToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(b.real_id + n0, nf.rid.data(), sizeof(uint16_t) * m, cudaMemcpyHostToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(d_spans, spans.data(), sizeof(ks::FragSpan) * ns, cudaMemcpyHostToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(d_row_span, row_span.data(), sizeof(int) * m, cudaMemcpyHostToDevice, ctx->stream));
        ks::launch_advance_spans(force_consts(), d_spans, d_row_span, n0, static_cast<int>(m), b.state[ctx->cur],
                                 b.alive[ctx->cur], ctx->stream);
    }
    if (nk > 0) {
        KS_CUDA(cudaMemcpyAsync(d_killed, nf.killed.data(), sizeof(int64_t) * nk, cudaMemcpyHostToDevice, ctx->stream));
        ks::launch_clear_alive(b.alive[ctx->cur], d_killed, static_cast<int>(nk), ctx->stream);
    }
    KS_CUDA(cudaGetLastError());
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    ks_ctx::Breakup& k = ctx->bk;
    for (int64_t q = 0; q < m; ++q) {
        const ks::SbmFragment& f = nf.rows[static_cast<size_t>(q)];
        k.size_m.push_back(f.size_m);
        k.mass_kg.push_back(f.mass_kg);
        k.area_to_mass.push_back(f.area_to_mass);
        k.event.push_back(nf.event[static_cast<size_t>(q)]);
        k.rid.push_back(nf.rid[static_cast<size_t>(q)]);
    }
    ctx->n = n0 + m;
    return seed_speculation(ctx);
}

// Fragments the collisions of the step that started at t0 (src/core/breakup.cpp:316-338):
// in (t, i, j) order, skipping pairs with a parent destroyed earlier in the
// step; parents are interpolated to the collision instant. Realisations draw
// from their own streams and own their objects, so they are fragmented in
// parallel; fragments are appended in the order of the collisions.
int apply_collisions(ks_ctx* ctx, int64_t step, double t0, const std::vector<ks_conjunction>& hits) {
    int rc = ensure_mirrors(ctx);
    if (rc) return rc;
    ensure_streams(ctx);
    ks_ctx::Breakup& k = ctx->bk;
    const double dt = ctx->dt;
    // Start- and end-of-step states of every parent, in one gather.
    std::vector<int64_t> idx;
    idx.reserve(2 * hits.size());
    for (const ks_conjunction& c : hits) {
        idx.push_back(c.i);
        idx.push_back(c.j);
    }
    std::sort(idx.begin(), idx.end());
    idx.erase(std::unique(idx.begin(), idx.end()), idx.end());
    const size_t u = idx.size();
    rc = ensure_frag_scratch(ctx, align256(sizeof(int64_t) * u) + sizeof(double) * 12 * u);
    if (rc) return rc;
    int64_t* d_idx = static_cast<int64_t*>(ctx->frag_scratch);
    double* d_rows = reinterpret_cast<double*>(static_cast<char*>(ctx->frag_scratch) + align256(sizeof(int64_t) * u));
    std::vector<double> rows(12 * u);
    KS_CUDA(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int64_t) * u, cudaMemcpyHostToDevice, ctx->stream));
    ks::launch_gather_rows(ctx->b.state[ctx->cur ^ 1], ctx->b.state[ctx->cur], d_idx, static_cast<int>(u), d_rows,
                           ctx->stream);
    KS_CUDA(cudaMemcpyAsync(rows.data(), d_rows, sizeof(double) * 12 * u, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    auto row_of = [&](int64_t o) {
        return &rows[12 * static_cast<size_t>(std::lower_bound(idx.begin(), idx.end(), o) - idx.begin())];
    };

    struct Result {
        bool done = false;
        ks_breakup_event ev{};
        std::vector<ks::SbmFragment> frags;
        ks::SbmOutcome oc;
        double remaining = 0, jd0 = 0;
    };
    std::vector<Result> res(hits.size());
    std::vector<std::vector<size_t>> by_real(static_cast<size_t>(ctx->realisations));
    for (size_t h = 0; h < hits.size(); ++h) by_real[k.rid[static_cast<size_t>(hits[h].i)]].push_back(h);
    auto fragment_realisation = [&](size_t r) {
        std::set<int64_t> dead;
        for (size_t h : by_real[r]) {
            const ks_conjunction& c = hits[h];
            if (dead.count(c.i) || dead.count(c.j)) continue;
            const double s = (c.t - t0) / dt;
            auto parent = [&](int64_t o) {
                const double* rw = row_of(o);
                ks::SbmParent p;
                p.index = o;
                ks::interpolate_state(rw, rw + 6, dt, s, p.s);
                p.mass_kg = ks::sbm_mass_or_default(k.mass_kg[static_cast<size_t>(o)]);
                p.size_m = k.size_m[static_cast<size_t>(o)];
                return p;
            };
            const ks::SbmParent pa = parent(c.i), pb = parent(c.j);
            const bool a_heavier = pa.mass_kg >= pb.mass_kg;
            const ks::SbmParent& tgt = a_heavier ? pa : pb;
            const ks::SbmParent& prj = a_heavier ? pb : pa;
            Result& out = res[h];
            out.ev.step = step;
            out.ev.id = k.next_event[r]++;
            out.ev.realisation = static_cast<int32_t>(r);
            out.ev.target = tgt.index;
            out.ev.projectile = prj.index;
            ks::sbm_fragment(k.rng[r], k.params, tgt, prj, c.t, out.ev, out.frags, out.oc);
            if (out.oc.kill_projectile) dead.insert(prj.index);
            if (out.oc.kill_target) dead.insert(tgt.index);
            if (out.oc.reduce_target) k.mass_kg[static_cast<size_t>(tgt.index)] = out.oc.target_mass_after;
            out.remaining = t0 + dt - c.t;
            out.jd0 = ctx->epoch_jd + c.t / 86400.0;
            out.done = true;
        }
    };
    std::vector<size_t> active;
    for (size_t r = 0; r < by_real.size(); ++r)
        if (!by_real[r].empty()) active.push_back(r);
    const size_t workers = std::min<size_t>(active.size(), std::max(1u, std::thread::hardware_concurrency()));
    if (workers <= 1) {
        for (size_t r : active) fragment_realisation(r);
    } else {
        std::atomic<size_t> next{0};
        std::vector<std::thread> pool;
        for (size_t w = 0; w < workers; ++w)
            pool.emplace_back([&]() {
                for (size_t q = next++; q < active.size(); q = next++) fragment_realisation(active[q]);
            });
        for (std::thread& th : pool) th.join();
    }

    NewFragments nf;
    for (size_t h = 0; h < hits.size(); ++h) {
        Result& out = res[h];
        if (!out.done) continue;
        out.ev.first_fragment = ctx->n + static_cast<int64_t>(nf.rows.size());
        if (out.oc.kill_projectile) nf.killed.push_back(out.ev.projectile);
        if (out.oc.kill_target) nf.killed.push_back(out.ev.target);
        nf.spans.push_back({out.ev.first_fragment, out.ev.fragments, out.remaining, out.jd0});
        nf.rows.insert(nf.rows.end(), out.frags.begin(), out.frags.end());
        nf.rid.resize(nf.rows.size(), static_cast<uint16_t>(out.ev.realisation));
        nf.event.resize(nf.rows.size(), out.ev.id);
        k.out.push_back(out.ev);
    }
    return commit_fragments(ctx, nf);
}

}  // namespace

namespace {

// Population file: header, then per-object arrays, then the fragmentation
// streams (Mersenne Twister state as the C++ standard library prints it).
constexpr char kPopMagic[8] = {'K', 'S', 'P', 'O', 'P', 'v', '1', '\0'};

struct PopHeader {
    char magic[8];
    int64_t n;
    int32_t realisations, streams;
    double epoch_jd, t, dt;
    int64_t steps_done;
    int32_t breakup_on, pad;
    double lc_m, catastrophic_j_per_g;
    uint64_t seed;
};

template <typename T>
bool put(std::ofstream& f, const T* p, size_t count) {
    f.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(sizeof(T) * count));
    return static_cast<bool>(f);
}
template <typename T>
bool get(std::ifstream& f, T* p, size_t count) {
    f.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(sizeof(T) * count));
    return static_cast<bool>(f);
}

}  // namespace

extern "C" {

int ks_create(int device, ks_ctx** out) {
    if (!out) return KS_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return KS_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return KS_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return KS_ERR_NO_DEVICE;
    ks_ctx* ctx = new ks_ctx;
    ctx->device = device;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    char buf[640];
    std::snprintf(buf, sizeof(buf), "%s (sm_%d%d, %d SMs, %.1f GiB)", prop.name, prop.major, prop.minor,
                  prop.multiProcessorCount, prop.totalGlobalMem / 1073741824.0);
    ctx->name = buf;
    int rc = KS_OK;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->b.chunk, sizeof(ks::ChunkCtrl)) != cudaSuccess ||
        cudaHostAlloc(&ctx->h_chunk, sizeof(ks::ChunkCtrl), cudaHostAllocDefault) != cudaSuccess)
        rc = KS_ERR_CUDA;
    if (!rc) rc = ensure_chunk(ctx, 64);
    if (!rc) rc = ensure_survivors(ctx, 1 << 20);
    if (!rc) rc = ensure_items(ctx, 1 << 18);
    if (!rc) rc = ensure_conj(ctx, 1 << 16);
    if (rc) {
        ks_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return KS_OK;
}

void ks_destroy(ks_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
    free_objects(ctx);
    if (ctx->l2_flush) cudaFree(ctx->l2_flush);
    dfree(ctx->b.survivors);
    dfree(ctx->b.items);
    if (ctx->frag_scratch) cudaFree(ctx->frag_scratch);
    free_conj(ctx);
    dfree(ctx->b.ctrl);
    dfree(ctx->b.chunk);
    dfree(ctx->b.params);
    if (ctx->h_params) cudaFreeHost(ctx->h_params);
    if (ctx->h_ctrl) cudaFreeHost(ctx->h_ctrl);
    if (ctx->h_chunk) cudaFreeHost(ctx->h_chunk);
    if (ctx->h_conj) cudaFreeHost(ctx->h_conj);
    for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->ev_chunk) if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* ks_last_error(const ks_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
const char* ks_device_name(const ks_ctx* ctx) { return ctx ? ctx->name.c_str() : ""; }
void* ks_stream(ks_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int ks_set_population(ks_ctx* ctx, int64_t n, const double* states, const double* size_m, const uint8_t* alive) {
    if (!ctx || n < 0 || (n > 0 && (!states || !size_m))) return fail(ctx, KS_ERR_ARG, "ks_set_population: bad arguments");
    cudaSetDevice(ctx->device);
    const int old_rbits = ctx->rbits;
    ctx->realisations = 1;
    ctx->rbits = 0;
    ctx->offsets.assign({0, n});
    reset_breakup_run(ctx);
    int rc = ensure_objects(ctx, n);
    if (rc) return rc;
    if (n != ctx->n || old_rbits != 0) drop_graphs(ctx);  // graphs hold the population size in their arguments
    ctx->n = n;
    ctx->cur = 0;
    rc = upload_population(ctx, n, states, size_m, alive, 0);
    if (rc) return rc;
    if ((rc = init_device_fragmentation(ctx, true))) return rc;
    rc = seed_speculation(ctx);
    if (rc) return rc;
    ctx->has_pop = true;
    ctx->steps_done = 0;
    clear_records(ctx);
    ctx->stats_out.clear();
    return KS_OK;
}

int ks_set_population_batch(ks_ctx* ctx, int32_t realisations, const int64_t* offsets, const double* states,
                            const double* size_m, const uint8_t* alive) {
    if (!ctx || realisations < 1 || realisations > 65535 || !offsets || offsets[0] != 0)
        return fail(ctx, KS_ERR_ARG, "ks_set_population_batch: bad arguments");
    for (int r = 0; r < realisations; ++r)
        if (offsets[r + 1] < offsets[r]) return fail(ctx, KS_ERR_ARG, "ks_set_population_batch: offsets must not decrease");
    const int64_t n = offsets[realisations];
    if (n > 0 && (!states || !size_m)) return fail(ctx, KS_ERR_ARG, "ks_set_population_batch: bad arguments");
    cudaSetDevice(ctx->device);
    int rc = ensure_objects(ctx, n);
    if (rc) return rc;
    std::vector<uint16_t> rid(static_cast<size_t>(n));
    for (int r = 0; r < realisations; ++r)
        for (int64_t i = offsets[r]; i < offsets[r + 1]; ++i) rid[static_cast<size_t>(i)] = static_cast<uint16_t>(r);
    if (n > 0) KS_CUDA(cudaMemcpy(ctx->b.real_id, rid.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice));
    int rbits = 0;
    while ((1 << rbits) < realisations) ++rbits;
    ctx->realisations = realisations;
    ctx->rbits = rbits;
    ctx->offsets.assign(offsets, offsets + realisations + 1);
    reset_breakup_run(ctx);
    ctx->n = n;
    ctx->cur = 0;
    drop_graphs(ctx);
    rc = upload_population(ctx, n, states, size_m, alive, 0);
    if (rc) return rc;
    if ((rc = init_device_fragmentation(ctx, false))) return rc;
    rc = seed_speculation(ctx);
    if (rc) return rc;
    ctx->has_pop = true;
    ctx->steps_done = 0;
    clear_records(ctx);
    ctx->stats_out.clear();
    return KS_OK;
}

int ks_get_population(ks_ctx* ctx, int64_t n, double* states, uint8_t* alive) {
    if (!ctx) return KS_ERR_ARG;
    if (!ctx->has_pop) return fail(ctx, KS_ERR_STATE, "no resident population");
    if (n != ctx->n) return fail(ctx, KS_ERR_ARG, "ks_get_population: size mismatch");
    cudaSetDevice(ctx->device);
    ks::DeviceBuffers& b = ctx->b;
    if (n > 0) {
        if (states)
            KS_CUDA(cudaMemcpyAsync(states, b.state[ctx->cur], sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, ctx->stream));
        if (alive) KS_CUDA(cudaMemcpyAsync(alive, b.alive[ctx->cur], n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    return KS_OK;
}

int64_t ks_population_size(const ks_ctx* ctx) { return ctx ? ctx->n : -1; }

int ks_set_clock(ks_ctx* ctx, double epoch_jd, double t, double dt) {
    if (!ctx || !(dt > 0.0)) return fail(ctx, KS_ERR_ARG, "ks_set_clock: dt must be positive");
    if (dt != ctx->dt) drop_graphs(ctx);
    ctx->epoch_jd = epoch_jd;
    ctx->t = t;
    ctx->dt = dt;
    if (ctx->has_pop) {
        cudaSetDevice(ctx->device);
        return seed_speculation(ctx);
    }
    return KS_OK;
}

int ks_get_clock(const ks_ctx* ctx, double* t, int64_t* steps_done) {
    if (!ctx) return KS_ERR_ARG;
    if (t) *t = ctx->t;
    if (steps_done) *steps_done = ctx->steps_done;
    return KS_OK;
}

int ks_set_screening(ks_ctx* ctx, int enabled, double threshold_km, double radius_scale,
                     double min_encounter_speed_km_s) {
    if (!ctx || threshold_km < 0.0 || radius_scale < 0.0 || min_encounter_speed_km_s < 0.0)
        return fail(ctx, KS_ERR_ARG, "ks_set_screening: bad arguments");
    drop_graphs(ctx);
    ctx->screening = enabled ? 1 : 0;
    ctx->thr = threshold_km;
    ctx->rscale = radius_scale;
    ctx->vmin = min_encounter_speed_km_s;
    if (ctx->has_pop) {
        cudaSetDevice(ctx->device);
        return seed_speculation(ctx);
    }
    return KS_OK;
}

int ks_set_precision(ks_ctx* ctx, int precision) {
    if (!ctx || (precision != KS_PRECISION_FP64 && precision != KS_PRECISION_SPLIT))
        return fail(ctx, KS_ERR_ARG, "ks_set_precision: unknown mode");
    drop_graphs(ctx);
    ctx->precision = precision;
    return KS_OK;
}

int ks_set_steps_per_graph(ks_ctx* ctx, int steps_per_graph) {
    if (!ctx || steps_per_graph < 0 || steps_per_graph > 4096) return fail(ctx, KS_ERR_ARG, "ks_set_steps_per_graph: 0..4096");
    drop_graphs(ctx);
    ctx->steps_per_graph = steps_per_graph;
    return KS_OK;
}

int ks_set_buffer_limits(ks_ctx* ctx, int64_t survivor_pairs, int64_t conjunctions) {
    if (!ctx || survivor_pairs < 0 || conjunctions < 0) return fail(ctx, KS_ERR_ARG, "ks_set_buffer_limits: bad arguments");
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    if (survivor_pairs > 0) {
        dfree(ctx->b.survivors);
        ctx->b.surv_cap = 0;
        int rc = ensure_survivors(ctx, survivor_pairs);
        if (rc) return rc;
    }
    if (conjunctions > 0) {
        free_conj(ctx);
        int rc = ensure_conj(ctx, conjunctions);
        if (rc) return rc;
    }
    return KS_OK;
}

int ks_set_tuning(ks_ctx* ctx, const char* key, int64_t value) {
    if (!ctx || !key) return KS_ERR_ARG;
    const std::string k(key);
    if (k == "pair_variant" && value >= 0 && value <= 2) ctx->tune.pair_variant = static_cast<int>(value);
    else if (k == "pair_blocks_per_sm" && value >= 0 && value <= 32) ctx->tune.pair_blocks_per_sm = static_cast<int>(value);
    else if (k == "subcell_bits" && value >= 0 && value <= 3) {
        ctx->tune.subcell_bits = static_cast<int>(value);
        if (ctx->has_pop) {
            drop_graphs(ctx);
            return seed_speculation(ctx);
        }
    } else if (k == "box_min_rows" && value >= 0 && value <= 33) ctx->tune.box_min_rows = static_cast<int>(value);
    else if (k == "prop_block" && value >= 32 && value <= 128 && value % 32 == 0) ctx->tune.prop_block = static_cast<int>(value);
    else if (k == "item_col_blocks" && value >= 1 && value <= 64) ctx->tune.item_col_blocks = static_cast<int>(value);
    else if (k == "pair_gate_x2" && (value == 0 || value == 1)) ctx->tune.pair_gate_x2 = static_cast<int>(value);
    else if (k == "pair_stage2" && value >= 0 && value <= 2) ctx->tune.pair_stage2 = static_cast<int>(value);
    else if (k == "prop_min_blocks" && value >= 4 && value <= 6) ctx->tune.prop_min_blocks = static_cast<int>(value);
    else if (k == "hash_slots_per_cell" && value >= 0 && value <= 64) {
        ctx->tune.hash_slots_per_cell = static_cast<int>(value);
        drop_graphs(ctx);
    }
    else if (k == "sort_digit_bits" && (value == 8 || value == 11)) {
        ctx->tune.sort_digit_bits = static_cast<int>(value);
        drop_graphs(ctx);
    }
    else if (k == "sort_fused" && (value == 0 || value == 1)) {
        ctx->tune.sort_fused = static_cast<int>(value);
        drop_graphs(ctx);
    }
    else if (k == "sort_rank_ballot" && (value == 0 || value == 1)) {
        ctx->tune.sort_rank_ballot = static_cast<int>(value);
        drop_graphs(ctx);
    }
    else if (k == "lookback_polls" && value >= 0 && value <= (int64_t(1) << 30)) {
        ctx->tune.lookback_polls = static_cast<int>(value);
        drop_graphs(ctx);  // graphs hold the limit in their kernel arguments
    }
    else if (k == "pack_keys" && (value == 0 || value == 1)) {
        ctx->allow_pack = value != 0;
        if (ctx->has_pop) {
            drop_graphs(ctx);
            return seed_speculation(ctx);
        }
    }
    else if (k == "cell_scale_permille" && value >= 1000 && value <= 4000) {
        ctx->tune.cell_scale = static_cast<double>(value) / 1000.0;
        if (ctx->has_pop) {
            drop_graphs(ctx);
            return seed_speculation(ctx);
        }
    }
    else return fail(ctx, KS_ERR_ARG, "ks_set_tuning: unknown key or value out of range: " + k);
    drop_graphs(ctx);
    return KS_OK;
}

namespace {

struct Knobs {
    int spg, pair_variant, pair_bps, subcell, box_rows, cell_permille, prop_block, item_cols;
};

Knobs current_knobs(const ks_ctx* ctx) {
    return Knobs{ctx->steps_per_graph, ctx->tune.pair_variant, ctx->tune.pair_blocks_per_sm, ctx->tune.subcell_bits,
                 ctx->tune.box_min_rows, static_cast<int>(std::lround(ctx->tune.cell_scale * 1000.0)),
                 ctx->tune.prop_block, ctx->tune.item_col_blocks};
}

void put_knobs(ks_ctx* ctx, const Knobs& k, const Ctrl& carry) {
    drop_graphs(ctx);
    ctx->steps_per_graph = k.spg;
    ctx->tune.pair_variant = k.pair_variant;
    ctx->tune.pair_blocks_per_sm = k.pair_bps;
    ctx->tune.subcell_bits = k.subcell;
    ctx->tune.box_min_rows = k.box_rows;
    ctx->tune.cell_scale = k.cell_permille / 1000.0;
    ctx->tune.prop_block = k.prop_block;
    ctx->tune.item_col_blocks = k.item_cols;
    ctx->sort_passes = passes_for_bits(
        estimate_bits(carry, ctx->dt, ctx->thr, ctx->tune.subcell_bits, ctx->rbits, ctx->tune.cell_scale));
}

}  // namespace

int ks_autotune(ks_ctx* ctx, int32_t trial_steps, ks_tuning_choice* out) {
    if (!ctx || trial_steps < 1 || trial_steps > 4096) return fail(ctx, KS_ERR_ARG, "ks_autotune: bad arguments");
    if (!ctx->has_pop) return fail(ctx, KS_ERR_STATE, "ks_autotune: no population");
    if (ctx && ctx->dev_sbm) return fail(ctx, KS_ERR_STATE, "ks_autotune: not available with fragmentation on the device");
    cudaSetDevice(ctx->device);
    static const int kSpg[] = {8, 16, 32, 64};
    int rc = ensure_chunk(ctx, 64);
    if (rc) return rc;
    // Snapshot of everything a trial run changes; restored after every trial
    // and at the end, so tuning leaves the simulation where it was.
    const int64_t n = ctx->n;
    const int cur0 = ctx->cur;
    const int64_t steps0 = ctx->steps_done;
    const double t0 = ctx->t;
    stash_pending(ctx);
    const size_t conj0 = ctx->conj_out.size(), stats0 = ctx->stats_out.size();
    const ks_timing timing0 = ctx->timing;
    const bool breakup0 = ctx->bk.on;
    const int sort_passes0 = ctx->sort_passes;
    const Knobs start = current_knobs(ctx);
    Ctrl carry{};
    KS_CUDA(cudaMemcpy(&carry, carry_slot(ctx), sizeof(Ctrl), cudaMemcpyDeviceToHost));
    double* snap_state = nullptr;
    uint8_t* snap_alive = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        dfree(snap_state);
        dfree(snap_alive);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    if (n > 0) {
        KS_CUDA(cudaMalloc(&snap_state, sizeof(double) * 6 * n));
        KS_CUDA(cudaMalloc(&snap_alive, n));
        KS_CUDA(cudaMemcpyAsync(snap_state, ctx->b.state[cur0], sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(snap_alive, ctx->b.alive[cur0], n, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    KS_CUDA(cudaEventCreate(&e0));
    KS_CUDA(cudaEventCreate(&e1));
    ctx->bk.on = false;

    auto restore = [&]() -> int {
        ctx->cur = cur0;
        ctx->steps_done = steps0;
        ctx->t = t0;
        if (n > 0) {
            KS_CUDA(cudaMemcpyAsync(ctx->b.state[cur0], snap_state, sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, ctx->stream));
            KS_CUDA(cudaMemcpyAsync(ctx->b.alive[cur0], snap_alive, n, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        KS_CUDA(cudaMemcpyAsync(carry_slot(ctx), &carry, sizeof(Ctrl), cudaMemcpyHostToDevice, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->conj_out.resize(conj0);
        ctx->pend_begin = ctx->pend_end = 0;
        ctx->stats_out.resize(stats0);
        return KS_OK;
    };
    auto run_steps = [&](int64_t steps) -> int {
        const int64_t end = ctx->steps_done + steps;
        while (ctx->steps_done < end) {
            const int chunk = ctx->steps_per_graph > 0 ? ctx->steps_per_graph : 64;
            const int r = run_chunk(ctx, static_cast<int>(std::min<int64_t>(end - ctx->steps_done, chunk)));
            if (r) return r;
        }
        return KS_OK;
    };
    int trials = 0;
    // Milliseconds per step of a configuration: one untimed run (graph
    // capture, buffer growth), then the timed run, both from the snapshot.
    auto trial = [&](const Knobs& k, double* ms) -> int {
        put_knobs(ctx, k, carry);
        const int64_t steps = std::max<int64_t>(trial_steps, 2 * std::max(k.spg, 1));
        int r = restore();
        if (!r) r = run_steps(steps);
        if (!r) r = restore();
        if (r) return r;
        KS_CUDA(cudaEventRecord(e0, ctx->stream));
        r = run_steps(steps);
        if (r) return r;
        KS_CUDA(cudaEventRecord(e1, ctx->stream));
        KS_CUDA(cudaEventSynchronize(e1));
        float el = 0.f;
        KS_CUDA(cudaEventElapsedTime(&el, e0, e1));
        *ms = static_cast<double>(el) / static_cast<double>(steps);
        ++trials;
        return KS_OK;
    };

    Knobs best = start;
    double best_ms = 0, first_ms = 0;
    rc = trial(best, &best_ms);
    first_ms = best_ms;
    // Coordinate descent over the knobs; a change must gain 2% to be kept.
    auto consider = [&](Knobs cand) -> int {
        double ms = 0;
        const int r = trial(cand, &ms);
        if (r) return r;
        if (ms < 0.98 * best_ms) {
            best = cand;
            best_ms = ms;
        }
        return KS_OK;
    };
    if (!rc) for (int v : kSpg) if (!rc && v != best.spg) { Knobs c = best; c.spg = v; rc = consider(c); }
    if (ctx->screening) {
        const int pv_bps[][2] = {{1, 0}, {1, 2}, {1, 4}, {0, 0}, {0, 3}, {2, 0}, {2, 3}};
        for (const auto& pb : pv_bps)
            if (!rc && !(pb[0] == best.pair_variant && pb[1] == best.pair_bps)) {
                Knobs c = best;
                c.pair_variant = pb[0];
                c.pair_bps = pb[1];
                rc = consider(c);
            }
        for (int v : {0, 1, 2, 3}) if (!rc && v != best.subcell) { Knobs c = best; c.subcell = v; rc = consider(c); }
        for (int v : {0, 4, 8, 16}) if (!rc && v != best.box_rows) { Knobs c = best; c.box_rows = v; rc = consider(c); }
        for (int v : {1000, 1150, 1300, 1500}) if (!rc && v != best.cell_permille) { Knobs c = best; c.cell_permille = v; rc = consider(c); }
    }
    if (ctx->screening)
        for (int v : {4, 8, 16, 32}) if (!rc && v != best.item_cols) { Knobs c = best; c.item_cols = v; rc = consider(c); }
    for (int v : {64, 96, 128}) if (!rc && v != best.prop_block) { Knobs c = best; c.prop_block = v; rc = consider(c); }

    // Leave the chosen configuration in place and the simulation untouched.
    put_knobs(ctx, rc ? start : best, carry);
    const int rr = restore();
    if (rc) ctx->sort_passes = sort_passes0;
    ctx->timing = timing0;
    ctx->bk.on = breakup0;
    cleanup();
    if (rc) return rc;
    if (rr) return rr;
    if (out) {
        out->steps_per_graph = best.spg;
        out->pair_variant = best.pair_variant;
        out->pair_blocks_per_sm = best.pair_bps;
        out->subcell_bits = best.subcell;
        out->box_min_rows = best.box_rows;
        out->cell_scale_permille = best.cell_permille;
        out->prop_block = best.prop_block;
        out->item_col_blocks = best.item_cols;
        out->trials = trials;
        out->ms_per_step_start = first_ms;
        out->ms_per_step_best = best_ms;
    }
    return KS_OK;
}

int ks_set_l2_flush(ks_ctx* ctx, int64_t bytes) {
    if (!ctx || bytes < 0) return fail(ctx, KS_ERR_ARG, "ks_set_l2_flush: bad arguments");
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    if (ctx->l2_flush) cudaFree(ctx->l2_flush);
    ctx->l2_flush = nullptr;
    ctx->l2_flush_bytes = 0;
    if (bytes > 0) {
        KS_CUDA(cudaMalloc(&ctx->l2_flush, bytes));
        ctx->l2_flush_bytes = bytes;
    }
    return KS_OK;
}

int ks_set_profiling(ks_ctx* ctx, int enabled) {
    if (!ctx) return KS_ERR_ARG;
    drop_graphs(ctx);
    ctx->profiling = enabled ? 1 : 0;
    return KS_OK;
}

int ks_run(ks_ctx* ctx, int64_t steps) {
    if (!ctx || steps < 0) return fail(ctx, KS_ERR_ARG, "ks_run: bad arguments");
    if (!ctx->has_pop) return fail(ctx, KS_ERR_STATE, "ks_run: no population");
    cudaSetDevice(ctx->device);
    ctx->timing = ks_timing{};
    const int chunk = ctx->steps_per_graph > 0 ? ctx->steps_per_graph : 64;
    int rc = ensure_chunk(ctx, chunk);
    if (rc) return rc;
    const int64_t end = ctx->steps_done + steps;
    while (ctx->steps_done < end) {
        // A chunk may end early, at a step that holds a collision to fragment;
        // while collisions are frequent the chunks stay short (chunk_hint).
        const int want = ctx->bk.on && ctx->chunk_hint > 0 ? std::min(chunk, ctx->chunk_hint) : chunk;
        const int k = static_cast<int>(std::min<int64_t>(end - ctx->steps_done, want));
        const HostClock::time_point h0 = HostClock::now();
        rc = run_chunk(ctx, k);
        ctx->timing.host_chunk_ms += host_ms(h0, HostClock::now());
        if (rc) return rc;
    }
    return KS_OK;
}

int ks_prepare_run(ks_ctx* ctx) {
    if (!ctx) return KS_ERR_ARG;
    if (!ctx->has_pop) return fail(ctx, KS_ERR_STATE, "ks_prepare_run: no population");
    cudaSetDevice(ctx->device);
    if (ctx->steps_per_graph <= 0 || ctx->dev_sbm) return KS_OK;
    const int k = ctx->steps_per_graph;
    int rc = ensure_chunk(ctx, k);
    if (!rc) rc = plan_chunk(ctx, k);
    // Both parities: a chunk of an odd number of steps leaves the next one on the other.
    const int cur = ctx->cur;
    for (int p = 0; p < 2 && !rc; ++p) {
        ctx->cur = p;
        rc = ensure_graph(ctx, k);
    }
    ctx->cur = cur;
    return rc;
}

int ks_take_conjunctions(ks_ctx* ctx, ks_conjunction* out, int64_t cap, int64_t* count) {
    if (!ctx || !count || cap < 0) return KS_ERR_ARG;
    const int64_t older = static_cast<int64_t>(ctx->conj_out.size());
    const int64_t avail = older + (ctx->pend_end - ctx->pend_begin);
    if (!out) {
        *count = avail;
        return KS_OK;
    }
    const int64_t m = std::min(avail, cap);
    const int64_t m1 = std::min(older, m);  // the older records first
    if (m1 > 0) {
        std::memcpy(out, ctx->conj_out.data(), sizeof(ks_conjunction) * m1);
        ctx->conj_out.erase(ctx->conj_out.begin(), ctx->conj_out.begin() + m1);
    }
    if (m > m1) {
        std::memcpy(out + m1, ctx->h_conj + ctx->pend_begin, sizeof(ks_conjunction) * (m - m1));
        ctx->pend_begin += m - m1;
    }
    *count = m;
    return KS_OK;
}

int ks_take_conjunctions_view(ks_ctx* ctx, const ks_conjunction** first, int64_t* count) {
    if (!ctx || !first || !count) return KS_ERR_ARG;
    if (!ctx->conj_out.empty()) {
        // Older records (chunks not taken before the next one ran): handed out
        // from a holder that the next call of this function or ks_run replaces.
        ctx->conj_view.clear();
        ctx->conj_view.swap(ctx->conj_out);
        *first = ctx->conj_view.data();
        *count = static_cast<int64_t>(ctx->conj_view.size());
        return KS_OK;
    }
    // The last chunk's records where the device copied them (pinned memory).
    *first = ctx->h_conj ? ctx->h_conj + ctx->pend_begin : nullptr;
    *count = ctx->pend_end - ctx->pend_begin;
    ctx->pend_begin = ctx->pend_end;
    return KS_OK;
}

int ks_take_step_stats(ks_ctx* ctx, ks_step_stats* out, int64_t cap, int64_t* count) {
    if (!ctx || !count || cap < 0) return KS_ERR_ARG;
    const int64_t avail = static_cast<int64_t>(ctx->stats_out.size());
    if (!out) {
        *count = avail;
        return KS_OK;
    }
    const int64_t m = std::min(avail, cap);
    std::memcpy(out, ctx->stats_out.data(), sizeof(ks_step_stats) * m);
    ctx->stats_out.erase(ctx->stats_out.begin(), ctx->stats_out.begin() + m);
    *count = m;
    return KS_OK;
}

int ks_set_breakup(ks_ctx* ctx, int on, double lc_m, double catastrophic_j_per_g, uint64_t seed) {
    if (!ctx || !(lc_m > 0.0) || !(catastrophic_j_per_g > 0.0)) return fail(ctx, KS_ERR_ARG, "ks_set_breakup: bad arguments");
    drop_graphs(ctx);  // device fragmentation: its kernels and parameters are part of the graphs
    ctx->bk.on = on != 0;
    ctx->bk.params.lc_m = lc_m;
    ctx->bk.params.catastrophic_j_per_g = catastrophic_j_per_g;
    ctx->bk.seed = seed;
    ctx->bk.rng.clear();
    ctx->bk.next_event.clear();
    return KS_OK;
}

int ks_set_breakup_mode(ks_ctx* ctx, int mode, int64_t max_objects) {
    if (!ctx || (mode != KS_BREAKUP_HOST && mode != KS_BREAKUP_DEVICE) ||
        (mode == KS_BREAKUP_DEVICE && max_objects <= 0))
        return fail(ctx, KS_ERR_ARG, "ks_set_breakup_mode: bad arguments");
    if (max_objects > (int64_t(1) << 30)) return fail(ctx, KS_ERR_RANGE, "ks_set_breakup_mode: budget above 2^30 objects");
    if (ctx->has_pop) return fail(ctx, KS_ERR_STATE, "ks_set_breakup_mode: set the mode before the population");
    cudaSetDevice(ctx->device);
    if (mode == KS_BREAKUP_DEVICE) KS_CUDA(ks::sbm_init_attributes());
    ctx->dev_sbm = mode == KS_BREAKUP_DEVICE;
    ctx->dev_cap = ctx->dev_sbm ? max_objects : 0;
    drop_graphs(ctx);
    return KS_OK;
}

int ks_set_masses(ks_ctx* ctx, int64_t n, const double* mass_kg) {
    if (!ctx || !ctx->has_pop || n != ctx->n || (n > 0 && !mass_kg))
        return fail(ctx, KS_ERR_ARG, "ks_set_masses: needs one mass per object of the population");
    cudaSetDevice(ctx->device);
    if (ctx->dev_sbm) {
        if (n > 0) KS_CUDA(cudaMemcpy(ctx->b.mass_kg, mass_kg, sizeof(double) * n, cudaMemcpyHostToDevice));
        return KS_OK;
    }
    const int rc = ensure_mirrors(ctx);
    if (rc) return rc;
    std::copy(mass_kg, mass_kg + n, ctx->bk.mass_kg.begin());
    return KS_OK;
}

// Forced impact with fragmentation on the device: the parents as the host SBM
// builds them (one uniform draw for the side of the crossing, from a stream
// of its own), then the device SBM for this one event at the current time.
static int impact_device(ks_ctx* ctx, int64_t target, double projectile_mass_kg, double v_rel_km_s) {
    ks::DeviceBuffers& b = ctx->b;
    double s[6], mass = 0.0, size = 0.0;
    uint16_t rid = 0;
    int next = 0;
    KS_CUDA(cudaMemcpyAsync(s, b.state[ctx->cur] + 6 * target, 48, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaMemcpyAsync(&mass, b.mass_kg + target, 8, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaMemcpyAsync(&size, b.size_m + target, 8, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaMemcpyAsync(&rid, b.real_id + target, 2, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    const int r = ctx->rbits > 0 ? rid : 0;
    KS_CUDA(cudaMemcpy(&next, b.sbm_next_event + r, sizeof(int), cudaMemcpyDeviceToHost));
    const int id = next++;
    KS_CUDA(cudaMemcpy(b.sbm_next_event + r, &next, sizeof(int), cudaMemcpyHostToDevice));
    ks::SbmRng side(ctx->bk.seed ^ (0x9E3779B97F4A7C15ull * (static_cast<uint64_t>(r) * 65536u + static_cast<uint64_t>(id) + 1)));
    ks::SbmParent tgt, prj;
    ks::sbm_impact_parents(side, target, s, ks::sbm_mass_or_default(mass), size, projectile_mass_kg, v_rel_km_s, tgt,
                           prj);
    ks::SbmEventWork w{};
    for (int q = 0; q < 6; ++q) {
        w.s[0][q] = tgt.s[q];
        w.s[1][q] = prj.s[q];
    }
    w.size_m[0] = tgt.size_m;
    w.size_m[1] = prj.size_m;
    w.mass[0] = tgt.mass_kg;
    w.mass[1] = prj.mass_kg;
    double dv2 = 0.0;
    for (int q = 3; q < 6; ++q) dv2 += (w.s[0][q] - w.s[1][q]) * (w.s[0][q] - w.s[1][q]);
    w.vrel = std::sqrt(dv2);
    const double energy = 500.0 * w.mass[1] * w.vrel * w.vrel / w.mass[0];
    w.catastrophic = energy >= ctx->bk.params.catastrophic_j_per_g ? 1 : 0;
    w.budget[0] = w.catastrophic ? w.mass[0] : std::max(0.0, w.mass[1] * w.vrel * w.vrel - w.mass[1]);
    w.budget[1] = w.mass[1];
    w.t = ctx->t;
    w.rem = 0.0;
    w.target = static_cast<int>(tgt.index);
    w.projectile = static_cast<int>(prj.index);
    w.realisation = r;
    w.id = id;
    w.record = 0;
    KS_CUDA(cudaMemcpy(b.sbm_work, &w, sizeof(w), cudaMemcpyHostToDevice));
    KS_CUDA(cudaMemsetAsync(&b.chunk->flags, 0, sizeof(int), ctx->stream));
    ks::launch_sbm_prepared(b, sbm_args(ctx), force_consts(), 1, ctx->steps_done, b.state[ctx->cur], b.alive[ctx->cur],
                            carry_slot(ctx), b.chunk, ctx->stream);
    KS_CUDA(cudaGetLastError());
    ks_breakup_event ev{};
    int n_live = 0, flags = 0;
    KS_CUDA(cudaMemcpyAsync(&ev, b.sbm_events, sizeof(ev), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaMemcpyAsync(&n_live, b.n_live, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaMemcpyAsync(&flags, &b.chunk->flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (flags & ks::FLAG_POP_BUDGET)
        return fail(ctx, KS_ERR_OVERFLOW, "fragments would pass the population budget of " + std::to_string(b.cap) +
                                              " objects (ks_set_breakup_mode)");
    // The real object's fate: destroyed as the SBM projectile or above the
    // catastrophic threshold, else eroded by the ejected mass.
    const uint8_t dead = 0;
    if (prj.index >= 0) KS_CUDA(cudaMemcpy(b.alive[ctx->cur] + prj.index, &dead, 1, cudaMemcpyHostToDevice));
    if (tgt.index >= 0) {
        if (w.catastrophic) KS_CUDA(cudaMemcpy(b.alive[ctx->cur] + tgt.index, &dead, 1, cudaMemcpyHostToDevice));
        else {
            const double left = std::max(w.mass[0] - w.budget[0], 0.0);
            KS_CUDA(cudaMemcpy(b.mass_kg + tgt.index, &left, sizeof(left), cudaMemcpyHostToDevice));
        }
    }
    ctx->n = n_live;
    ctx->bk.out.push_back(ev);
    drop_graphs(ctx);
    return KS_OK;
}

int ks_impact(ks_ctx* ctx, int64_t target, double projectile_mass_kg, double v_rel_km_s) {
    if (!ctx || !ctx->has_pop || target < 0 || target >= ctx->n || !(projectile_mass_kg > 0.0) || !(v_rel_km_s >= 0.0))
        return fail(ctx, KS_ERR_ARG, "ks_impact: bad arguments");
    cudaSetDevice(ctx->device);
    if (ctx->dev_sbm) return impact_device(ctx, target, projectile_mass_kg, v_rel_km_s);
    int rc = ensure_mirrors(ctx);
    if (rc) return rc;
    ensure_streams(ctx);
    ks_ctx::Breakup& k = ctx->bk;
    double s[6];
    KS_CUDA(cudaMemcpyAsync(s, ctx->b.state[ctx->cur] + 6 * target, 48, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    const int r = k.rid[static_cast<size_t>(target)];
    ks::SbmParent tgt, prj;
    ks::sbm_impact_parents(k.rng[static_cast<size_t>(r)], target, s, k.mass_kg[static_cast<size_t>(target)],
                           k.size_m[static_cast<size_t>(target)], projectile_mass_kg, v_rel_km_s, tgt, prj);
    ks_breakup_event ev{};
    ev.step = ctx->steps_done;
    ev.id = k.next_event[static_cast<size_t>(r)]++;
    ev.realisation = r;
    ev.target = tgt.index;
    ev.projectile = prj.index;
    ev.first_fragment = ctx->n;
    NewFragments nf;
    ks::SbmOutcome oc;
    ks::sbm_fragment(k.rng[static_cast<size_t>(r)], k.params, tgt, prj, ctx->t, ev, nf.rows, oc);
    if (oc.kill_projectile) nf.killed.push_back(prj.index);
    if (oc.kill_target) nf.killed.push_back(tgt.index);
    if (oc.reduce_target) k.mass_kg[static_cast<size_t>(tgt.index)] = oc.target_mass_after;
    nf.spans.push_back({ev.first_fragment, ev.fragments, 0.0, ctx->epoch_jd + ctx->t / 86400.0});
    nf.rid.assign(nf.rows.size(), static_cast<uint16_t>(r));
    nf.event.assign(nf.rows.size(), ev.id);
    k.out.push_back(ev);
    return commit_fragments(ctx, nf);
}

int64_t ks_sbm_impact(uint64_t seed, double lc_m, double catastrophic_j_per_g, const double* state,
                      double target_mass_kg, double target_size_m, double projectile_mass_kg, double v_rel_km_s,
                      double t, ks_breakup_event* event, double* frag_states, double* frag_size, double* frag_mass,
                      double* frag_area_to_mass, int64_t cap, double* target_after) {
    if (!state || !event || cap < 0 || !(lc_m > 0.0) || !(projectile_mass_kg > 0.0)) return -1;
    ks::SbmRng rng(seed);
    ks::SbmParams p;
    p.lc_m = lc_m;
    p.catastrophic_j_per_g = catastrophic_j_per_g;
    ks::SbmParent tgt, prj;
    ks::sbm_impact_parents(rng, 0, state, target_mass_kg, target_size_m, projectile_mass_kg, v_rel_km_s, tgt, prj);
    ks_breakup_event ev{};
    ev.target = tgt.index;
    ev.projectile = prj.index;
    ev.first_fragment = 1;
    std::vector<ks::SbmFragment> rows;
    ks::SbmOutcome oc;
    ks::sbm_fragment(rng, p, tgt, prj, t, ev, rows, oc);
    *event = ev;
    const int64_t m = static_cast<int64_t>(rows.size());
    for (int64_t k = 0; k < m && k < cap; ++k) {
        const ks::SbmFragment& f = rows[static_cast<size_t>(k)];
        if (frag_states) std::copy(f.s, f.s + 6, frag_states + 6 * k);
        if (frag_size) frag_size[k] = f.size_m;
        if (frag_mass) frag_mass[k] = f.mass_kg;
        if (frag_area_to_mass) frag_area_to_mass[k] = f.area_to_mass;
    }
    if (target_after) {
        const bool killed = (oc.kill_target && tgt.index == 0) || (oc.kill_projectile && prj.index == 0);
        target_after[0] = killed ? 0.0 : 1.0;
        target_after[1] = oc.reduce_target && tgt.index == 0 ? oc.target_mass_after : target_mass_kg;
    }
    return m;
}

int ks_save_population(ks_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, KS_ERR_ARG, "ks_save_population: bad arguments");
    if (!ctx->has_pop) return fail(ctx, KS_ERR_STATE, "ks_save_population: no population");
    if (ctx && ctx->dev_sbm) return fail(ctx, KS_ERR_STATE, "ks_save_population: not available with fragmentation on the device");
    cudaSetDevice(ctx->device);
    int rc = ensure_mirrors(ctx);
    if (rc) return rc;
    const size_t n = static_cast<size_t>(ctx->n);
    std::vector<double> st(6 * n);
    std::vector<uint8_t> al(n);
    if (n > 0) {
        KS_CUDA(cudaMemcpyAsync(st.data(), ctx->b.state[ctx->cur], sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(al.data(), ctx->b.alive[ctx->cur], n, cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    const ks_ctx::Breakup& k = ctx->bk;
    PopHeader h{};
    std::memcpy(h.magic, kPopMagic, 8);
    h.n = ctx->n;
    h.realisations = ctx->realisations;
    h.streams = static_cast<int32_t>(k.rng.size());
    h.epoch_jd = ctx->epoch_jd;
    h.t = ctx->t;
    h.dt = ctx->dt;
    h.steps_done = ctx->steps_done;
    h.breakup_on = k.on ? 1 : 0;
    h.lc_m = k.params.lc_m;
    h.catastrophic_j_per_g = k.params.catastrophic_j_per_g;
    h.seed = k.seed;
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    bool ok = static_cast<bool>(f) && put(f, &h, 1) && put(f, st.data(), 6 * n) && put(f, al.data(), n) &&
              put(f, k.size_m.data(), n) && put(f, k.mass_kg.data(), n) && put(f, k.area_to_mass.data(), n) &&
              put(f, k.event.data(), n) && put(f, k.rid.data(), n);
    for (size_t r = 0; ok && r < k.rng.size(); ++r) {
        const std::string text = k.rng[r].state();
        const int32_t ne = k.next_event[r];
        const uint32_t len = static_cast<uint32_t>(text.size());
        ok = put(f, &ne, 1) && put(f, &len, 1) && put(f, text.data(), len);
    }
    if (!ok) return fail(ctx, KS_ERR_ARG, std::string("ks_save_population: cannot write ") + path);
    return KS_OK;
}

int ks_load_population(ks_ctx* ctx, const char* path) {
    if (ctx && ctx->dev_sbm) return fail(ctx, KS_ERR_STATE, "ks_load_population: not available with fragmentation on the device");
    if (!ctx || !path) return fail(ctx, KS_ERR_ARG, "ks_load_population: bad arguments");
    std::ifstream f(path, std::ios::binary);
    PopHeader h{};
    if (!f || !get(f, &h, 1) || std::memcmp(h.magic, kPopMagic, 8) != 0)
        return fail(ctx, KS_ERR_ARG, std::string("ks_load_population: not a population file: ") + path);
    if (h.n < 0 || h.n > (int64_t(1) << 30) || h.realisations < 1 || h.realisations > 65535 || h.streams < 0 ||
        h.streams > h.realisations || !(h.dt > 0.0))
        return fail(ctx, KS_ERR_ARG, "ks_load_population: inconsistent header");
    const size_t n = static_cast<size_t>(h.n);
    std::vector<double> st(6 * n), size_m(n), mass(n), a2m(n);
    std::vector<uint8_t> al(n);
    std::vector<int32_t> ev(n);
    std::vector<uint16_t> rid(n);
    bool ok = get(f, st.data(), 6 * n) && get(f, al.data(), n) && get(f, size_m.data(), n) && get(f, mass.data(), n) &&
              get(f, a2m.data(), n) && get(f, ev.data(), n) && get(f, rid.data(), n);
    std::vector<ks::SbmRng> rngs;
    std::vector<int32_t> next_event;
    for (int32_t r = 0; ok && r < h.streams; ++r) {
        int32_t ne = 0;
        uint32_t len = 0;
        ok = get(f, &ne, 1) && get(f, &len, 1) && len < (1u << 20);
        std::string text(ok ? len : 0, '\0');
        ok = ok && (len == 0 || get(f, &text[0], len));
        ks::SbmRng g;
        ok = ok && g.set_state(text);
        rngs.push_back(g);
        next_event.push_back(ne);
    }
    for (size_t i = 0; ok && i < n; ++i) ok = rid[i] < h.realisations;
    if (!ok) return fail(ctx, KS_ERR_ARG, std::string("ks_load_population: truncated or corrupt file: ") + path);
    cudaSetDevice(ctx->device);
    int rc = ensure_objects(ctx, h.n);
    if (rc) return rc;
    ctx->n = h.n;
    ctx->cur = 0;
    ctx->realisations = h.realisations;
    int rbits = 0;
    while ((1 << rbits) < h.realisations) ++rbits;
    ctx->rbits = rbits;
    ctx->offsets.assign({0, h.n});
    drop_graphs(ctx);
    rc = upload_population(ctx, h.n, st.data(), size_m.data(), al.data(), 0);
    if (rc) return rc;
    if (n > 0) KS_CUDA(cudaMemcpyAsync(ctx->b.real_id, rid.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    KS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->epoch_jd = h.epoch_jd;
    ctx->t = h.t;
    ctx->dt = h.dt;
    ctx->steps_done = h.steps_done;
    ks_ctx::Breakup& k = ctx->bk;
    reset_breakup_run(ctx);
    k.on = h.breakup_on != 0;
    k.params.lc_m = h.lc_m;
    k.params.catastrophic_j_per_g = h.catastrophic_j_per_g;
    k.seed = h.seed;
    k.rng = std::move(rngs);
    k.next_event = std::move(next_event);
    k.size_m = std::move(size_m);
    k.mass_kg = std::move(mass);
    k.area_to_mass = std::move(a2m);
    k.event = std::move(ev);
    k.rid = std::move(rid);
    k.mirrors = true;
    rc = seed_speculation(ctx);
    if (rc) return rc;
    ctx->has_pop = true;
    clear_records(ctx);
    ctx->stats_out.clear();
    return KS_OK;
}

int ks_take_breakups(ks_ctx* ctx, ks_breakup_event* out, int64_t cap, int64_t* count) {
    if (!ctx || !count || cap < 0) return KS_ERR_ARG;
    std::vector<ks_breakup_event>& v = ctx->bk.out;
    if (!out) {
        *count = static_cast<int64_t>(v.size());
        return KS_OK;
    }
    const int64_t m = std::min(static_cast<int64_t>(v.size()), cap);
    std::memcpy(out, v.data(), sizeof(ks_breakup_event) * m);
    v.erase(v.begin(), v.begin() + m);
    *count = m;
    return KS_OK;
}

int ks_get_objects(ks_ctx* ctx, int64_t n, double* size_m, double* mass_kg, double* area_to_mass, int32_t* event,
                   int32_t* realisation) {
    if (!ctx || !ctx->has_pop || n != ctx->n) return fail(ctx, KS_ERR_ARG, "ks_get_objects: n must be the population size");
    cudaSetDevice(ctx->device);
    if (ctx->dev_sbm) {
        const ks::DeviceBuffers& b = ctx->b;
        std::vector<uint16_t> rid(static_cast<size_t>(n));
        if (n > 0) {
            if (size_m) KS_CUDA(cudaMemcpyAsync(size_m, b.size_m, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
            if (mass_kg) KS_CUDA(cudaMemcpyAsync(mass_kg, b.mass_kg, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
            if (area_to_mass)
                KS_CUDA(cudaMemcpyAsync(area_to_mass, b.a2m, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
            if (event) KS_CUDA(cudaMemcpyAsync(event, b.event_of, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
            if (realisation)
                KS_CUDA(cudaMemcpyAsync(rid.data(), b.real_id, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        }
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (realisation)
            for (int64_t i = 0; i < n; ++i) realisation[i] = rid[static_cast<size_t>(i)];
        return KS_OK;
    }
    const int rc = ensure_mirrors(ctx);
    if (rc) return rc;
    const ks_ctx::Breakup& k = ctx->bk;
    for (int64_t i = 0; i < n; ++i) {
        const size_t q = static_cast<size_t>(i);
        if (size_m) size_m[i] = k.size_m[q];
        if (mass_kg) mass_kg[i] = k.mass_kg[q];
        if (area_to_mass) area_to_mass[i] = k.area_to_mass[q];
        if (event) event[i] = k.event[q];
        if (realisation) realisation[i] = k.rid[q];
    }
    return KS_OK;
}

int ks_screen(ks_ctx* ctx, int64_t n, const double* before, const double* after, const uint8_t* alive_after,
              const double* size_m, double t0, double dt, ks_conjunction* out, int64_t cap, int64_t* count,
              ks_step_stats* stats) {
    if (!ctx || n < 0 || !count || (n > 0 && (!before || !after || !alive_after || !size_m)) || !(dt > 0.0))
        return fail(ctx, KS_ERR_ARG, "ks_screen: bad arguments");
    if (ctx && ctx->dev_sbm) return fail(ctx, KS_ERR_STATE, "ks_screen: not available with fragmentation on the device");
    cudaSetDevice(ctx->device);
    int rc = ensure_objects(ctx, n);
    if (rc) return rc;
    rc = ensure_chunk(ctx, 1);
    if (rc) return rc;
    ctx->has_pop = false;
    ctx->n = n;
    ctx->realisations = 1;
    ctx->rbits = 0;
    ctx->offsets.assign({0, n});
    reset_breakup_run(ctx);
    rc = upload_population(ctx, n, before, size_m, nullptr, 0);
    if (!rc) rc = upload_population(ctx, n, after, nullptr, alive_after, 1);
    if (rc) return rc;
    const double saved_dt = ctx->dt;
    ctx->dt = dt;
    StepParams sp{};
    sp.t0 = t0;
    sp.step = 0;
    ctx->h_params[0] = sp;
    KS_CUDA(cudaMemcpyAsync(ctx->b.params, ctx->h_params, sizeof(StepParams), cudaMemcpyHostToDevice, ctx->stream));
    std::vector<ks_conjunction> found;
    ks_step_stats st{};
    for (int attempt = 0;; ++attempt) {
        ks::launch_chunk_init(ctx->b, 1, ctx->stream);
        StepArgs a = step_args(ctx, 0, 1, 0);
        a.hist = nullptr;  // keys come from k_screen_keys: the sort counts their digits itself
        a.pack_bits = 0;
        ks::launch_seed_ctrl(ctx->b, static_cast<int>(n), 0, a.ctrl, 0, ctx->stream);
        ks::launch_screen_keys(ctx->b, a, ctx->stream);
        ks::launch_sort(ctx->b, a, ctx->stream);
        ks::launch_cells(ctx->b, a, ctx->stream);
        ks::launch_pairs(ctx->b, a, ctx->stream);
        ks::launch_refine(ctx->b, a, ctx->b.conj, ctx->b.conj_cap, ctx->b.chunk, ctx->stream);
        KS_CUDA(cudaGetLastError());
        KS_CUDA(cudaMemcpyAsync(ctx->h_ctrl, ctx->b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaMemcpyAsync(ctx->h_chunk, ctx->b.chunk, sizeof(ks::ChunkCtrl), cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        const Ctrl& c = ctx->h_ctrl[0];
        const int flags = c.flags | ctx->h_chunk->flags;
        const bool surv_over = c.refined > static_cast<unsigned long long>(ctx->b.surv_cap);
        const bool items_over = ks::items_total(c) > ctx->b.items_cap;
        if (flags & ks::FLAG_KEY_RANGE) { ctx->dt = saved_dt; return fail(ctx, KS_ERR_RANGE, "cell key outside its grid bounds or wider than 63 bits"); }
        if (flags & ks::FLAG_TIMEOUT) { ctx->dt = saved_dt; return fail(ctx, KS_ERR_TIMEOUT, "radix sort look-back or grid barrier wait gave up"); }
        if (!(flags & (ks::FLAG_CONJ_OVERFLOW | ks::FLAG_SORT_BITS)) && !surv_over && !items_over) {
            st.step = 0;
            st.candidate_pairs = static_cast<int64_t>(c.candidates);
            st.refined_pairs = static_cast<int64_t>(c.refined);
            st.co_orbiting = static_cast<int64_t>(c.co_orbiting);
            st.conjunctions = static_cast<int64_t>(c.conj);
            st.cell_km = c.grid.cell;
            st.max_cell_objects = c.max_cell;
            st.alive = c.n_alive;
            break;
        }
        if (attempt >= kMaxReplays) { ctx->dt = saved_dt; return fail(ctx, KS_ERR_OVERFLOW, "ks_screen: buffers overflow"); }
        if (flags & ks::FLAG_SORT_BITS) ctx->sort_passes = std::max(ctx->sort_passes, passes_for_bits(c.grid.bits));
        if (surv_over && (rc = ensure_survivors(ctx, static_cast<int64_t>(c.refined) * 2))) { ctx->dt = saved_dt; return rc; }
        if (items_over && (rc = ensure_items(ctx, ks::items_total(c) * 3 / 2 + 1024))) { ctx->dt = saved_dt; return rc; }
        if ((flags & ks::FLAG_CONJ_OVERFLOW) && (rc = ensure_conj(ctx, static_cast<int64_t>(ctx->h_chunk->conj_count) * 2))) {
            ctx->dt = saved_dt;
            return rc;
        }
    }
    ctx->dt = saved_dt;
    const int64_t nc = static_cast<int64_t>(ctx->h_chunk->conj_count);
    stash_pending(ctx);
    if (nc > 0) {
        KS_CUDA(cudaMemcpyAsync(ctx->h_conj, ctx->b.conj, sizeof(ks_conjunction) * nc, cudaMemcpyDeviceToHost, ctx->stream));
        KS_CUDA(cudaStreamSynchronize(ctx->stream));
        found.assign(ctx->h_conj, ctx->h_conj + nc);
        std::sort(found.begin(), found.end(), conj_less);
    }
    const int64_t m = std::min<int64_t>(nc, cap);
    if (out && m > 0) std::memcpy(out, found.data(), sizeof(ks_conjunction) * m);
    *count = nc;
    if (stats) *stats = st;
    return KS_OK;
}

int ks_propagate(ks_ctx* ctx, int64_t n, double* states, uint8_t* alive, double epoch_jd, double t, double dt,
                 int64_t steps) {
    if (!ctx || n < 0 || steps < 0 || (n > 0 && !states) || !(dt > 0.0))
        return fail(ctx, KS_ERR_ARG, "ks_propagate: bad arguments");
    std::vector<double> dummy_size(static_cast<size_t>(n > 0 ? n : 1), 0.0);
    const int saved_screen = ctx->screening;
    const double saved_epoch = ctx->epoch_jd, saved_t = ctx->t, saved_dt = ctx->dt;
    ctx->screening = 0;
    drop_graphs(ctx);
    int rc = ks_set_population(ctx, n, states, dummy_size.data(), alive);
    if (!rc) {
        ctx->epoch_jd = epoch_jd;
        ctx->t = t;
        ctx->dt = dt;
        rc = ks_run(ctx, steps);
    }
    if (!rc) rc = ks_get_population(ctx, n, states, alive);
    ctx->screening = saved_screen;
    ctx->epoch_jd = saved_epoch;
    ctx->t = saved_t;
    ctx->dt = saved_dt;
    ctx->has_pop = false;
    drop_graphs(ctx);
    return rc;
}

int ks_get_timing(const ks_ctx* ctx, ks_timing* out) {
    if (!ctx || !out) return KS_ERR_ARG;
    *out = ctx->timing;
    return KS_OK;
}

int ks_measure_fp64(ks_ctx* ctx, double* addmul_per_s, double* fma_per_s) {
    if (!ctx || !addmul_per_s || !fma_per_s) return KS_ERR_ARG;
    if (ctx && ctx->dev_sbm) return fail(ctx, KS_ERR_STATE, "ks_propagate: not available with fragmentation on the device");
    cudaSetDevice(ctx->device);
    KS_CUDA(ks::measure_fp64(addmul_per_s, fma_per_s, ctx->stream));
    return KS_OK;
}

int ks_measure_fp32(ks_ctx* ctx, double* addmul_per_s, double* fma_per_s) {
    if (!ctx || !addmul_per_s || !fma_per_s) return KS_ERR_ARG;
    cudaSetDevice(ctx->device);
    KS_CUDA(ks::measure_fp32(addmul_per_s, fma_per_s, ctx->stream));
    return KS_OK;
}

int ks_measure_fp32x2(ks_ctx* ctx, double* fma_ops_per_s) {
    if (!ctx || !fma_ops_per_s) return KS_ERR_ARG;
    cudaSetDevice(ctx->device);
    KS_CUDA(ks::measure_fp32x2(fma_ops_per_s, ctx->stream));
    return KS_OK;
}

}  // extern "C"
