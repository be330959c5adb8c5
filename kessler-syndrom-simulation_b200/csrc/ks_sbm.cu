// Fragmentation on the device: the NASA Standard Breakup Model inside the
// step loop, with counter-based random numbers (ks_sbm_device.cuh).
//
// The reference fragments after each step, on the host, every collision of
// the step in (t, i, j) order (src/main.cpp:401-407 ->
// src/core/breakup.cpp:316-338): a parent already destroyed earlier in the
// step cannot collide again; the heavier body is the target; the projectile is
// destroyed, the target too above the catastrophic energy threshold, else it
// loses the ejected mass; fragments are drawn from the SBM laws, start from the
// parent's state at the collision time plus their Delta-v and are carried to
// the end of the step. Here the same happens on the device, after the step's
// refinement and before the next step's propagation, inside the chunk's graph:
//
//   launch_step_gate  a step whose buffers overflowed (or whose sort gave up)
//                     is void: it and every later step of the chunk do nothing
//                     (FLAG_HALTED), and the host starts the next chunk at it
//   k_sbm_order       one block: the step's collisions (listed by the
//                     refinement) in (t, i, j) order
//   k_sbm_parents     parents at the collision time (Hermite); each object's
//                     first event of the step
//   k_sbm_simple      events whose parents meet no earlier event: decided in
//                     parallel (roles, catastrophic test, budgets, fates)
//   k_sbm_conflicts   one block: the other events, in order, on the parents'
//                     state the earlier events left
//   k_sbm_number      one block: event numbers per realisation and records
//   k_sbm_prepare     one thread per event: the Poisson number of candidates
//   k_sbm_fragments   one warp per event, run twice: first counting the
//                     fragments each event keeps, then (after k_sbm_place)
//                     writing them; both passes draw the same numbers
//   k_sbm_place       one block: offsets of every event's fragments after the
//                     live population, the new population size, the records
//
// Fragments are written into the end-of-step buffers at [n, n + added), so the
// next step's propagation, grid and screening include them; their speeds and
// positions join the speculation of the next step's grid.
#include <cstdint>

#include "ks_engine.h"
#include "ks_sbm_device.cuh"

namespace ks {
namespace {

constexpr int kFragWarps = 4;             // k_sbm_fragments: warps per block, one event at a time each
constexpr int kNumberRealisations = 16384;  // k_sbm_number: realisations counted in shared memory

__device__ __forceinline__ unsigned long long enc_pos(double x) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Cubic Hermite state at fraction s of a step of length dt between the start
// state a and the end state b (positions with tangents v dt).
__device__ void hermite_state(const double* a, const double* b, double dt, double s, double out[6]) {
    const double s2 = s * s, s3 = s2 * s;
    const double h00 = 2 * s3 - 3 * s2 + 1, h10 = s3 - 2 * s2 + s, h01 = -2 * s3 + 3 * s2, h11 = s3 - s2;
    const double d00 = 6 * s2 - 6 * s, d10 = 3 * s2 - 4 * s + 1, d01 = -6 * s2 + 6 * s, d11 = 3 * s2 - 2 * s;
    for (int q = 0; q < 3; ++q) {
        const double p0 = a[q], p1 = b[q], m0 = a[3 + q] * dt, m1 = b[3 + q] * dt;
        out[q] = h00 * p0 + h10 * m0 + h01 * p1 + h11 * m1;
        out[3 + q] = (d00 * p0 + d10 * m0 + d01 * p1 + d11 * m1) / dt;
    }
}

// Lunar stage at fraction tau of the step, quadratic through the step's three
// stages (start, middle, end). The Moon moves ~1 km/s on a 384 000 km orbit:
// over a 10 s step the interpolation error is far below a metre.
__device__ MoonStage moon_at(const MoonStage* m, double tau) {
    const double l0 = 2.0 * (tau - 0.5) * (tau - 1.0), l1 = -4.0 * tau * (tau - 1.0), l2 = 2.0 * tau * (tau - 0.5);
    MoonStage o;
    o.mx = l0 * m[0].mx + l1 * m[1].mx + l2 * m[2].mx;
    o.my = l0 * m[0].my + l1 * m[1].my + l2 * m[2].my;
    o.mz = l0 * m[0].mz + l1 * m[1].mz + l2 * m[2].mz;
    o.ix = l0 * m[0].ix + l1 * m[1].ix + l2 * m[2].ix;
    o.iy = l0 * m[0].iy + l1 * m[1].iy + l2 * m[2].iy;
    o.iz = l0 * m[0].iz + l1 * m[1].iz + l2 * m[2].iz;
    return o;
}

// The fate of an event's parents and its roles (src/core/breakup.cpp:198-230):
// masses mi, mj of the objects c.i, c.j now (0 or less: unknown, 100 kg), the
// heavier is the target (ties: the first object), relative speed, specific
// energy, catastrophic test, mass budgets.
__device__ void decide_event(SbmEventWork& w, double mi, double mj, const SbmArgs& sa) {
    if (mi <= 0.0) mi = kSbmFallbackMassKg;
    if (mj <= 0.0) mj = kSbmFallbackMassKg;
    w.mass[0] = mi;
    w.mass[1] = mj;
    if (!(mi >= mj)) {
        for (int q = 0; q < 6; ++q) { const double x = w.s[0][q]; w.s[0][q] = w.s[1][q]; w.s[1][q] = x; }
        double x = w.size_m[0]; w.size_m[0] = w.size_m[1]; w.size_m[1] = x;
        x = w.mass[0]; w.mass[0] = w.mass[1]; w.mass[1] = x;
        const int k = w.target; w.target = w.projectile; w.projectile = k;
    }
    double dv2 = 0.0;
    for (int q = 3; q < 6; ++q) dv2 += (w.s[0][q] - w.s[1][q]) * (w.s[0][q] - w.s[1][q]);
    w.vrel = sqrt(dv2);
    const double energy = 500.0 * w.mass[1] * w.vrel * w.vrel / w.mass[0];
    w.catastrophic = energy >= sa.catastrophic_j_per_g ? 1 : 0;
    w.budget[0] = w.catastrophic ? w.mass[0] : fmax(0.0, w.mass[1] * w.vrel * w.vrel - w.mass[1]);
    w.budget[1] = w.mass[1];
}

constexpr int kOrderThreads = 1024;
constexpr int kConflictMax = 2048;     // events per step whose parent met an earlier event of the step
constexpr int kConflictSlots = 8192;   // shared table of those events' parents (power of two)
constexpr int kNoEvent = 0x7F7F7F7F;   // "no event yet" in the per-object first-event array
constexpr int kValidEvent = -2;        // an event that fragments, before its number is given

// Order of the step's collisions by (t, i, j) (src/core/breakup.cpp:320, the
// order Screener::finish sorts them in): 64-bit keys, the collision time as a
// fraction of the step in 50 bits above the collision's index, sorted in
// shared memory; runs with equal 50-bit times are put in exact (t, i, j) order.
__global__ void __launch_bounds__(kOrderThreads) k_sbm_order(StepArgs a, int* order, int* misc) {
    extern __shared__ unsigned long long okeys[];
    if (step_void(a.ctrl)) return;
    const unsigned int n_coll = a.ctrl->n_coll;
    const int E = static_cast<int>(min(n_coll, static_cast<unsigned int>(a.coll_cap)));
    if (threadIdx.x == 0) misc[0] = 0;  // conflicting events of this step
    if (E == 0) return;
    const double t0 = a.sp->t0;
    int N = 1;
    while (N < E) N <<= 1;
    for (int u = threadIdx.x; u < N; u += blockDim.x) {
        unsigned long long k = ~0ull;
        if (u < E) {
            double f = (a.coll[u].t - t0) / a.dt;
            f = fmin(fmax(f, 0.0), 1.0 - 1e-15);
            k = (static_cast<unsigned long long>(f * 1125899906842624.0) << 14) | static_cast<unsigned long long>(u);
        }
        okeys[u] = k;
    }
    __syncthreads();
    for (int size = 2; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int u = threadIdx.x; u < N; u += blockDim.x) {
                const int partner = u ^ stride;
                if (partner > u) {
                    const unsigned long long x = okeys[u], y = okeys[partner];
                    const bool up = (u & size) == 0;
                    if ((x > y) == up) {
                        okeys[u] = y;
                        okeys[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        // Equal 50-bit times (ties or nearly): insertion by the exact (t, i, j).
        for (int p = 1; p < E; ++p) {
            if ((okeys[p] >> 14) != (okeys[p - 1] >> 14)) continue;
            const unsigned long long v = okeys[p];
            const CollisionRec cv = a.coll[v & 0x3FFFull];
            int q = p;
            while (q > 0 && (okeys[q - 1] >> 14) == (v >> 14)) {
                const CollisionRec cq = a.coll[okeys[q - 1] & 0x3FFFull];
                const bool after = cq.t != cv.t ? cq.t > cv.t : (cq.i != cv.i ? cq.i > cv.i : cq.j > cv.j);
                if (!after) break;
                okeys[q] = okeys[q - 1];
                --q;
            }
            okeys[q] = v;
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < E; p += blockDim.x) order[p] = static_cast<int>(okeys[p] & 0x3FFFull);
}

// Parents at the collision time (src/core/breakup.cpp:324-330) and each
// object's first event of the step.
__global__ void k_sbm_parents(StepArgs a, const double* __restrict__ before, const double* __restrict__ after,
                              const double* __restrict__ size_m, const double* __restrict__ mass_kg,
                              const uint16_t* __restrict__ real_id, const int* __restrict__ order, SbmEventWork* work,
                              int* first) {
    if (step_void(a.ctrl)) return;
    const int E = static_cast<int>(min(a.ctrl->n_coll, static_cast<unsigned int>(a.coll_cap)));
    const double t0 = a.sp->t0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < E; p += gridDim.x * blockDim.x) {
        const CollisionRec c = a.coll[order[p]];
        SbmEventWork& w = work[p];
        const double s = (c.t - t0) / a.dt;
        const int idx[2] = {c.i, c.j};
        for (int q2 = 0; q2 < 2; ++q2) {
            double b6[6], a6[6];
            for (int q = 0; q < 6; ++q) {
                b6[q] = before[6 * static_cast<int64_t>(idx[q2]) + q];
                a6[q] = after[6 * static_cast<int64_t>(idx[q2]) + q];
            }
            hermite_state(b6, a6, a.dt, s, w.s[q2]);
            w.size_m[q2] = size_m[idx[q2]];
            w.mass[q2] = mass_kg[idx[q2]];
        }
        w.target = c.i;
        w.projectile = c.j;
        w.t = c.t;
        w.rem = t0 + a.dt - c.t;
        w.realisation = real_id ? real_id[c.i] : 0;
        w.id = -1;
        w.record = -1;
        atomicMin(&first[c.i], p);
        atomicMin(&first[c.j], p);
    }
}

// Events whose parents meet no earlier event of the step are independent of
// every other: decided and applied in parallel. The rest are listed for the
// ordered pass.
__global__ void k_sbm_simple(StepArgs a, SbmArgs sa, uint8_t* alive_after, double* mass_kg, SbmEventWork* work,
                             const int* __restrict__ first, int* misc, int* pending) {
    if (step_void(a.ctrl)) return;
    const int E = static_cast<int>(min(a.ctrl->n_coll, static_cast<unsigned int>(a.coll_cap)));
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < E; p += gridDim.x * blockDim.x) {
        SbmEventWork& w = work[p];
        if (first[w.target] == p && first[w.projectile] == p) {
            decide_event(w, w.mass[0], w.mass[1], sa);
            alive_after[w.projectile] = 0;
            if (w.catastrophic) alive_after[w.target] = 0;
            else mass_kg[w.target] = fmax(w.mass[0] - w.budget[0], 0.0);
            w.id = kValidEvent;
        } else {
            const int k = atomicAdd(&misc[0], 1);
            if (k < kConflictMax) pending[k] = p;
            else atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW);
        }
    }
}

// Shared table of the parents of conflicting events: alive flag and mass now.
struct ConflictTable {
    int key[kConflictSlots];
    double mass[kConflictSlots];
    uint8_t alive[kConflictSlots];
    __device__ int find(int idx) const {
        unsigned h = (static_cast<unsigned>(idx) * 2654435761u) & (kConflictSlots - 1);
        for (int p = 0; p < kConflictSlots; ++p) {
            if (key[h] == idx || key[h] == -1) return static_cast<int>(h);
            h = (h + 1) & (kConflictSlots - 1);
        }
        return -1;
    }
};

// The conflicting events in order, one thread, on the parents' state as the
// parallel events left it: a parent destroyed earlier in the step cannot
// collide again (src/core/breakup.cpp:322-323), an eroded one collides with
// its remaining mass.
__global__ void __launch_bounds__(kOrderThreads) k_sbm_conflicts(StepArgs a, SbmArgs sa, uint8_t* alive_after,
                                                                 double* mass_kg, SbmEventWork* work,
                                                                 const int* misc, const int* pending_in) {
    extern __shared__ __align__(16) unsigned char conflict_smem[];
    ConflictTable& tab = *reinterpret_cast<ConflictTable*>(conflict_smem);
    int* plist = reinterpret_cast<int*>(conflict_smem + sizeof(ConflictTable));
    if (step_void(a.ctrl)) return;
    const int P = min(misc[0], kConflictMax);
    if (P == 0) return;
    int N = 1;
    while (N < P) N <<= 1;
    for (int u = threadIdx.x; u < N; u += blockDim.x) plist[u] = u < P ? pending_in[u] : 0x7FFFFFFF;
    for (int k = threadIdx.x; k < kConflictSlots; k += blockDim.x) tab.key[k] = -1;
    __syncthreads();
    for (int size = 2; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int u = threadIdx.x; u < N; u += blockDim.x) {
                const int partner = u ^ stride;
                if (partner > u) {
                    const int x = plist[u], y = plist[partner];
                    const bool up = (u & size) == 0;
                    if ((x > y) == up) {
                        plist[u] = y;
                        plist[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    // The parents into the table (at most 2 P <= 4096 keys in 8192 slots).
    for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) {
        const SbmEventWork& w = work[plist[k >> 1]];
        const int idx = (k & 1) ? w.projectile : w.target;
        unsigned h = (static_cast<unsigned>(idx) * 2654435761u) & (kConflictSlots - 1);
        for (int probe = 0; probe < kConflictSlots; ++probe) {
            const int prev = atomicCAS(&tab.key[h], -1, idx);
            if (prev == -1 || prev == idx) break;
            h = (h + 1) & (kConflictSlots - 1);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kConflictSlots; k += blockDim.x) {
        const int idx = tab.key[k];
        if (idx < 0) continue;
        tab.alive[k] = alive_after[idx];
        tab.mass[k] = mass_kg[idx];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < P; ++k) {
            SbmEventWork& w = work[plist[k]];
            const int hi = tab.find(w.target), hj = tab.find(w.projectile);
            if (hi < 0 || hj < 0 || !tab.alive[hi] || !tab.alive[hj]) continue;  // destroyed earlier
            const int i0 = w.target;
            decide_event(w, tab.mass[hi], tab.mass[hj], sa);
            const int ht = w.target == i0 ? hi : hj, hp = w.target == i0 ? hj : hi;
            tab.alive[hp] = 0;
            if (w.catastrophic) tab.alive[ht] = 0;
            else tab.mass[ht] = fmax(w.mass[0] - w.budget[0], 0.0);
            w.id = kValidEvent;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kConflictSlots; k += blockDim.x) {
        const int idx = tab.key[k];
        if (idx < 0) continue;
        alive_after[idx] = tab.alive[k];
        mass_kg[idx] = tab.mass[k];
    }
}

// Event numbers (per realisation, in event order) and record slots of the
// step's events; the per-object first-event marks are cleared for the next
// step.
__global__ void __launch_bounds__(kOrderThreads) k_sbm_number(StepArgs a, SbmEventWork* work, int* next_event,
                                                              int* first, int64_t records_cap, int n_real) {
    extern __shared__ __align__(16) unsigned char number_smem[];
    uint8_t* valid = number_smem;                                         // kSbmStepEvents
    uint16_t* real = reinterpret_cast<uint16_t*>(number_smem + kSbmStepEvents);  // kSbmStepEvents
    int* counter = reinterpret_cast<int*>(number_smem + 3 * kSbmStepEvents);     // kNumberRealisations
    if (step_void(a.ctrl)) return;
    const int E = static_cast<int>(min(a.ctrl->n_coll, static_cast<unsigned int>(a.coll_cap)));
    if (E == 0) return;
    const bool few = n_real <= kNumberRealisations;
    for (int p = threadIdx.x; p < E; p += blockDim.x) {
        const SbmEventWork& w = work[p];
        valid[p] = w.id == kValidEvent ? 1 : 0;
        real[p] = static_cast<uint16_t>(w.realisation);
        first[w.target] = kNoEvent;
        first[w.projectile] = kNoEvent;
    }
    if (few)
        for (int r = threadIdx.x; r < n_real; r += blockDim.x) counter[r] = next_event[r];
    __syncthreads();
    if (threadIdx.x == 0) {
        int nv = 0;
        const int base = static_cast<int>(a.chunk->events);
        for (int p = 0; p < E; ++p) {
            if (!valid[p]) continue;
            SbmEventWork& w = work[p];
            if (base + nv >= records_cap) {
                atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW);
                w.id = -1;
                continue;
            }
            w.id = few ? counter[real[p]]++ : next_event[real[p]]++;
            w.record = base + nv++;
        }
        a.chunk->events = static_cast<unsigned int>(base + nv);
    }
    __syncthreads();
    if (few)
        for (int r = threadIdx.x; r < n_real; r += blockDim.x) next_event[r] = counter[r];
}

constexpr size_t kOrderSmem = sizeof(unsigned long long) * kSbmStepEvents;
constexpr size_t kConflictSmem = sizeof(ConflictTable) + sizeof(int) * kConflictMax;
constexpr size_t kNumberSmem = 3 * kSbmStepEvents + sizeof(int) * kNumberRealisations;
static_assert(kOrderSmem <= 227 * 1024 && kConflictSmem <= 227 * 1024 && kNumberSmem <= 227 * 1024,
              "shared memory of the device SBM's ordering kernels");
static_assert((kSbmStepEvents & (kSbmStepEvents - 1)) == 0 && kSbmStepEvents <= 16384,
              "collision indices take 14 bits of the ordering keys");

// Number of candidate fragments of each event (src/core/breakup.cpp:237-244)
// and the event's record, except its fragment counts.
__global__ void k_sbm_prepare(const Ctrl* ctrl, int count, SbmArgs sa, const StepParams* sp, int64_t step,
                              SbmEventWork* work, ks_breakup_event* records) {
    if (ctrl && step_void(ctrl)) return;
    const int E = ctrl ? static_cast<int>(min(ctrl->n_coll, static_cast<unsigned int>(count))) : count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    SbmEventWork& w = work[e];
    if (w.id < 0) continue;
    const double M = w.budget[0] + w.budget[1];
    w.expected = M > 0.0 ? 0.1 * pow(M, 0.75) * pow(sa.lc_m, -kSbmExponent) : 0.0;
    EventStream g{sa.seed + static_cast<unsigned long long>(w.realisation), static_cast<uint32_t>(w.id)};
    long long n = w.expected > 0.0 ? poisson_draw(g, w.expected) : 0;
    w.n_cand = n < kSbmMaxFragments ? n : kSbmMaxFragments;
    w.kept = 0;
    w.escaped = 0;
    w.kept_mass = 0.0;
    ks_breakup_event& r = records[w.record];
    r.step = sp ? sp->step : step;
    r.t = w.t;
    r.id = w.id;
    r.realisation = w.realisation;
    r.target = w.target;
    r.projectile = w.projectile;
    r.catastrophic = w.catastrophic;
    r.fragments = 0;
    r.escaped = 0;
    r.pad = 0;
    r.first_fragment = -1;
    r.v_rel_km_s = w.vrel;
    r.energy_j_per_g = 500.0 * w.mass[1] * w.vrel * w.vrel / w.mass[0];
    r.target_mass_kg = w.mass[0];
    r.projectile_mass_kg = w.mass[1];
    r.sbm_mass_kg = M;
    r.expected_fragments = w.expected;
    r.fragments_mass_kg = 0.0;
    for (int q = 0; q < 3; ++q) r.position[q] = w.s[0][q];
    }
}

// Where a pass of k_sbm_fragments sends a kept fragment.
struct FragmentSink {
    double* state;          // null: count only
    uint8_t* alive;
    double* size_m;
    double* mass_kg;
    double* a2m;
    int32_t* event_of;
    uint16_t* real_id;
    Ctrl* spec;             // next step's speculation (or null)
    const StepParams* sp;   // the step: start time and three lunar stages (null: no sub-step)
    double dt;
    ForceConsts fc;
};

// The candidates of every event, one warp per event: draws, the mass budget in
// candidate order (src/core/breakup.cpp:262-271), escape (:286-289). With a
// sink that writes, kept fragments go to slots work.offset + rank, carried
// to the end of the step (:301-306).
__global__ void __launch_bounds__(32 * kFragWarps) k_sbm_fragments(const Ctrl* ctrl, int count, SbmArgs sa,
                                                                 SbmEventWork* work, FragmentSink sink,
                                                                 const ChunkCtrl* chunk) {
    if (ctrl && step_void(ctrl)) return;
    if (sink.state && chunk && (chunk->flags & FLAG_POP_BUDGET)) return;
    const int lane = threadIdx.x & 31;
    const int E = ctrl ? static_cast<int>(min(ctrl->n_coll, static_cast<unsigned int>(count))) : count;
    for (int e = blockIdx.x * kFragWarps + (threadIdx.x >> 5); e < E; e += gridDim.x * kFragWarps) {
    SbmEventWork& w = work[e];
    if (w.id < 0) continue;
    const uint64_t seed = sa.seed + static_cast<unsigned long long>(w.realisation);
    const double p_target = (w.budget[0] + w.budget[1]) > 0.0 ? w.budget[0] / (w.budget[0] + w.budget[1]) : 0.0;
    double used[2] = {0.0, 0.0};
    int kept = 0, escaped = 0;
    double kept_mass = 0.0;
    const unsigned below = (1u << lane) - 1u;
    for (long long k0 = 0; k0 < w.n_cand; k0 += 32) {
        const long long k = k0 + lane;
        const bool have = k < w.n_cand;
        CandidateDraws d;
        int side = 0;
        bool ok = false;
        double L = 0.0, chi = 0.0, m = 0.0;
        if (have) {
            d = candidate_draws(seed, static_cast<uint32_t>(w.id), static_cast<uint32_t>(k));
            side = d.u[kDrawSide] < p_target ? 0 : 1;
            DevParent par;
            par.size_m = w.size_m[side];
            ok = candidate_mass(par, sa.lc_m, d, L, chi, m);
        }
        // Budget in candidate order: all at once when every candidate fits,
        // else lane by lane.
        bool accept = false;
        double tot[2] = {0.0, 0.0};
        for (int sd = 0; sd < 2; ++sd) {
            double v = (ok && side == sd) ? m : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            tot[sd] = v;
        }
        if (used[0] + tot[0] <= w.budget[0] && used[1] + tot[1] <= w.budget[1]) {
            accept = ok;
            used[0] += tot[0];
            used[1] += tot[1];
        } else {
            for (int l = 0; l < 32; ++l) {
                const double ml = __shfl_sync(0xffffffffu, m, l);
                const int sl = __shfl_sync(0xffffffffu, side, l);
                const bool okl = __shfl_sync(0xffffffffu, ok ? 1 : 0, l) != 0;
                const bool acc = okl && used[sl] + ml <= w.budget[sl];
                if (acc) used[sl] += ml;
                if (lane == l) accept = acc;
            }
        }
        double birth[6];
        bool bound = false;
        if (accept) {
            DevParent par;
            for (int q = 0; q < 6; ++q) par.s[q] = w.s[side][q];
            bound = candidate_birth(par, chi, w.vrel, d, sink.fc.neg_mu_earth * -1.0, birth);
        }
        const unsigned kb = __ballot_sync(0xffffffffu, accept && bound);
        escaped += __popc(__ballot_sync(0xffffffffu, accept && !bound));
        double mk = (accept && bound) ? m : 0.0;
        for (int o = 16; o > 0; o >>= 1) mk += __shfl_xor_sync(0xffffffffu, mk, o);
        kept_mass += mk;
        if (sink.state && accept && bound) {
            const int64_t slot = static_cast<int64_t>(w.offset) + kept + __popc(kb & below);
            double s[6];
            for (int q = 0; q < 6; ++q) s[q] = birth[q];
            if (w.rem > 0.0 && sink.sp) {
                // Carried over the rest of the step (src/core/breakup.cpp:304-306).
                const double tau = (w.t - sink.sp->t0) / sink.dt;
                const MoonStage m0 = moon_at(sink.sp->m, tau), m1 = moon_at(sink.sp->m, 0.5 * (tau + 1.0));
                rk4_exact(sink.fc, w.rem, m0, m1, sink.sp->m[2], s);
            }
            for (int q = 0; q < 6; ++q) sink.state[6 * slot + q] = s[q];
            const double r = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
            const bool alive = r >= sink.fc.r_earth;
            sink.alive[slot] = alive ? 1 : 0;
            sink.size_m[slot] = L;
            sink.mass_kg[slot] = m;
            sink.a2m[slot] = exp10(chi);
            sink.event_of[slot] = w.id;
            if (sink.real_id) sink.real_id[slot] = static_cast<uint16_t>(w.realisation);
            if (alive && sink.spec) {
                const double v = sqrt(s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
                atomicMax(&sink.spec->spec_vmax, static_cast<unsigned long long>(__double_as_longlong(v)));
                for (int q = 0; q < 3; ++q) {
                    atomicMin(&sink.spec->bb_min[q], enc_pos(s[q]));
                    atomicMax(&sink.spec->bb_max[q], enc_pos(s[q]));
                }
            }
        }
        kept += __popc(kb);
    }
    if (lane == 0 && !sink.state) {
        w.kept = kept;
        w.escaped = escaped;
        w.kept_mass = kept_mass;
    }
    }
}

// Offsets of every event's fragments after the live population, the new
// size, and the records' fragment counts. Fragments that would pass the
// capacity are not written (FLAG_POP_BUDGET: the run fails with KS_ERR_OVERFLOW).
__global__ void __launch_bounds__(1024) k_sbm_place(Ctrl* ctrl, int count, SbmArgs sa, SbmEventWork* work,
                                                   ks_breakup_event* records, int* n_live, ChunkCtrl* chunk) {
    __shared__ int warp_sum_sh[32];
    __shared__ int base_sh;
    if (ctrl && step_void(ctrl)) return;
    const int E = ctrl ? static_cast<int>(min(ctrl->n_coll, static_cast<unsigned int>(count))) : count;
    if (E == 0) return;
    if (threadIdx.x == 0) base_sh = *n_live;
    __syncthreads();
    int run = 0;
    for (int e0 = 0; e0 < E; e0 += blockDim.x) {
        const int e = e0 + threadIdx.x;
        const int v = (e < E && work[e].id >= 0) ? work[e].kept : 0;
        // Block-wide exclusive scan of v.
        int incl = v;
        const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sum_sh[wp] = incl;
        __syncthreads();
        if (wp == 0) {
            int ws = lane < static_cast<int>(blockDim.x >> 5) ? warp_sum_sh[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            warp_sum_sh[lane] = ws;
        }
        __syncthreads();
        const int excl = run + (wp > 0 ? warp_sum_sh[wp - 1] : 0) + incl - v;
        if (e < E && work[e].id >= 0) {
            SbmEventWork& w = work[e];
            w.offset = base_sh + excl;
            ks_breakup_event& r = records[w.record];
            r.fragments = w.kept;
            r.escaped = w.escaped;
            r.first_fragment = w.kept > 0 ? static_cast<int64_t>(w.offset) : -1;
            r.fragments_mass_kg = w.kept_mass;
        }
        run += warp_sum_sh[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const long long total = static_cast<long long>(base_sh) + run;
        if (total > sa.cap) {
            atomicOr(&chunk->flags, FLAG_POP_BUDGET);
            if (ctrl) atomicOr(&ctrl->flags, FLAG_POP_BUDGET);
        } else {
            *n_live = static_cast<int>(total);
        }
    }
}

__global__ void k_step_gate(Ctrl* ctrl, int step_in_chunk, int steps_in_chunk, ChunkCtrl* chunk, int64_t surv_cap,
                            int64_t items_cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (ctrl->flags & FLAG_HALTED) return;
    const int f = ctrl->flags;
    const bool void_step = (f & (FLAG_TIMEOUT | FLAG_SORT_BITS | FLAG_KEY_RANGE | FLAG_PACK_WIDTH |
                                 FLAG_COLL_OVERFLOW | FLAG_ITEMS_OVERFLOW)) != 0 ||
                           ctrl->refined > static_cast<unsigned long long>(surv_cap) ||
                           static_cast<int64_t>(ctrl->n_items) > items_cap || (chunk->flags & FLAG_CONJ_OVERFLOW) != 0;
    if (!void_step) return;
    chunk->halt_step = step_in_chunk;
    Ctrl* first = ctrl - step_in_chunk;
    for (int k = step_in_chunk; k < steps_in_chunk; ++k) atomicOr(&first[k].flags, FLAG_HALTED);
}

FragmentSink make_sink(const DeviceBuffers& b, double* state, uint8_t* alive, Ctrl* spec, const StepParams* sp,
                       double dt, const ForceConsts& fc) {
    FragmentSink k;
    k.state = state;
    k.alive = alive;
    k.size_m = b.size_m;
    k.mass_kg = b.mass_kg;
    k.a2m = b.a2m;
    k.event_of = b.event_of;
    k.real_id = b.real_id;
    k.spec = spec;
    k.sp = sp;
    k.dt = dt;
    k.fc = fc;
    return k;
}

}  // namespace

cudaError_t sbm_init_attributes() {
    cudaError_t e = cudaFuncSetAttribute(k_sbm_order, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kOrderSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sbm_conflicts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kConflictSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sbm_number, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kNumberSmem));
    return e;
}

void launch_step_gate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_step_gate<<<1, 32, 0, stream>>>(a.ctrl, a.step_in_chunk, a.steps_in_chunk, a.chunk, b.surv_cap, b.items_cap);
}

void launch_sbm_step(const DeviceBuffers& b, const StepArgs& a, const SbmArgs& s, cudaStream_t stream) {
    const int cap = b.coll_cap;
    const int blocks = sm_count() * 2;
    k_sbm_order<<<1, kOrderThreads, kOrderSmem, stream>>>(a, b.sbm_order, b.sbm_misc);
    k_sbm_parents<<<blocks, 128, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src], b.size_m, b.mass_kg, a.real_id,
                                              b.sbm_order, b.sbm_work, b.sbm_first);
    k_sbm_simple<<<blocks, 128, 0, stream>>>(a, s, b.alive[1 - a.src], b.mass_kg, b.sbm_work, b.sbm_first,
                                             b.sbm_misc, b.sbm_pending);
    k_sbm_conflicts<<<1, kOrderThreads, kConflictSmem, stream>>>(a, s, b.alive[1 - a.src], b.mass_kg, b.sbm_work,
                                                                 b.sbm_misc, b.sbm_pending);
    k_sbm_number<<<1, kOrderThreads, kNumberSmem, stream>>>(a, b.sbm_work, b.sbm_next_event, b.sbm_first,
                                                           b.sbm_events_cap, s.realisations);
    k_sbm_prepare<<<blocks, 128, 0, stream>>>(a.ctrl, cap, s, a.sp, -1, b.sbm_work, b.sbm_events);
    FragmentSink count_only{};
    count_only.fc = a.fc;
    k_sbm_fragments<<<blocks * 2, 32 * kFragWarps, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, count_only, a.chunk);
    k_sbm_place<<<1, 1024, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, b.sbm_events, b.n_live, a.chunk);
    const FragmentSink sink = make_sink(b, b.state[1 - a.src], b.alive[1 - a.src], a.ctrl_next, a.sp, a.dt, a.fc);
    k_sbm_fragments<<<blocks * 2, 32 * kFragWarps, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, sink, a.chunk);
}

void launch_sbm_prepared(const DeviceBuffers& b, const SbmArgs& s, const ForceConsts& fc, int count, int64_t step,
                         double* state, uint8_t* alive, Ctrl* spec, ChunkCtrl* chunk, cudaStream_t stream) {
    if (count <= 0) return;
    k_sbm_prepare<<<(count + 127) / 128, 128, 0, stream>>>(nullptr, count, s, nullptr, step, b.sbm_work, b.sbm_events);
    const int blocks = (count + kFragWarps - 1) / kFragWarps;  // one warp per event
    FragmentSink count_only{};
    count_only.fc = fc;
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(nullptr, count, s, b.sbm_work, count_only, chunk);
    k_sbm_place<<<1, 1024, 0, stream>>>(nullptr, count, s, b.sbm_work, b.sbm_events, b.n_live, chunk);
    const FragmentSink sink = make_sink(b, state, alive, spec, nullptr, 1.0, fc);
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(nullptr, count, s, b.sbm_work, sink, chunk);
}

}  // namespace ks
