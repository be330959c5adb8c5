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
//   k_sbm_collect     one block: the step's collisions (listed by the
//                     refinement) in (t, i, j) order, parents at the collision
//                     time (Hermite), the sequential part (destroyed parents,
//                     target roles, eroded masses), event numbers and records
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

constexpr int kCollectThreads = 1024;  // k_sbm_collect: one block
constexpr int kCollectMax = kSbmStepEvents;  // collisions a step can hold (power of two)
constexpr int kFragWarps = 4;          // k_sbm_fragments: events per block (one warp each)
constexpr int kDeadSlots = 2 * kCollectMax;  // k_sbm_collect: shared table of parents touched this step
constexpr int kDeadProbeLimit = kDeadSlots;

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

// Shared table of the parents touched by this step's events: dead, or eroded
// to a new mass. Open addressing on the object index; one thread uses it.
struct Touched {
    int key[kDeadSlots];
    double mass[kDeadSlots];  // < 0: destroyed
    __device__ int find(int idx) const {
        unsigned h = (static_cast<unsigned>(idx) * 2654435761u) & (kDeadSlots - 1);
        for (int p = 0; p < kDeadProbeLimit; ++p) {
            if (key[h] == idx || key[h] == -1) return h;
            h = (h + 1) & (kDeadSlots - 1);
        }
        return -1;
    }
};

// The step's collisions into events. Tail of the sequential part of the
// reference's loop (src/core/breakup.cpp:320-336, 192-230).
__global__ void __launch_bounds__(kCollectThreads) k_sbm_collect(StepArgs a, SbmArgs sa, const double* __restrict__ before,
                                                                const double* __restrict__ after,
                                                                uint8_t* __restrict__ alive_after,
                                                                const double* __restrict__ size_m, double* mass_kg,
                                                                const uint16_t* __restrict__ real_id, int* next_event,
                                                                SbmEventWork* work, ks_breakup_event* records,
                                                                int64_t records_cap) {
    extern __shared__ __align__(16) unsigned char collect_smem[];
    CollisionRec* sc = reinterpret_cast<CollisionRec*>(collect_smem);
    Touched& touched = *reinterpret_cast<Touched*>(sc + kCollectMax);
    int* ord = reinterpret_cast<int*>(&touched + 1);
    if (step_void(a.ctrl)) return;
    const int E = static_cast<int>(min(a.ctrl->n_coll, static_cast<unsigned int>(a.coll_cap)));
    if (E == 0) return;
    const int t = threadIdx.x;
    int N = 1;  // sorted length: a power of two >= E
    while (N < E) N <<= 1;
    for (int e = t; e < N; e += blockDim.x) {
        if (e < E) sc[e] = a.coll[e];
        ord[e] = e;
    }
    for (int k = t; k < kDeadSlots; k += blockDim.x) touched.key[k] = -1;
    __syncthreads();
    // Bitonic sort of the event order by (t, i, j); padding sorts last.
    for (int size = 2; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int u = t; u < N; u += blockDim.x) {
                const int partner = u ^ stride;
                if (partner > u) {
                    const int x = ord[u], y = ord[partner];
                    bool x_after_y;
                    if (x >= E) x_after_y = y < E || x > y;
                    else if (y >= E) x_after_y = false;
                    else {
                        const CollisionRec& cx = sc[x];
                        const CollisionRec& cy = sc[y];
                        x_after_y = cx.t != cy.t ? cx.t > cy.t : (cx.i != cy.i ? cx.i > cy.i : cx.j > cy.j);
                    }
                    const bool up = (u & size) == 0;
                    if (x_after_y == up) {
                        ord[u] = y;
                        ord[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    // Parents at the collision time (src/core/breakup.cpp:324-330).
    const double t0 = a.sp->t0;
    for (int e = t; e < E; e += blockDim.x) {
        const CollisionRec c = sc[ord[e]];
        SbmEventWork& w = work[e];
        const double s = (c.t - t0) / a.dt;
        const int idx[2] = {c.i, c.j};
        for (int p = 0; p < 2; ++p) {
            double b6[6], a6[6];
            for (int q = 0; q < 6; ++q) {
                b6[q] = before[6 * static_cast<int64_t>(idx[p]) + q];
                a6[q] = after[6 * static_cast<int64_t>(idx[p]) + q];
            }
            hermite_state(b6, a6, a.dt, s, w.s[p]);
            w.size_m[p] = size_m[idx[p]];
            const double m = mass_kg[idx[p]];
            w.mass[p] = m > 0.0 ? m : kSbmFallbackMassKg;
        }
        w.target = c.i;
        w.projectile = c.j;
        w.t = c.t;
        w.rem = t0 + a.dt - c.t;
        w.realisation = real_id ? real_id[c.i] : 0;
        w.id = -1;
    }
    __syncthreads();
    // The order-dependent part, one thread: destroyed parents, roles, masses.
    if (t == 0) {
        int nv = 0;
        const int base = static_cast<int>(a.chunk->events);
        for (int e = 0; e < E; ++e) {
            SbmEventWork& w = work[e];
            const int hi = touched.find(w.target), hj = touched.find(w.projectile);
            if (hi < 0 || hj < 0) { atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW); break; }
            const bool dead_i = touched.key[hi] == w.target && touched.mass[hi] < 0.0;
            const bool dead_j = touched.key[hj] == w.projectile && touched.mass[hj] < 0.0;
            if (dead_i || dead_j) continue;  // destroyed earlier in this step
            double mi = touched.key[hi] == w.target ? touched.mass[hi] : w.mass[0];
            double mj = touched.key[hj] == w.projectile ? touched.mass[hj] : w.mass[1];
            if (mi <= 0.0) mi = kSbmFallbackMassKg;
            if (mj <= 0.0) mj = kSbmFallbackMassKg;
            w.mass[0] = mi;
            w.mass[1] = mj;
            if (!(mi >= mj)) {  // the heavier body is the target (ties: the first object)
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
            // Parents' fate, seen by the later events of this step.
            const int ht = touched.find(w.target), hp = touched.find(w.projectile);
            if (ht < 0 || hp < 0) { atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW); break; }
            touched.key[hp] = w.projectile;
            touched.mass[hp] = -1.0;
            touched.key[ht] = w.target;
            touched.mass[ht] = w.catastrophic ? -1.0 : fmax(w.mass[0] - w.budget[0], 0.0);
            w.id = next_event[w.realisation]++;
            w.record = base + nv;
            if (base + nv >= records_cap) { atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW); w.id = -1; break; }
            ++nv;
        }
        a.chunk->events = static_cast<unsigned int>(base + nv);
    }
    __syncthreads();
    // Write the parents' fate for the next step.
    for (int k = t; k < kDeadSlots; k += blockDim.x) {
        const int idx = touched.key[k];
        if (idx < 0) continue;
        if (touched.mass[k] < 0.0) alive_after[idx] = 0;
        else mass_kg[idx] = touched.mass[k];
    }
}

constexpr size_t kCollectSmem = sizeof(CollisionRec) * kCollectMax + sizeof(Touched) + sizeof(int) * kCollectMax;
static_assert(kCollectSmem <= 227 * 1024, "k_sbm_collect's shared memory");
static_assert((kCollectMax & (kCollectMax - 1)) == 0, "the bitonic sort needs a power of two");

// Number of candidate fragments of each event (src/core/breakup.cpp:237-244)
// and the event's record, except its fragment counts.
__global__ void k_sbm_prepare(const Ctrl* ctrl, int count, SbmArgs sa, const StepParams* sp, int64_t step,
                              SbmEventWork* work, ks_breakup_event* records) {
    if (ctrl && step_void(ctrl)) return;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int E = ctrl ? static_cast<int>(min(ctrl->n_coll, static_cast<unsigned int>(count))) : count;
    if (e >= E) return;
    SbmEventWork& w = work[e];
    if (w.id < 0) return;
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
    const int e = blockIdx.x * kFragWarps + (threadIdx.x >> 5);
    const int E = ctrl ? static_cast<int>(min(ctrl->n_coll, static_cast<unsigned int>(count))) : count;
    if (e >= E) return;
    SbmEventWork& w = work[e];
    if (w.id < 0) return;
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
    return cudaFuncSetAttribute(k_sbm_collect, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kCollectSmem));
}

void launch_step_gate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_step_gate<<<1, 32, 0, stream>>>(a.ctrl, a.step_in_chunk, a.steps_in_chunk, a.chunk, b.surv_cap, b.items_cap);
}

void launch_sbm_step(const DeviceBuffers& b, const StepArgs& a, const SbmArgs& s, cudaStream_t stream) {
    const int cap = b.coll_cap;
    k_sbm_collect<<<1, kCollectThreads, kCollectSmem, stream>>>(a, s, b.state[a.src], b.state[1 - a.src], b.alive[1 - a.src],
                                                     b.size_m, b.mass_kg, a.real_id, b.sbm_next_event, b.sbm_work,
                                                     b.sbm_events, b.sbm_events_cap);
    k_sbm_prepare<<<(cap + 127) / 128, 128, 0, stream>>>(a.ctrl, cap, s, a.sp, -1, b.sbm_work, b.sbm_events);
    const int blocks = (cap + kFragWarps - 1) / kFragWarps;
    FragmentSink count_only{};
    count_only.fc = a.fc;
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, count_only, a.chunk);
    k_sbm_place<<<1, 1024, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, b.sbm_events, b.n_live, a.chunk);
    const FragmentSink sink = make_sink(b, b.state[1 - a.src], b.alive[1 - a.src], a.ctrl_next, a.sp, a.dt, a.fc);
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(a.ctrl, cap, s, b.sbm_work, sink, a.chunk);
}

void launch_sbm_prepared(const DeviceBuffers& b, const SbmArgs& s, const ForceConsts& fc, int count, int64_t step,
                         double* state, uint8_t* alive, Ctrl* spec, ChunkCtrl* chunk, cudaStream_t stream) {
    if (count <= 0) return;
    k_sbm_prepare<<<(count + 127) / 128, 128, 0, stream>>>(nullptr, count, s, nullptr, step, b.sbm_work, b.sbm_events);
    const int blocks = (count + kFragWarps - 1) / kFragWarps;
    FragmentSink count_only{};
    count_only.fc = fc;
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(nullptr, count, s, b.sbm_work, count_only, chunk);
    k_sbm_place<<<1, 1024, 0, stream>>>(nullptr, count, s, b.sbm_work, b.sbm_events, b.n_live, chunk);
    const FragmentSink sink = make_sink(b, state, alive, spec, nullptr, 1.0, fc);
    k_sbm_fragments<<<blocks, 32 * kFragWarps, 0, stream>>>(nullptr, count, s, b.sbm_work, sink, chunk);
}

}  // namespace ks
