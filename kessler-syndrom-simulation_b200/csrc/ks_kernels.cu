// B200 kernels of the per-step hot path (plain FP64 form).
//
// Per step, in stream order:
//   propagate   fused RK4 (src/core/orbital.cpp:107-118) over SoA FP64 state, one
//               thread per object in a grid-stride loop; also emits the object's
//               cell key from the start-of-step position and reduces the speed and
//               position bounds that define the next step's grid
//   fix_keys    recomputes keys only when an object that held the top speed died
//   sort        LSD radix sort of (key, index), 8-bit digits, only over the key
//               bits the compact key layout needs
//   cells       cell ranges, open-addressing hash of cell keys, 13 forward
//               neighbours per cell, start-of-step states gathered in cell order
//   pairs       one thread per sorted object: own cell + 13 forward cells, exact
//               filter_pair (src/core/collision_filter.hpp:37-66), warp-ballot
//               compaction of the pairs sent to refinement
//   refine      one thread per surviving pair: Hermite + golden-section TCA
//               (src/core/collision.cpp:77-132)
#include <atomic>
#include <cstdio>

#include "kessler_b200.h"
#include "ks_engine.h"
#include "ks_split.cuh"

namespace ks {

namespace {

constexpr int kBlock = 256;
constexpr unsigned long long kEmpty = ~0ull;
constexpr int kSortTile = 2048;            // keys per radix tile (256 threads x 8)
constexpr int kSortItems = kSortTile / kBlock;
constexpr int kWarps = kBlock / 32;
constexpr int kCellTile = 1024;            // sorted entries per cell-build tile
constexpr int kPropBlock = 128;            // propagation: 4 blocks per SM (at most 128 registers)

// Forward neighbour offset o in 0..12 (src/core/collision_filter.hpp:137-140):
// with the pairs inside a cell they visit every pair of neighbouring cells
// once. o < 9 is (1, o/3 - 1, o%3 - 1), 9..11 is (0, 1, o - 10), 12 is
// (0, 0, 1); computed rather than read from a table at a lane-varying index,
// which constant memory serialises.
__device__ __forceinline__ void forward_offset(int o, int& dx, int& dy, int& dz) {
    dx = o < 9 ? 1 : 0;
    dy = o < 9 ? o / 3 - 1 : (o < 12 ? 1 : 0);
    dz = o < 9 ? o % 3 - 1 : (o < 12 ? o - 10 : 1);
}

// Order-preserving map of doubles to u64 (for atomicMin / atomicMax).
__device__ __forceinline__ unsigned long long enc_double(double x) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dec_double(unsigned long long u) {
    return __longlong_as_double(static_cast<long long>((u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u));
}



// Cell edge (src/core/collision.cpp:339-356) from the largest start speed, and
// the compact key layout over the position bounds.
__device__ void make_grid(double vmax, const unsigned long long* bb_min, const unsigned long long* bb_max,
                          double dt, double threshold_km, int sub, int rbits, double scale, GridParams& g) {
    const double vrel = xmul(2.0, vmax);
    const double c = xadd(xadd(xmul(vrel, dt), threshold_km),
                          xmul(xmul(xmul(xmul(kGravityGradient, vrel), dt), dt), dt));
    g.cell = c > 1.0 ? c : 1.0;
    if (scale > 1.0) g.cell = xmul(g.cell, scale);
    g.inv_cell = xdiv(1.0, g.cell);
    int bits = 0;
    for (int a = 0; a < 3; ++a) {
        const double mn = dec_double(bb_min[a]), mx = dec_double(bb_max[a]);
        long long lo = 0, span = 0;
        if (mn <= mx) {
            lo = static_cast<long long>(floor(xdiv(mn, g.cell)));
            span = static_cast<long long>(floor(xdiv(mx, g.cell))) - lo;
        }
        g.lo[a] = lo;
        g.span[a] = span;
        g.w[a] = span > 0 ? 64 - __clzll(span) : 0;
        bits += g.w[a];
    }
    g.sub = sub;
    g.rbits = rbits;
    g.bits = rbits + bits + 3 * sub;
}

__device__ __forceinline__ unsigned sub_coord(double q, double fq, int sub) {
    const int s = static_cast<int>((q - fq) * static_cast<double>(1 << sub));
    return static_cast<unsigned>(min(max(s, 0), (1 << sub) - 1));
}

// floor(x / c) of the correctly rounded quotient, the reference's cell
// coordinate (src/core/collision.cpp:393-395), without a division where it
// can: y = x * (1/c), both rounded once, lies within 2 units in the last place
// of the quotient, so where y is farther than 2^-50 |y| (4 units) from every
// integer the two have the same floor (the distances below are computed
// exactly or within an ulp of themselves; where the compiler fuses the product
// into them, they are those of the exact product, within the same bound);
// elsewhere the quotient is divided out exactly. *q receives y or the quotient, for the sub-cell code: any value
// inside the cell serves there, as the order of objects within a cell changes
// no result.
__device__ __forceinline__ double floor_quot(double x, double c, double inv_c, double* q) {
    const double y = x * inv_c;
    const double f = floor(y);
    const double tol = fabs(y) * 0x1p-50 + 0x1p-1000;
    if (y - f > tol && (f + 1.0) - y > tol) {
        *q = y;
        return f;
    }
    *q = xdiv(x, c);
    return floor(*q);
}

// Key of a start-of-step position: realisation index, then compact cell
// coordinates (floor(r / cell), the reference's cell, src/core/collision.cpp:393-395),
// then the Morton code of the sub-cell; sets *bad if the cell lies outside the bounds.
__device__ __forceinline__ unsigned long long cell_key(const GridParams& g, double x, double y, double z,
                                                       unsigned rid, int* bad) {
    double qx, qy, qz;
    const double fx = floor_quot(x, g.cell, g.inv_cell, &qx), fy = floor_quot(y, g.cell, g.inv_cell, &qy),
                 fz = floor_quot(z, g.cell, g.inv_cell, &qz);
    const long long cx = static_cast<long long>(fx) - g.lo[0];
    const long long cy = static_cast<long long>(fy) - g.lo[1];
    const long long cz = static_cast<long long>(fz) - g.lo[2];
    if (cx < 0 || cx > g.span[0] || cy < 0 || cy > g.span[1] || cz < 0 || cz > g.span[2] || g.bits > 62) *bad = 1;
    const unsigned long long cell = (static_cast<unsigned long long>(rid) << (g.w[0] + g.w[1] + g.w[2])) |
                                    (static_cast<unsigned long long>(cx) << (g.w[1] + g.w[2])) |
                                    (static_cast<unsigned long long>(cy) << g.w[2]) |
                                    static_cast<unsigned long long>(cz);
    unsigned long long morton = 0;
    if (g.sub > 0) {
        const unsigned sx = sub_coord(qx, fx, g.sub), sy = sub_coord(qy, fy, g.sub), sz = sub_coord(qz, fz, g.sub);
        for (int b = 0; b < g.sub; ++b)
            morton |= static_cast<unsigned long long>(((sx >> b) & 1u) << (3 * b + 2) | ((sy >> b) & 1u) << (3 * b + 1) |
                                                      ((sz >> b) & 1u) << (3 * b));
    }
    return (cell << (3 * g.sub)) | morton;
}

__device__ __forceinline__ unsigned long long dead_key(const GridParams& g) { return 1ull << min(g.bits, 63); }

// FP32 record of an object whose cell key (sub-cell bits included) is `key`
// and whose start-of-step state is s: position relative to its cell's corner
// and velocity, rounded to FP32 (separately rounded FP64 steps before that).
__device__ __forceinline__ void f32_record(const GridParams& g, unsigned long long key, double x, double y, double z,
                                           double vx, double vy, double vz, float4* __restrict__ out) {
    const unsigned long long cell = key >> (3 * g.sub);
    const unsigned long long mz = (1ull << g.w[2]) - 1, my = (1ull << g.w[1]) - 1, mx = (1ull << g.w[0]) - 1;
    const double cx = xmul(static_cast<double>(static_cast<long long>((cell >> (g.w[1] + g.w[2])) & mx) + g.lo[0]), g.cell);
    const double cy = xmul(static_cast<double>(static_cast<long long>((cell >> g.w[2]) & my) + g.lo[1]), g.cell);
    const double cz = xmul(static_cast<double>(static_cast<long long>(cell & mz) + g.lo[2]), g.cell);
    out[0] = make_float4(static_cast<float>(xsub(x, cx)), static_cast<float>(xsub(y, cy)),
                         static_cast<float>(xsub(z, cz)), 0.0f);
    out[1] = make_float4(static_cast<float>(vx), static_cast<float>(vy), static_cast<float>(vz), 0.0f);
}

// Sort key of object i: the cell key above the object index when packing (the
// sort then carries no index array), else the cell key alone.
__device__ __forceinline__ unsigned long long sort_key(unsigned long long key, int i, int pack_bits) {
    return pack_bits ? (key << pack_bits) | static_cast<unsigned long long>(i) : key;
}
// Flags grids whose keys, dead flag and object index overflow 64 bits.
__device__ __forceinline__ void check_pack_width(const GridParams& g, int pack_bits, Ctrl* ctrl) {
    if (pack_bits && g.bits + 1 + pack_bits > 64) atomicOr(&ctrl->flags, FLAG_PACK_WIDTH);
}

__device__ __forceinline__ unsigned long long hash_slot(unsigned long long k, unsigned long long mask) {
    // 64-bit finaliser (Stafford's mix 13); spreads neighbouring keys.
    k ^= k >> 30; k *= 0xbf58476d1ce4e5b9ull;
    k ^= k >> 27; k *= 0x94d049bb133111ebull;
    k ^= k >> 31;
    return k & mask;
}

__device__ __forceinline__ int hash_find(const unsigned long long* __restrict__ hk, const int* __restrict__ hv,
                                         unsigned long long mask, unsigned long long key) {
    unsigned long long h = hash_slot(key, mask);
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        const unsigned long long k = hk[h];
        if (k == key) return hv[h];
        if (k == kEmpty) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// One 256-bit access (sm_100 ld/st .v8.f32, .v4.u64) for a 32-byte FP32
// record or a four-slot hash bucket: half the load instructions of two
// 16-byte accesses, which is what bounds the cell build's divergent gathers
// and bucket reads. Record arrays and the hash start at allocation
// boundaries, so record i and bucket k sit at 32-byte aligned addresses.
// ld_rec32 reads records no kernel writes while it runs (no memory clobber).
struct __align__(32) Rec32 {
    float4 p, v;
};
__device__ __forceinline__ Rec32 ld_rec32(const float4* q) {
    Rec32 r;
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(r.p.x), "=f"(r.p.y), "=f"(r.p.z), "=f"(r.p.w), "=f"(r.v.x), "=f"(r.v.y), "=f"(r.v.z), "=f"(r.v.w)
                 : "l"(q));
    return r;
}
__device__ __forceinline__ void st_rec32(float4* q, const Rec32& r) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(q), "f"(r.p.x), "f"(r.p.y), "f"(r.p.z),
                 "f"(r.p.w), "f"(r.v.x), "f"(r.v.y), "f"(r.v.z), "f"(r.v.w)
                 : "memory");
}
__device__ __forceinline__ void ld_bucket_cg(const unsigned long long* q, unsigned long long (&e)[4]) {
    asm volatile("ld.global.cg.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(e[0]), "=l"(e[1]), "=l"(e[2]), "=l"(e[3])
                 : "l"(q)
                 : "memory");
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Object states are stored as the reference's State: 6 contiguous doubles
// {rx, ry, rz, vx, vy, vz} (src/core/orbital.hpp:51), read as three 16-byte words.
__device__ __forceinline__ void ld6(const double* __restrict__ base, int64_t i, double s[6]) {
    const double2* p = reinterpret_cast<const double2*>(base + 6 * i);
    const double2 a = p[0], b = p[1], c = p[2];
    s[0] = a.x; s[1] = a.y; s[2] = b.x; s[3] = b.y; s[4] = c.x; s[5] = c.y;
}
__device__ __forceinline__ void st6(double* __restrict__ base, int64_t i, const double s[6]) {
    double2* p = reinterpret_cast<double2*>(base + 6 * i);
    p[0] = make_double2(s[0], s[1]);
    p[1] = make_double2(s[2], s[3]);
    p[2] = make_double2(s[4], s[5]);
}
// Streaming (evict-first) forms for the propagation: each state is read and
// written once per step, so they do not displace the step's keys and records in L2.
__device__ __forceinline__ void ld6s(const double* __restrict__ base, int64_t i, double s[6]) {
    const double2* p = reinterpret_cast<const double2*>(base + 6 * i);
    const double2 a = __ldcs(p), b = __ldcs(p + 1), c = __ldcs(p + 2);
    s[0] = a.x; s[1] = a.y; s[2] = b.x; s[3] = b.y; s[4] = c.x; s[5] = c.y;
}
__device__ __forceinline__ void st6s(double* __restrict__ base, int64_t i, const double s[6]) {
    double2* p = reinterpret_cast<double2*>(base + 6 * i);
    __stcs(p, make_double2(s[0], s[1]));
    __stcs(p + 1, make_double2(s[2], s[3]));
    __stcs(p + 2, make_double2(s[4], s[5]));
}

// Reduces per-thread speculation values over the block and applies them with
// one atomic per quantity per block.
// Squared speeds are accumulated (one square root per block, in flush_spec):
// square roots are correctly rounded and monotone, so the root of the largest
// square is exactly the largest of the roots.
struct SpecAccum {
    double vtrue2, vnext2;
    unsigned long long mn[3], mx[3];
    int alive;
    unsigned long long props;
    int bad;
    __device__ void init() {
        vtrue2 = 0.0; vnext2 = 0.0;
        for (int a = 0; a < 3; ++a) { mn[a] = kEmpty; mx[a] = 0ull; }
        alive = 0; props = 0; bad = 0;
    }
};

__device__ void flush_spec(SpecAccum& s, Ctrl* cur, Ctrl* next, bool screening) {
    __shared__ unsigned long long sh[kWarps][10];
    __shared__ int sh_alive[kWarps], sh_bad[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long vals[10];
    vals[0] = warp_max(static_cast<unsigned long long>(__double_as_longlong(s.vtrue2)));
    vals[1] = warp_max(static_cast<unsigned long long>(__double_as_longlong(s.vnext2)));
    for (int a = 0; a < 3; ++a) { vals[2 + a] = warp_min(s.mn[a]); vals[5 + a] = warp_max(s.mx[a]); }
    vals[8] = warp_sum(s.props);
    vals[9] = 0;
    const int al = warp_sum(s.alive);
    const int bd = warp_max(s.bad);
    if (lane == 0) {
        for (int q = 0; q < 10; ++q) sh[warp][q] = vals[q];
        sh_alive[warp] = al;
        sh_bad[warp] = bd;
    }
    __syncthreads();
    const int nwarps = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        for (int w = 1; w < nwarps; ++w) {
            vals[0] = max(vals[0], sh[w][0]);
            vals[1] = max(vals[1], sh[w][1]);
            for (int a = 0; a < 3; ++a) { vals[2 + a] = min(vals[2 + a], sh[w][2 + a]); vals[5 + a] = max(vals[5 + a], sh[w][5 + a]); }
            vals[8] += sh[w][8];
        }
        int alive = 0, bad = 0;
        for (int w = 0; w < nwarps; ++w) { alive += sh_alive[w]; bad |= sh_bad[w]; }
        atomicAdd(&cur->n_alive, alive);
        atomicAdd(&cur->object_steps, vals[8]);
        if (screening) {
            // Bit patterns of non-negative doubles order like their values.
            const double vt = xsqrt(__longlong_as_double(static_cast<long long>(vals[0])));
            const double vn = xsqrt(__longlong_as_double(static_cast<long long>(vals[1])));
            atomicMax(&cur->vmax_true, static_cast<unsigned long long>(__double_as_longlong(vt)));
            atomicMax(&next->spec_vmax, static_cast<unsigned long long>(__double_as_longlong(vn)));
            for (int a = 0; a < 3; ++a) {
                atomicMin(&next->bb_min[a], vals[2 + a]);
                atomicMax(&next->bb_max[a], vals[5 + a]);
            }
            if (bad) atomicOr(&cur->flags, FLAG_KEY_RANGE);
        }
    }
}

// ---------------------------------------------------------------------------
// Chunk bookkeeping
// ---------------------------------------------------------------------------

__device__ void ctrl_reset(Ctrl& c) {
    c.spec_vmax = 0ull;
    for (int a = 0; a < 3; ++a) { c.bb_min[a] = kEmpty; c.bb_max[a] = 0ull; }
    c.vmax_true = 0ull;
    c.candidates = c.co_orbiting = c.refined = c.conj = c.object_steps = c.exact_evals = 0ull;
    c.n_alive = c.n_cells = c.max_cell = c.flags = 0;
    c.n_items = 0u;
    c.item_ticket = 0u;
    c.n_coll = 0u;
    c.grid = GridParams{};
}

// ctrl[0..k) reset; ctrl[0] takes the carried speculation, the carry slot is reset.
__global__ void k_chunk_init(Ctrl* ctrl, int k_steps, Ctrl* carry, ChunkCtrl* chunk, Ctrl* carry_ckpt) {
    __shared__ Ctrl saved;
    if (threadIdx.x == 0) {
        saved = *carry;
        if (carry_ckpt) *carry_ckpt = saved;  // the chunk's checkpoint of the carried speculation
    }
    __syncthreads();
    for (int s = threadIdx.x; s < k_steps; s += blockDim.x) ctrl_reset(ctrl[s]);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctrl[0].spec_vmax = saved.spec_vmax;
        for (int a = 0; a < 3; ++a) { ctrl[0].bb_min[a] = saved.bb_min[a]; ctrl[0].bb_max[a] = saved.bb_max[a]; }
        ctrl_reset(*carry);
        chunk->conj_count = 0ull;
        chunk->flags = 0;
        chunk->halt_step = -1;
        chunk->events = 0u;
    }
}

__global__ void k_ctrl_reset(Ctrl* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctrl_reset(*c);
}

// Speed and position bounds over alive objects of one state buffer.
__global__ void k_seed_ctrl(const double* __restrict__ st, const uint8_t* __restrict__ alive, int n, Ctrl* target) {
    SpecAccum s;
    s.init();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!alive[i]) continue;
        double x[6];
        ld6(st, i, x);
        s.vnext2 = fmax(s.vnext2, xdot3(x[3], x[4], x[5]));
        for (int a = 0; a < 3; ++a) {
            const unsigned long long e = enc_double(x[a]);
            s.mn[a] = min(s.mn[a], e);
            s.mx[a] = max(s.mx[a], e);
        }
    }
    __shared__ Ctrl dummy;
    if (threadIdx.x == 0) ctrl_reset(dummy);
    __syncthreads();
    flush_spec(s, &dummy, target, true);
}

// ---------------------------------------------------------------------------
// Propagation
// ---------------------------------------------------------------------------

// Radix digit histogram of the keys a block emits (all sort passes at once),
// aggregated per warp with __match_any_sync and flushed once per block.
__device__ __forceinline__ void hist_zero(unsigned int* sh, int passes) {
    for (int t = threadIdx.x; t < passes * 256; t += blockDim.x) sh[t] = 0u;
}
// Called by all 32 lanes; `have` marks lanes holding a key. The top pass's
// digits are nearly all equal, so that pass is aggregated over the warp; the
// lower passes' digits are spread and go straight to shared atomics.
__device__ __forceinline__ void warp_hist_add(unsigned int* sh, bool have, unsigned long long key, int passes,
                                              int lane) {
    for (int pass = 0; pass + 1 < passes; ++pass)
        if (have) atomicAdd(&sh[pass * 256 + static_cast<unsigned>((key >> (8 * pass)) & 0xFF)], 1u);
    const int top = passes - 1;
    const unsigned d = have ? static_cast<unsigned>((key >> (8 * top)) & 0xFF) : 256u + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (have && lane == __ffs(peers) - 1) atomicAdd(&sh[top * 256 + d], __popc(peers));
}
__device__ __forceinline__ void hist_flush(const unsigned int* sh, unsigned int* hist, int passes) {
    for (int t = threadIdx.x; t < passes * 256; t += blockDim.x) {
        const unsigned int v = sh[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kPropBlock, kMinBlocks) k_propagate_exact(StepArgs a, const double* __restrict__ in,
                                                            double* __restrict__ out,
                                                            const uint8_t* __restrict__ alive_in,
                                                            uint8_t* __restrict__ alive_out,
                                                            unsigned long long* __restrict__ keys) {
    if (step_void(a.ctrl)) return;  // an earlier step of the chunk was left void
    const int n = live_n(a);
    __shared__ GridParams g;
    __shared__ MoonStage moon[3];
    if (threadIdx.x == 0) {
        if (a.screening)
            make_grid(__longlong_as_double(static_cast<long long>(a.ctrl->spec_vmax)), a.ctrl->bb_min,
                      a.ctrl->bb_max, a.dt, a.threshold_km, a.tune.subcell_bits, a.rbits, a.tune.cell_scale, g);
        for (int q = 0; q < 3; ++q) moon[q] = a.sp->m[q];
        if (blockIdx.x == 0 && a.screening) {
            a.ctrl->grid = g;
            check_pack_width(g, a.pack_bits, a.ctrl);
        }
    }
    __shared__ unsigned int sh_hist[8 * 256];
    const bool with_hist = a.screening && a.hist != nullptr;
    if (with_hist) hist_zero(sh_hist, a.sort_passes);
    __syncthreads();
    const ForceConsts fc = a.fc;
    SpecAccum acc;
    acc.init();
    const int lane = threadIdx.x & 31;
    // Warp-uniform loop (whole warps iterate together) so that the digit
    // histogram can aggregate over the warp.
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        unsigned long long out_key = 0ull;
        if (i < n) {
            double s[6];
            ld6s(in, i, s);
            if (!alive_in[i]) {
                st6s(out, i, s);
                alive_out[i] = 0;
                out_key = dead_key(g);
            } else {
                acc.props += 1;
                unsigned long long key = 0ull;
                double vb2 = 0.0;
                if (a.screening) {
                    key = cell_key(g, s[0], s[1], s[2], a.real_id ? a.real_id[i] : 0u, &acc.bad);
                    vb2 = xdot3(s[3], s[4], s[5]);
                    if (a.rec32) f32_record(g, key, s[0], s[1], s[2], s[3], s[4], s[5], a.rec32 + 2 * static_cast<int64_t>(i));
                }
                rk4_exact(fc, a.dt, moon[0], moon[1], moon[2], s);
                st6s(out, i, s);
                // Re-entry (src/core/orbital.cpp:297).
                const bool alive = !(xsqrt(xdot3(s[0], s[1], s[2])) < fc.r_earth);
                alive_out[i] = alive ? 1 : 0;
                if (alive) {
                    acc.alive += 1;
                    if (a.screening) {
                        acc.vtrue2 = fmax(acc.vtrue2, vb2);
                        acc.vnext2 = fmax(acc.vnext2, xdot3(s[3], s[4], s[5]));
                        for (int q = 0; q < 3; ++q) {
                            const unsigned long long e = enc_double(s[q]);
                            acc.mn[q] = min(acc.mn[q], e);
                            acc.mx[q] = max(acc.mx[q], e);
                        }
                    }
                }
                out_key = alive ? key : dead_key(g);
            }
            if (a.screening) keys[i] = sort_key(out_key, i, a.pack_bits);
        }
        if (with_hist) {
            __syncwarp();
            warp_hist_add(sh_hist, i < n, out_key, a.sort_passes, lane);
        }
    }
    if (with_hist) {
        __syncthreads();
        hist_flush(sh_hist, a.hist, a.sort_passes);
    }
    flush_spec(acc, a.ctrl, a.ctrl_next, a.screening != 0);
}

// Fragments born inside a step, carried from their event to the end of the
// step (src/core/breakup.cpp:304-306): one RK4 step of the event's remaining
// time with its lunar stages (none when the event closes the step), then
// alive unless below the surface. Row first + k belongs to span row_span[k].
__global__ void __launch_bounds__(kPropBlock) k_advance_spans(ForceConsts fc, const FragSpan* __restrict__ spans,
                                                               const int* __restrict__ row_span, int64_t first,
                                                               int count, double* __restrict__ state,
                                                               uint8_t* __restrict__ alive) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    const FragSpan& sp = spans[row_span[k]];
    double s[6];
    ld6(state, i, s);
    if (sp.dt > 0) {
        rk4_exact(fc, sp.dt, sp.m[0], sp.m[1], sp.m[2], s);
        st6(state, i, s);
    }
    alive[i] = xsqrt(xdot3(s[0], s[1], s[2])) >= fc.r_earth ? 1 : 0;
}

// rows[2q] / rows[2q+1] = start / end-of-step state of object idx[q].
__global__ void __launch_bounds__(kBlock) k_gather_rows(const double* __restrict__ before,
                                                        const double* __restrict__ after,
                                                        const int64_t* __restrict__ idx, int count,
                                                        double* __restrict__ rows) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 12 * count) return;
    const int q = t / 12, c = t % 12;
    rows[12 * static_cast<int64_t>(q) + c] = (c < 6 ? before : after)[6 * idx[q] + (c % 6)];
}

__global__ void __launch_bounds__(kBlock) k_clear_alive(uint8_t* __restrict__ alive, const int64_t* __restrict__ idx,
                                                        int count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) alive[idx[t]] = 0;
}

// Split-precision propagation (FP32 J2 and lunar terms, FP64 state and central
// term); keys and speculation exactly as in k_propagate_exact.
__global__ void __launch_bounds__(kPropBlock, 5) k_propagate_split(StepArgs a, const double* __restrict__ in,
                                                                   double* __restrict__ out,
                                                                   const uint8_t* __restrict__ alive_in,
                                                                   uint8_t* __restrict__ alive_out,
                                                                   unsigned long long* __restrict__ keys) {
    if (step_void(a.ctrl)) return;  // an earlier step of the chunk was left void
    const int n = live_n(a);
    __shared__ GridParams g;
    __shared__ MoonStageF moon[3];
    if (threadIdx.x == 0) {
        if (a.screening)
            make_grid(__longlong_as_double(static_cast<long long>(a.ctrl->spec_vmax)), a.ctrl->bb_min,
                      a.ctrl->bb_max, a.dt, a.threshold_km, a.tune.subcell_bits, a.rbits, a.tune.cell_scale, g);
        for (int q = 0; q < 3; ++q) moon[q] = to_f32(a.sp->m[q]);
        if (blockIdx.x == 0 && a.screening) {
            a.ctrl->grid = g;
            check_pack_width(g, a.pack_bits, a.ctrl);
        }
    }
    __shared__ unsigned int sh_hist[8 * 256];
    const bool with_hist = a.screening && a.hist != nullptr;
    if (with_hist) hist_zero(sh_hist, a.sort_passes);
    __syncthreads();
    const SplitConsts sc{-a.fc.neg_mu_earth, static_cast<float>(a.fc.k_j2), static_cast<float>(a.fc.mu_moon)};
    const double re2 = a.fc.r_earth * a.fc.r_earth;
    SpecAccum acc;
    acc.init();
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        unsigned long long out_key = 0ull;
        if (i < n) {
            double s[6];
            ld6s(in, i, s);
            if (!alive_in[i]) {
                st6s(out, i, s);
                alive_out[i] = 0;
                out_key = dead_key(g);
            } else {
                acc.props += 1;
                unsigned long long key = 0ull;
                double vb2 = 0.0;
                if (a.screening) {
                    key = cell_key(g, s[0], s[1], s[2], a.real_id ? a.real_id[i] : 0u, &acc.bad);
                    vb2 = xdot3(s[3], s[4], s[5]);
                    if (a.rec32) f32_record(g, key, s[0], s[1], s[2], s[3], s[4], s[5], a.rec32 + 2 * static_cast<int64_t>(i));
                }
                rk4_split(sc, a.dt, moon[0], moon[1], moon[2], s);
                st6s(out, i, s);
                const bool alive = !(fma(s[0], s[0], fma(s[1], s[1], s[2] * s[2])) < re2);
                alive_out[i] = alive ? 1 : 0;
                if (alive) {
                    acc.alive += 1;
                    if (a.screening) {
                        acc.vtrue2 = fmax(acc.vtrue2, vb2);
                        acc.vnext2 = fmax(acc.vnext2, xdot3(s[3], s[4], s[5]));
                        for (int q = 0; q < 3; ++q) {
                            const unsigned long long e = enc_double(s[q]);
                            acc.mn[q] = min(acc.mn[q], e);
                            acc.mx[q] = max(acc.mx[q], e);
                        }
                    }
                }
                out_key = alive ? key : dead_key(g);
            }
            if (a.screening) keys[i] = sort_key(out_key, i, a.pack_bits);
        }
        if (with_hist) {
            __syncwarp();
            warp_hist_add(sh_hist, i < n, out_key, a.sort_passes, lane);
        }
    }
    if (with_hist) {
        __syncthreads();
        hist_flush(sh_hist, a.hist, a.sort_passes);
    }
    flush_spec(acc, a.ctrl, a.ctrl_next, a.screening != 0);
}

// Keys for one-shot screening of given states: alive_after selects the objects,
// positions come from the start-of-step buffer. ctrl->spec_* already hold the
// bounds of exactly these objects, so the speculation is the true grid.
__global__ void __launch_bounds__(kBlock) k_screen_keys(StepArgs a, const double* __restrict__ before,
                                                        const uint8_t* __restrict__ alive_after,
                                                        unsigned long long* __restrict__ keys) {
    __shared__ GridParams g;
    if (threadIdx.x == 0) {
        make_grid(__longlong_as_double(static_cast<long long>(a.ctrl->spec_vmax)), a.ctrl->bb_min,
                  a.ctrl->bb_max, a.dt, a.threshold_km, a.tune.subcell_bits, a.rbits, a.tune.cell_scale, g);
        if (blockIdx.x == 0) {
            a.ctrl->grid = g;
            a.ctrl->vmax_true = a.ctrl->spec_vmax;
            check_pack_width(g, a.pack_bits, a.ctrl);
            if (g.bits + 1 > 8 * a.sort_passes) atomicOr(&a.ctrl->flags, FLAG_SORT_BITS);
        }
    }
    __syncthreads();
    const int n = live_n(a);
    int bad = 0, alive = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (alive_after[i]) {
            const double* s = before + 6 * static_cast<int64_t>(i);
            const unsigned long long key = cell_key(g, s[0], s[1], s[2], a.real_id ? a.real_id[i] : 0u, &bad);
            if (a.rec32) f32_record(g, key, s[0], s[1], s[2], s[3], s[4], s[5], a.rec32 + 2 * static_cast<int64_t>(i));
            keys[i] = sort_key(key, i, a.pack_bits);
            ++alive;
        } else {
            keys[i] = sort_key(dead_key(g), i, a.pack_bits);
        }
    }
    alive = warp_sum(alive);
    bad = warp_max(bad);
    if ((threadIdx.x & 31) == 0) {
        if (alive) atomicAdd(&a.ctrl->n_alive, alive);
        if (bad) atomicOr(&a.ctrl->flags, FLAG_KEY_RANGE);
    }
}

// When an object holding the top start speed re-entered during the step, the
// grid of the reference (speeds of objects alive AFTER the step,
// src/core/collision.cpp:339-356) is smaller than the speculated one: rebuild
// the keys with it. Otherwise every block returns at once.
__global__ void __launch_bounds__(kBlock) k_fix_keys(StepArgs a, const double* __restrict__ before,
                                                     const uint8_t* __restrict__ alive_after,
                                                     unsigned long long* __restrict__ keys) {
    if (step_void(a.ctrl)) return;
    const int n = live_n(a);
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.ctrl->grid.bits + 1 > 8 * a.sort_passes)
        atomicOr(&a.ctrl->flags, FLAG_SORT_BITS);  // more key bits than the sort's passes cover
    const unsigned long long vt = a.ctrl->vmax_true;
    if (vt == a.ctrl->spec_vmax) return;
    __shared__ GridParams g;
    if (threadIdx.x == 0) {
        make_grid(__longlong_as_double(static_cast<long long>(vt)), a.ctrl->bb_min, a.ctrl->bb_max, a.dt,
                  a.threshold_km, a.tune.subcell_bits, a.rbits, a.tune.cell_scale, g);
        if (blockIdx.x == 0) {
            a.ctrl->grid = g;
            atomicOr(&a.ctrl->flags, FLAG_KEYS_REBUILT);
            check_pack_width(g, a.pack_bits, a.ctrl);
            if (g.bits + 1 > 8 * a.sort_passes) atomicOr(&a.ctrl->flags, FLAG_SORT_BITS);
        }
    }
    // The propagation's digit histogram describes the old keys: the rebuilt
    // keys' digits are counted into the histogram's second half (cleared with
    // the first before the step), which the sort then reads.
    __shared__ unsigned int sh_hist[8 * 256];
    unsigned int* hist_rebuilt = a.hist ? a.hist + 8 * 256 : nullptr;
    if (hist_rebuilt) hist_zero(sh_hist, a.sort_passes);
    __syncthreads();
    int bad = 0;
    const int lane = threadIdx.x & 31;
    // Warp-uniform loop: the digit counts aggregate over whole warps.
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        unsigned long long key = dead_key(g);
        if (i < n) {
            if (alive_after[i]) {
                const double* s = before + 6 * static_cast<int64_t>(i);
                key = cell_key(g, s[0], s[1], s[2], a.real_id ? a.real_id[i] : 0u, &bad);
                if (a.rec32)
                    f32_record(g, key, s[0], s[1], s[2], s[3], s[4], s[5], a.rec32 + 2 * static_cast<int64_t>(i));
            }
            keys[i] = sort_key(key, i, a.pack_bits);
        }
        if (hist_rebuilt) {
            __syncwarp();
            warp_hist_add(sh_hist, i < n, key, a.sort_passes, lane);
        }
    }
    if (hist_rebuilt) {
        __syncthreads();
        hist_flush(sh_hist, hist_rebuilt, a.sort_passes);
    }
    bad = warp_max(bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(&a.ctrl->flags, FLAG_KEY_RANGE);
}

// ---------------------------------------------------------------------------
// Block and single-block exclusive scans of u32 counters
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned int block_exclusive_scan(unsigned int v, unsigned int* total) {
    __shared__ unsigned int wsum[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    unsigned int off = 0, tot = 0;
    for (int w = 0; w < kWarps; ++w) {
        if (w < warp) off += wsum[w];
        tot += wsum[w];
    }
    __syncthreads();
    *total = tot;
    return off + incl - v;
}

// Exclusive scan in place, one block, coalesced rounds of 1024 entries.
// Optionally stores the grand total.
// With n_cells, the length is per_chunk entries per chunk of kBlock cells.
__global__ void __launch_bounds__(1024) k_scan_small(unsigned int* __restrict__ v, int len,
                                                     unsigned int* __restrict__ total, const int* n_cells,
                                                     int per_chunk) {
    if (n_cells) len = min(len, per_chunk * ((*n_cells + kBlock - 1) / kBlock));
    __shared__ unsigned int wsum[32];
    __shared__ unsigned int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = 0; r < len; r += 1024) {
        const int p = r + threadIdx.x;
        const unsigned int x = p < len ? v[p] : 0u;
        unsigned int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            unsigned int t = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[lane] = t;
        }
        __syncthreads();
        const unsigned int c = carry;
        if (p < len) v[p] = c + incl - x + (warp > 0 ? wsum[warp - 1] : 0u);
        __syncthreads();
        if (threadIdx.x == 0) carry = c + wsum[31];
        __syncthreads();
    }
    if (total && threadIdx.x == 0) *total = carry;
}

// ---------------------------------------------------------------------------
// Radix sort: LSD, 8-bit digits, one pass per digit with decoupled look-back
// (each tile publishes its digit counts, then sums its predecessors' counts).
// ---------------------------------------------------------------------------

constexpr unsigned int kStatAgg = 1u << 30;   // tile's own count is published
constexpr unsigned int kStatInc = 2u << 30;   // count includes all previous tiles
constexpr unsigned int kStatMask = (1u << 30) - 1;
constexpr int kLookbackLimit = 1 << 22;       // polls before a wait gives up (default)

__device__ __forceinline__ unsigned int ld_relaxed(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned int* p, unsigned int v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}



// Lanes of the warp holding the same DB-bit digit as this lane, among the
// lanes with `valid` set: either the hardware match, or DB ballots (one per
// digit bit) intersected. The ballot form issues more instructions but each has the
// short latency of a vote.
template <int DB = 8>
__device__ __forceinline__ unsigned digit_peers(unsigned d, bool valid, bool by_ballot) {
    if (!by_ballot) return __match_any_sync(0xffffffffu, valid ? d : (1u << DB) + (threadIdx.x & 31));
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < DB; ++b) {
        const bool bit = (d >> b) & 1u;
        const unsigned bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Digit histograms of every pass in one read of the keys.
// only_if_rebuilt: the propagation already counted the digits; recount only
// if k_fix_keys rebuilt the keys (it cleared the histogram then).
__global__ void __launch_bounds__(kBlock) k_sort_upsweep(const unsigned long long* __restrict__ keys, int n,
                                                         const int* __restrict__ n_dev, int passes,
                                                         unsigned int* __restrict__ hist, const Ctrl* ctrl,
                                                         int only_if_rebuilt, int shift0) {
    __shared__ unsigned int h[8][256];
    if (only_if_rebuilt && !(ctrl->flags & FLAG_KEYS_REBUILT)) return;
    if (n_dev) n = min(n, *n_dev);
    if (blockIdx.x * kSortTile >= n) return;
    for (int p = 0; p < 8; ++p) h[p][threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < kSortItems; ++j) {
        const int p = base + j * kBlock + threadIdx.x;
        const bool valid = p < n;
        const unsigned long long k = valid ? keys[p] : 0ull;
        for (int pass = 0; pass < passes; ++pass) {
            const unsigned d = valid ? static_cast<unsigned>((k >> (shift0 + 8 * pass)) & 0xFF) : 256u + lane;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[pass][d], __popc(peers));
        }
    }
    __syncthreads();
    for (int pass = 0; pass < passes; ++pass) {
        const unsigned int c = h[pass][threadIdx.x];
        if (c) atomicAdd(&hist[pass * 256 + threadIdx.x], c);
    }
}

__global__ void __launch_bounds__(kBlock) k_sort_onesweep(const unsigned long long* __restrict__ keys_in,
                                                          const int* __restrict__ idx_in,
                                                          unsigned long long* __restrict__ keys_out,
                                                          int* __restrict__ idx_out, int n,
                                                          const int* __restrict__ n_dev, int shift,
                                                          const unsigned int* __restrict__ digit_hist,
                                                          const unsigned int* __restrict__ digit_hist_rebuilt,
                                                          unsigned int* __restrict__ status,
                                                          unsigned int* __restrict__ ticket, int* flags,
                                                          int packed, int poll_limit, int rank_by_ballot) {
    __shared__ unsigned int wcnt[kWarps][256];
    __shared__ int gbase[256];
    __shared__ unsigned long long skeys[kSortTile];
    __shared__ int sidx[kSortTile];
    __shared__ int tile_sh;
    __shared__ int timed_out;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        tile_sh = static_cast<int>(atomicAdd(ticket, 1u));  // tiles start in ticket order
        timed_out = 0;
    }
    for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
    if (n_dev) n = min(n, *n_dev);
    __syncthreads();
    const int tile = tile_sh;
    const int tile0 = tile * kSortTile;
    if (tile0 >= n) return;  // tickets are in order: no later tile waits on this one
    const int count = min(kSortTile, n - tile0);
    // Where each digit's keys start in the output: exclusive scan of the pass's histogram.
    unsigned int hist_total;
    // Keys rebuilt by k_fix_keys after the propagation counted them: their
    // own digit counts.
    const unsigned int* hist = (digit_hist_rebuilt && (*flags & FLAG_KEYS_REBUILT)) ? digit_hist_rebuilt : digit_hist;
    const unsigned int digit_start = block_exclusive_scan(hist[threadIdx.x], &hist_total);

    constexpr int kPerWarp = kSortTile / kWarps;
    constexpr int kRounds = kPerWarp / 32;
    unsigned long long k[kRounds];
    int id[kRounds];
    unsigned d[kRounds];
    // Every load of the thread in flight first, then the ranking.
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const int l = warp * kPerWarp + r * 32 + lane;
        const bool valid = l < count;
        const int p = tile0 + l;
        k[r] = valid ? keys_in[p] : 0ull;
        id[r] = (valid && !packed) ? (idx_in ? idx_in[p] : p) : 0;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const bool valid = (warp * kPerWarp + r * 32 + lane) < count;
        d[r] = valid ? static_cast<unsigned>((k[r] >> shift) & 0xFF) : 256u + lane;
        const unsigned peers = digit_peers(d[r] & 0xFFu, valid, rank_by_ballot != 0);
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // Thread t owns digit t.
    const int t = threadIdx.x;
    unsigned int tot = 0;
    for (int w = 0; w < kWarps; ++w) tot += wcnt[w][t];
    unsigned int* my = status + static_cast<int64_t>(tile) * 256 + t;
    st_relaxed(my, (tile == 0 ? kStatInc : kStatAgg) | tot);
    unsigned int excl = 0;
    if (tile > 0) {
        int j = tile - 1;
        int polls = 0;
        while (true) {
            const unsigned int v = ld_relaxed(status + static_cast<int64_t>(j) * 256 + t);
            const unsigned int flag = v & ~kStatMask;
            if (flag == 0) {
                if (++polls > poll_limit) {
                    timed_out = 1;
                    break;
                }
                continue;
            }
            excl += v & kStatMask;
            if (flag == kStatInc) break;
            --j;
        }
        st_relaxed(my, kStatInc | (excl + tot));
    }
    unsigned int unused;
    const unsigned int start = block_exclusive_scan(tot, &unused);
    gbase[t] = static_cast<int>(digit_start + excl) - static_cast<int>(start);
    unsigned int run = start;
    for (int w = 0; w < kWarps; ++w) {
        const unsigned int c = wcnt[w][t];
        wcnt[w][t] = run;
        run += c;
    }
    __syncthreads();
    if (timed_out) {
        if (threadIdx.x == 0) atomicOr(flags, FLAG_TIMEOUT);
        return;  // results of this step are discarded by the host
    }
    for (int r = 0; r < kRounds; ++r) {
        const bool valid = (warp * kPerWarp + r * 32 + lane) < count;
        const unsigned peers = digit_peers(d[r] & 0xFFu, valid, rank_by_ballot != 0);
        if (valid) {
            const unsigned pos = wcnt[warp][d[r]] + __popc(peers & lanemask_lt());
            skeys[pos] = k[r];
            if (!packed) sidx[pos] = id[r];
        }
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int l = threadIdx.x; l < count; l += kBlock) {
        const unsigned long long kk = skeys[l];
        const int dst = gbase[static_cast<unsigned>((kk >> shift) & 0xFF)] + l;
        if (dst >= 0 && dst < n) {
            keys_out[dst] = kk;
            if (!packed) idx_out[dst] = sidx[l];
        }
    }
}

// ---------------------------------------------------------------------------
// Cells
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_cell_count(const unsigned long long* __restrict__ keys,
                                                       const Ctrl* __restrict__ ctrl, unsigned int* __restrict__ counts,
                                                       int pack_bits) {
    if (step_void(ctrl)) return;
    const int m = ctrl->n_alive;
    const int shift = 3 * ctrl->grid.sub + pack_bits;
    const int base = blockIdx.x * kCellTile;
    int c = 0;
    for (int j = threadIdx.x; j < kCellTile; j += kBlock) {
        const int p = base + j;
        if (p < m && (p == 0 || (keys[p] >> shift) != (keys[p - 1] >> shift))) ++c;
    }
    c = warp_sum(c);
    __shared__ int sh[kWarps];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kWarps; ++w) t += sh[w];
        counts[blockIdx.x] = t;
    }
}

// Cell ranges and hash entries; gathers start-of-step states in sorted order.
__global__ void __launch_bounds__(kBlock) k_cell_write(const unsigned long long* __restrict__ keys,
                                                       const int* __restrict__ idx,
                                                       const unsigned int* __restrict__ offsets, Ctrl* ctrl,
                                                       int* __restrict__ cell_begin,
                                                       unsigned long long* __restrict__ cell_key_out,
                                                       unsigned long long* __restrict__ hk, int* __restrict__ hv,
                                                       unsigned long long hmask, const double* __restrict__ before,
                                                       double* __restrict__ sorted,
                                                       int* __restrict__ sorted_orig, float4* __restrict__ sorted32,
                                                       const float4* __restrict__ rec32, int pack_bits) {
    if (step_void(ctrl)) return;
    constexpr int kPer = kCellTile / kBlock;  // consecutive entries per thread
    const int m = ctrl->n_alive;
    if (m == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { ctrl->n_cells = 0; cell_begin[0] = 0; }
        return;
    }
    if (blockIdx.x * kCellTile >= m) return;
    const int p0 = blockIdx.x * kCellTile + threadIdx.x * kPer;
    const int sh = 3 * ctrl->grid.sub + pack_bits;
    const unsigned long long idx_mask = pack_bits ? (1ull << pack_bits) - 1 : 0ull;
    int heads[kPer];
    unsigned int local = 0;
    for (int j = 0; j < kPer; ++j) {
        const int p = p0 + j;
        heads[j] = (p < m && (p == 0 || (keys[p] >> sh) != (keys[p - 1] >> sh))) ? 1 : 0;
        local += heads[j];
    }
    unsigned int unused;
    int run = static_cast<int>(offsets[blockIdx.x] + block_exclusive_scan(local, &unused));
    for (int j = 0; j < kPer; ++j) {
        const int p = p0 + j;
        if (p >= m) break;
        run += heads[j];
        const int cid = run - 1;
        if (heads[j]) {
            const unsigned long long key = keys[p] >> sh;  // cell part
            cell_begin[cid] = p;
            cell_key_out[cid] = key;
            unsigned long long h = hash_slot(key, hmask);
            for (unsigned long long probe = 0; probe <= hmask; ++probe) {
                const unsigned long long prev = atomicCAS(&hk[h], kEmpty, key);
                if (prev == kEmpty || prev == key) { hv[h] = cid; break; }
                h = (h + 1) & hmask;
            }
        }
        if (p == m - 1) {
            ctrl->n_cells = cid + 1;
            cell_begin[cid + 1] = m;
        }
    }
    // Gather in sorted order: entries strided across the block so that stores
    // coalesce, every load of a thread's entries issued before the first store.
    __shared__ GridParams g;
    if (threadIdx.x == 0) g = ctrl->grid;
    __syncthreads();
    const int base = blockIdx.x * kCellTile + threadIdx.x;
    int o[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int p = base + j * kBlock;
        o[j] = p < m ? (pack_bits ? static_cast<int>(keys[p] & idx_mask) : idx[p]) : -1;
    }
    if (!sorted) {
        // FP32 records only: the ones written with the keys (one 32-byte row each).
        float4 r[kPer][2];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (o[j] < 0) continue;
            r[j][0] = rec32[2 * static_cast<int64_t>(o[j])];
            r[j][1] = rec32[2 * static_cast<int64_t>(o[j]) + 1];
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int p = base + j * kBlock;
            if (o[j] < 0) continue;
            sorted_orig[p] = o[j];
            sorted32[2 * static_cast<int64_t>(p)] = r[j][0];
            sorted32[2 * static_cast<int64_t>(p) + 1] = r[j][1];
        }
        return;
    }
    // FP64 states (random rows of `before`), and FP32 records from them when asked.
    double2 st[kPer][3];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        if (o[j] < 0) continue;
        const double2* src = reinterpret_cast<const double2*>(before + 6 * static_cast<int64_t>(o[j]));
        st[j][0] = src[0];
        st[j][1] = src[1];
        st[j][2] = src[2];
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int p = base + j * kBlock;
        if (o[j] < 0) continue;
        sorted_orig[p] = o[j];
        double2* dst = reinterpret_cast<double2*>(sorted + 6 * static_cast<int64_t>(p));
        dst[0] = st[j][0];
        dst[1] = st[j][1];
        dst[2] = st[j][2];
        if (sorted32)
            f32_record(g, keys[p] >> pack_bits, st[j][0].x, st[j][0].y, st[j][1].x, st[j][1].y, st[j][2].x,
                       st[j][2].y, sorted32 + 2 * static_cast<int64_t>(p));
    }
}

// Thread per (cell, forward neighbour): the neighbour's cell index or -1.
__global__ void __launch_bounds__(kBlock) k_neighbours(Ctrl* ctrl, const unsigned long long* __restrict__ cell_key_in,
                                                       const unsigned long long* __restrict__ hk,
                                                       const int* __restrict__ hv, unsigned long long hmask,
                                                       int* __restrict__ nbr) {
    if (step_void(ctrl)) return;
    const int nc = ctrl->n_cells;
    const GridParams g = ctrl->grid;
    const unsigned long long mz = (1ull << g.w[2]) - 1, my = (1ull << g.w[1]) - 1;
    const int64_t total = 13 * static_cast<int64_t>(nc);
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(t / 13), o = static_cast<int>(t - 13 * static_cast<int64_t>(c));
        int dx, dy, dz;
        forward_offset(o, dx, dy, dz);
        const unsigned long long key = cell_key_in[c];
        const unsigned long long rid = key >> (g.w[0] + g.w[1] + g.w[2]);
        const long long x = static_cast<long long>((key >> (g.w[1] + g.w[2])) & ((1ull << g.w[0]) - 1)) + dx;
        const long long y = static_cast<long long>((key >> g.w[2]) & my) + dy;
        const long long z = static_cast<long long>(key & mz) + dz;
        int found = -1;
        if (x >= 0 && x <= g.span[0] && y >= 0 && y <= g.span[1] && z >= 0 && z <= g.span[2]) {
            const unsigned long long nk = (rid << (g.w[0] + g.w[1] + g.w[2])) |
                                          (static_cast<unsigned long long>(x) << (g.w[1] + g.w[2])) |
                                          (static_cast<unsigned long long>(y) << g.w[2]) |
                                          static_cast<unsigned long long>(z);
            found = hash_find(hk, hv, hmask, nk);
        }
        nbr[t] = found;
    }
}

// A cell's column list for the pair kernel, 16 int2: entries 0..nseg-1 the
// (first column, first sorted position) of each non-empty segment (the cell
// itself, then its forward neighbours in offset order); entry 14 the
// segments' ids, 4 bits each (0 the cell, 1 + o forward neighbour o); entry
// 15 (column-list length L, nseg). One warp reads it in one 128-byte load.
__device__ __forceinline__ void write_column_table(int2* __restrict__ t, int b0, int k, const int (&nb_begin)[13],
                                                   const int (&nb_len)[13]) {
    unsigned long long ids = 0;
    int nseg = 1, start = k;
    t[0] = make_int2(0, b0);
#pragma unroll
    for (int o = 0; o < 13; ++o) {
        if (nb_len[o] <= 0) continue;
        t[nseg] = make_int2(start, nb_begin[o]);
        ids |= static_cast<unsigned long long>(o + 1) << (4 * nseg);
        ++nseg;
        start += nb_len[o];
    }
    t[14] = make_int2(static_cast<int>(static_cast<unsigned int>(ids)), static_cast<int>(static_cast<unsigned int>(ids >> 32)));
    t[15] = make_int2(start, nseg);
}

// A pair work item, int4: (cell, row block | column blocks << 24, first column
// block, the cell's first sorted position).
__device__ __forceinline__ int4 work_item(int c, int row_block, int col_block, int col_blocks, int b0) {
    return make_int4(c, row_block | (col_blocks << 24), col_block, b0);
}

// Number of work items of row block a: its column blocks a .. tc-1 in groups.
__device__ __forceinline__ unsigned int row_block_items(int a, int tc, int per) {
    return static_cast<unsigned int>((tc - a + per - 1) / per);
}

// Cells whose items are expensive (more than one row block, or a long column
// list): their items are handed out first, so that the pair kernel ends on
// cheap items (largest first).
__device__ __forceinline__ bool heavy_cell(int k, int L) { return k > 32 || L > 128; }

// Items of a cell with ta row blocks over tc column blocks.
__device__ __forceinline__ unsigned int cell_items(int ta, int tc, int per) {
    unsigned int items = 0;
    for (int a = 0; a < ta; ++a) items += row_block_items(a, tc, per);
    return items;
}

// Lane per cell: the length L of the cell's column list (own objects plus the
// forward neighbours'), the candidate-pair count k(k-1)/2 + k(L-k) (the pairs
// the reference visits, src/core/collision.cpp:522-538), and per chunk of
// kBlock cells the number of heavy cells' work items (part[chunk]) and of
// light cells' (part[chunks + chunk]), so that one scan of part places every
// heavy item before every light item, each group in cell order.
__global__ void __launch_bounds__(kBlock) k_items_count(Ctrl* ctrl, const int* __restrict__ cell_begin,
                                                        const int* __restrict__ nbr, int* __restrict__ cell_len,
                                                        int2* __restrict__ col_tab, unsigned int* __restrict__ part,
                                                        int per) {
    if (step_void(ctrl)) return;
    const int nc = ctrl->n_cells;
    const int chunks = (nc + kBlock - 1) / kBlock;
    unsigned long long cand = 0;
    int biggest = 0;
    // Block-uniform loop over chunks of kBlock cells.
    for (int blk = blockIdx.x * blockDim.x; blk < nc; blk += gridDim.x * blockDim.x) {
        const int c = blk + threadIdx.x;
        unsigned int heavy_items = 0, light_items = 0;
        if (c < nc) {
            const int b0 = cell_begin[c];
            const int k = cell_begin[c + 1] - b0;
            int other = 0;
            const int* nb = nbr + 13 * static_cast<int64_t>(c);
            int nb_begin[13], nb_len[13];
#pragma unroll
            for (int o = 0; o < 13; ++o) {
                const int f = nb[o];
                nb_begin[o] = f >= 0 ? cell_begin[f] : 0;
                nb_len[o] = f >= 0 ? cell_begin[f + 1] - nb_begin[o] : 0;
                other += nb_len[o];
            }
            write_column_table(col_tab + 16 * static_cast<int64_t>(c), b0, k, nb_begin, nb_len);
            const int L = k + other;
            const unsigned int n_items = cell_items((k + 31) >> 5, (L + 31) >> 5, per);
            if (heavy_cell(k, L)) heavy_items = n_items;
            else light_items = n_items;
            cell_len[c] = L;
            cand += static_cast<unsigned long long>(k) * (k - 1) / 2 + static_cast<unsigned long long>(k) * other;
            biggest = max(biggest, k);
        }
        unsigned int heavy_total, light_total;
        block_exclusive_scan(heavy_items, &heavy_total);
        block_exclusive_scan(light_items, &light_total);
        if (threadIdx.x == 0) {
            part[blk / kBlock] = heavy_total;
            part[chunks + blk / kBlock] = light_total;
        }
    }
    cand = warp_sum(cand);
    biggest = warp_max(biggest);
    if ((threadIdx.x & 31) == 0) {
        if (cand) atomicAdd(&ctrl->candidates, cand);
        if (biggest > 0) atomicMax(&ctrl->max_cell, biggest);
    }
}

// Writes every cell's work items at their scanned places: heavy cells' items
// first, light cells' after them, each group in cell order (ctrl->n_items is
// the total); the pair kernel hands them out in that order, so the long items
// start first. A lane writes the items of a cell with at most 32 of them; the
// warp writes larger cells' together, row blocks spread over the lanes.
__global__ void __launch_bounds__(kBlock) k_items_write(Ctrl* ctrl, const int* __restrict__ cell_begin,
                                                        const int* __restrict__ cell_len,
                                                        const unsigned int* __restrict__ part,
                                                        int4* __restrict__ items, int64_t items_cap, int per) {
    if (step_void(ctrl)) return;
    const int nc = ctrl->n_cells;
    const int chunks = (nc + kBlock - 1) / kBlock;
    const int lane = threadIdx.x & 31;
    bool over = false;
    const int stride = gridDim.x * blockDim.x;
    for (int blk = blockIdx.x * blockDim.x; blk < nc; blk += stride) {
        const int c = blk + threadIdx.x;
        int k = 0, L = 0;
        unsigned int n_items = 0;
        bool heavy = false;
        int b0 = 0;
        if (c < nc) {
            b0 = cell_begin[c];
            k = cell_begin[c + 1] - b0;
            L = cell_len[c];
            heavy = heavy_cell(k, L);
            n_items = cell_items((k + 31) >> 5, (L + 31) >> 5, per);
        }
        unsigned int light_total, heavy_total;
        const int64_t loff = static_cast<int64_t>(part[chunks + blk / kBlock]) +
                             block_exclusive_scan(c < nc && !heavy ? n_items : 0u, &light_total);
        const int64_t hoff = static_cast<int64_t>(part[blk / kBlock]) +
                             block_exclusive_scan(heavy ? n_items : 0u, &heavy_total);
        const bool small = c < nc && n_items <= 32;
        if (small) {
            const int ta = (k + 31) >> 5, tc = (L + 31) >> 5;
            int64_t w = heavy ? hoff : loff;
            for (int a = 0; a < ta; ++a)
                for (int cb = a; cb < tc; cb += per, ++w) {
                    if (w < items_cap) items[w] = work_item(c, a, cb, min(per, tc - cb), b0);
                    else over = true;
                }
        }
        // Cells with more than 32 items are heavy (more than one row block).
        unsigned big = __ballot_sync(0xffffffffu, c < nc && !small);
        while (big) {
            const int src = __ffs(big) - 1;
            big &= big - 1;
            const int cc = blk + (threadIdx.x & ~31) + src;
            const int kk = __shfl_sync(0xffffffffu, k, src), LL = __shfl_sync(0xffffffffu, L, src);
            const int bb = __shfl_sync(0xffffffffu, b0, src);
            const int ta = (kk + 31) >> 5, tc = (LL + 31) >> 5;
            int64_t wbase = __shfl_sync(0xffffffffu, hoff, src);
            for (int a0 = 0; a0 < ta; a0 += 32) {
                const int a = a0 + lane;
                const unsigned int mine = a < ta ? row_block_items(a, tc, per) : 0u;
                unsigned int incl = mine;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                int64_t w = wbase + (incl - mine);
                for (int cb = a; a < ta && cb < tc; cb += per, ++w) {
                    if (w < items_cap) items[w] = work_item(cc, a, cb, min(per, tc - cb), bb);
                    else over = true;
                }
                wbase += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
    }
    if (over) atomicOr(&ctrl->flags, FLAG_ITEMS_OVERFLOW);
}

// ---------------------------------------------------------------------------
// Pairs: one warp per work item. Lanes hold consecutive columns of the cell's
// column list (its own objects, then those of its 13 forward neighbours); the
// warp loops over up to 32 rows of the cell, broadcast from shared memory.
// Inside the cell only pairs with column > row are visited, so every candidate
// pair of the reference (src/core/collision.cpp:522-538) is seen exactly once.
//
// The row loop is branch-free: each lane evaluates a conservative distance
// gate (no division, no square root) and records in a 32-bit mask the rows
// that the gate cannot reject. Those pairs then pass a conservative
// convexity test (a pair that is separating, not slow and convex over the
// step is rejected by filter_pair whatever its distance); only the rest run
// the exact filter_pair in FP64.
// ---------------------------------------------------------------------------

struct SortedState {
    double rx, ry, rz, vx, vy, vz;
};

__device__ __forceinline__ SortedState load_sorted(const double* __restrict__ sorted, int p) {
    const double2* s = reinterpret_cast<const double2*>(sorted + 6 * static_cast<int64_t>(p));
    const double2 a = s[0], b = s[1], c = s[2];
    return SortedState{a.x, a.y, b.x, b.y, c.x, c.y};
}

// 1 if the pair may pass the distance gate of filter_pair. With
// P = |dr|^2 |dv|^2 and m = min(dr.dv, 0), P - m^2 is |dv|^2 times the
// smallest squared distance of the linear relative motion over t >= 0; the
// gate can reject only if that exceeds |dv|^2 gate_hi^2. The 1e-12 P margin
// covers the rounding of P - m^2 (contraction is allowed here).
__device__ __forceinline__ unsigned gate_open(const SortedState& c, double2 ra, double2 rb, double2 rc,
                                              double gate_hi2) {
    const double rx = c.rx - ra.x, ry = c.ry - ra.y, rz = c.rz - rb.x;
    const double vx = c.vx - rb.y, vy = c.vy - rc.x, vz = c.vz - rc.y;
    const double r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const double dv2 = fma(vx, vx, fma(vy, vy, vz * vz));
    const double m = fmin(fma(rx, vx, fma(ry, vy, rz * vz)), 0.0);
    const double P = r2 * dv2;
    return fma(-m, m, P) <= fma(dv2, gate_hi2, 1e-12 * P) ? 1u : 0u;
}

// True only if filter_pair certainly returns FILTER_REJECT through its
// convexity clause or its distance gate, never FILTER_CO_ORBITING: the pair is
// faster than the minimum encounter speed, separating (dr.dv >= 0) and
// convex over the step (|dv|^2 > G |dr|^2). FP64 inputs are the filter's own
// dr, dv; the margins cover the contraction of the three sums.
__device__ __forceinline__ bool certainly_convex_reject(double rx, double ry, double rz, double vx, double vy,
                                                        double vz, double vmin2) {
    const double r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const double dv2 = fma(vx, vx, fma(vy, vy, vz * vz));
    const double rv = fma(rx, vx, fma(ry, vy, rz * vz));
    return dv2 > vmin2 * (1.0 + 1e-12) && rv > 0.0 && rv * rv > 1e-28 * (r2 * dv2) &&
           dv2 > kGravityGradient * r2 * (1.0 + 1e-12);
}

struct PairCounters {
    unsigned long long co = 0, full = 0;
};

// Next work item for this warp (one atomic per item).
__device__ __forceinline__ int next_item(Ctrl* ctrl) {
    unsigned int t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(&ctrl->item_ticket, 1u);
    return static_cast<int>(__shfl_sync(0xffffffffu, t, 0));
}

// Appends the pairs flagged `keep` (one atomic per warp).
__device__ __forceinline__ void append_pairs(bool keep, int row_orig, int col_orig, Ctrl* ctrl,
                                             int2* __restrict__ surv, int64_t surv_cap) {
    const int lane = threadIdx.x & 31;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (!bal) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&ctrl->refined, static_cast<unsigned long long>(__popc(bal)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) {
        const unsigned long long pos = base + __popc(bal & lanemask_lt());
        if (pos < static_cast<unsigned long long>(surv_cap))
            surv[pos] = make_int2(min(row_orig, col_orig), max(row_orig, col_orig));
    }
}

// Exact FP64 filter (src/core/collision_filter.hpp) of up to 32 queued pairs
// (column's sorted position, row of the tile), one pair per lane. kByObject:
// both states come from `states` by object index (the start-of-step states);
// otherwise the column from `states` in sorted order and the row from `rows`.
template <bool kByObject>
__device__ __forceinline__ void exact_flush(const int2* fq, int count, const double* __restrict__ states,
                                            const int* __restrict__ orig, const double2 (*rows)[3], const int* rorig,
                                            const StepArgs& a, int2* __restrict__ surv, int64_t surv_cap,
                                            PairCounters& pc) {
    const int lane = threadIdx.x & 31;
    int res = FILTER_REJECT;
    int row_orig = 0, col_orig = 0;
    if (lane < count) {
        const int2 e = fq[lane];
        col_orig = orig[e.x];
        row_orig = rorig[e.y];
        SortedState col, row;
        if (kByObject) {
            col = load_sorted(states, col_orig);
            row = load_sorted(states, row_orig);
        } else {
            col = load_sorted(states, e.x);
            const double2 ra = rows[e.y][0], rb = rows[e.y][1], rc = rows[e.y][2];
            row = SortedState{ra.x, ra.y, rb.x, rb.y, rc.x, rc.y};
        }
        ++pc.full;
        res = filter_pair_exact(xsub(col.rx, row.rx), xsub(col.ry, row.ry), xsub(col.rz, row.rz),
                                xsub(col.vx, row.vx), xsub(col.vy, row.vy), xsub(col.vz, row.vz), a.dt,
                                a.threshold_km, a.vmin2);
        if (res == FILTER_CO_ORBITING) ++pc.co;
    }
    append_pairs(res == FILTER_REFINE, row_orig, col_orig, a.ctrl, surv, surv_cap);
}

// Adds the pairs (q, r) for the rows r in `still` to the warp's queue fq
// (fcount entries, at most 63), one row per lane and round; every 32 queued
// pairs run the exact filter.
template <bool kByObject>
__device__ __forceinline__ void queue_exact(unsigned still, int q, int2* fq, int& fcount,
                                            const double* __restrict__ sorted, const int* __restrict__ orig,
                                            const double2 (*rows)[3], const int* rorig, const StepArgs& a,
                                            int2* __restrict__ surv, int64_t surv_cap, PairCounters& pc) {
    const int lane = threadIdx.x & 31;
    while (__any_sync(0xffffffffu, still != 0u)) {
        const bool have = still != 0u;
        const unsigned bal = __ballot_sync(0xffffffffu, have);
        if (have) {
            fq[fcount + __popc(bal & lanemask_lt())] = make_int2(q, __ffs(still) - 1);
            still &= still - 1;
        }
        fcount += __popc(bal);
        if (fcount >= 32) {
            __syncwarp();
            exact_flush<kByObject>(fq, 32, sorted, orig, rows, rorig, a, surv, surv_cap, pc);
            __syncwarp();
            if (lane < fcount - 32) fq[lane] = fq[32 + lane];
            __syncwarp();
            fcount -= 32;
        }
    }
}

// Rows flagged by the gate for the lane's column q (state col): the
// convexity test drops the pairs it proves rejected, the rest join the warp's
// queue for the exact filter.
__device__ __forceinline__ void exact_rows(unsigned need, const SortedState& col, int q,
                                           const double* __restrict__ sorted, const int* __restrict__ orig,
                                           const double2 (*rows)[3], const int* rorig, const StepArgs& a,
                                           int2* __restrict__ surv, int64_t surv_cap, PairCounters& pc, int2* fq,
                                           int& fcount) {
    unsigned todo = __reduce_or_sync(0xffffffffu, need);
    unsigned still = 0u;
    while (todo) {
        const int r = __ffs(todo) - 1;
        todo &= todo - 1;
        if ((need >> r) & 1u) {
            const double2 ra = rows[r][0], rb = rows[r][1], rc = rows[r][2];
            if (!certainly_convex_reject(xsub(col.rx, ra.x), xsub(col.ry, ra.y), xsub(col.rz, rb.x),
                                         xsub(col.vx, rb.y), xsub(col.vy, rc.x), xsub(col.vz, rc.y), a.vmin2))
                still |= 1u << r;
        }
    }
    queue_exact<false>(still, q, fq, fcount, sorted, orig, rows, rorig, a, surv, surv_cap, pc);
}

// Per-warp table of the item's non-empty column segments (the cell itself and
// its forward neighbours), for a binary search from column index to object.
struct SegTable {
    int start[16];   // first column index of the segment
    int begin[16];   // first sorted position of the segment's cell
    int id[16];      // 0 = the cell itself, 1 + o = forward neighbour o
};

// Builds the table for cell c; returns the column-list length L and the
// number of segments.
__device__ __forceinline__ int build_segments(SegTable& t, int c, int b0, int k, const int* __restrict__ cell_begin,
                                              const int* __restrict__ nbr, int* nseg_out) {
    const int lane = threadIdx.x & 31;
    int seg_begin = 0, seg_len = 0;
    if (lane == 0) {
        seg_begin = b0;
        seg_len = k;
    } else if (lane <= 13) {
        const int f = nbr[13 * static_cast<int64_t>(c) + lane - 1];
        if (f >= 0) {
            seg_begin = cell_begin[f];
            seg_len = cell_begin[f + 1] - seg_begin;
        }
    }
    int incl = seg_len;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned nz = __ballot_sync(0xffffffffu, seg_len > 0);
    if (seg_len > 0) {
        const int j = __popc(nz & lanemask_lt());
        t.start[j] = incl - seg_len;
        t.begin[j] = seg_begin;
        t.id[j] = lane;
    }
    __syncwarp();
    *nseg_out = __popc(nz);
    return __shfl_sync(0xffffffffu, incl, 31);
}

// Column index p -> sorted position and segment id (4 halvings cover 16 segments).
__device__ __forceinline__ int locate(const SegTable& t, int nseg, int p, int* sid) {
    int lo = 0, hi = nseg - 1;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        const int mid = (lo + hi + 1) >> 1;
        const bool ge = t.start[mid] <= p;
        lo = ge ? mid : lo;
        hi = ge ? hi : mid - 1;
    }
    *sid = t.id[lo];
    return t.begin[lo] + (p - t.start[lo]);
}

// Position / velocity bounding box of the 32 lanes' FP64 states.
struct BoxD {
    double pmin[3], pmax[3], vmin[3], vmax[3];
};

__device__ __forceinline__ double warp_min_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ BoxD warp_box_d(const SortedState& s) {
    BoxD b;
    const double p[3] = {s.rx, s.ry, s.rz}, v[3] = {s.vx, s.vy, s.vz};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        b.pmin[q] = warp_min_d(p[q]);
        b.pmax[q] = warp_max_d(p[q]);
        b.vmin[q] = warp_min_d(v[q]);
        b.vmax[q] = warp_max_d(v[q]);
    }
    return b;
}

// True if the column stays farther than gate from every state of the box
// over [0, dt]: |dr + dv t| >= |dr| - dt |dv| >= (box distance) - dt (largest
// relative speed), so filter_pair's distance gate rejects all those pairs.
// The factors cover the FP64 rounding of this test.
__device__ __forceinline__ bool apart_from_box_d(const BoxD& b, const SortedState& c, double dt, double gate) {
    const double p[3] = {c.rx, c.ry, c.rz}, v[3] = {c.vx, c.vy, c.vz};
    double d2 = 0.0, w2 = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double gap = fmax(0.0, fmax(p[q] - b.pmax[q], b.pmin[q] - p[q]));
        d2 = fma(gap, gap, d2);
        const double w = fmax(fabs(v[q] - b.vmin[q]), fabs(v[q] - b.vmax[q]));
        w2 = fma(w, w, w2);
    }
    return sqrt(d2) * (1.0 - 1e-12) - dt * sqrt(w2) * (1.0 + 1e-12) > gate;
}

template <int kCols>
__global__ void __launch_bounds__(kBlock, 3) k_pairs_tiles(StepArgs a, const double* __restrict__ sorted,
                                                        const int* __restrict__ orig,
                                                        const int* __restrict__ cell_begin,
                                                        const int* __restrict__ nbr, const int4* __restrict__ items,
                                                        int64_t items_cap, int2* __restrict__ surv, int64_t surv_cap) {
    __shared__ double2 rows[kWarps][32][3];
    __shared__ int rorig[kWarps][32];
    __shared__ SegTable segs[kWarps];
    // Per-warp queue of columns that survived the row-box test (sorted index, valid rows).
    __shared__ int qidx[kWarps][64];
    __shared__ unsigned qmask[kWarps][64];
    // Per-warp queue of pairs for the exact filter (column's sorted position, row).
    __shared__ int2 fq[kWarps][64];
    if (step_void(a.ctrl)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const int n_items = static_cast<int>(min(static_cast<int64_t>(a.ctrl->n_items), items_cap));
    const double vmax = __longlong_as_double(static_cast<long long>(a.ctrl->vmax_true));
    const double dt3 = a.dt * a.dt * a.dt;
    const double gate_hi = (a.threshold_km + kGravityGradient * (2.0 * vmax) * dt3 + 1e-3) * (1.0 + 1e-9);
    const double gate_hi2 = gate_hi * gate_hi;
    const int box_rows = kCols == 1 ? a.tune.box_min_rows : 0;
    PairCounters pc;
    int fcount = 0;
    // Items are handed out dynamically: their costs differ by orders of magnitude.
    for (int it = next_item(a.ctrl); it < n_items; it = next_item(a.ctrl)) {
        const int4 item = items[it];
        const int c = item.x, ra = item.y & 0xFFFFFF, cb0 = item.z;
        const int ncb = static_cast<int>(static_cast<unsigned int>(item.y) >> 24);
        const int b0 = cell_begin[c];
        const int k = cell_begin[c + 1] - b0;
        __syncwarp();
        int nseg;
        const int L = build_segments(segs[warp], c, b0, k, cell_begin, nbr, &nseg);
        const int r0 = 32 * ra;
        const int nr = min(32, k - r0);
        const unsigned nrmask = nr >= 32 ? 0xffffffffu : ((1u << nr) - 1u);
        if (lane < nr) {
            const double2* s = reinterpret_cast<const double2*>(sorted + 6 * static_cast<int64_t>(b0 + r0 + lane));
            rows[warp][lane][0] = s[0];
            rows[warp][lane][1] = s[1];
            rows[warp][lane][2] = s[2];
            rorig[warp][lane] = orig[b0 + r0 + lane];
        }
        __syncwarp();
        if (box_rows > 0 && nr >= box_rows) {
            // Columns tested against the rows' box, survivors compacted into full warps.
            const BoxD rbox = warp_box_d(load_sorted(sorted, b0 + r0 + (lane < nr ? lane : 0)));
            auto drain = [&](int count) {
                __syncwarp();
                const bool has = lane < count;
                const int q = qidx[warp][has ? lane : 0];
                const unsigned valid = has ? qmask[warp][lane] : 0u;
                __syncwarp();
                const SortedState col = load_sorted(sorted, q);
                unsigned need = 0u;
#pragma unroll 4
                for (int r = 0; r < nr; ++r)
                    need |= gate_open(col, rows[warp][r][0], rows[warp][r][1], rows[warp][r][2], gate_hi2) << r;
                need &= valid;
                if (__any_sync(0xffffffffu, need != 0u))
                    exact_rows(need, col, q, sorted, orig, rows[warp], rorig[warp], a, surv, surv_cap, pc, fq[warp],
                               fcount);
            };
            int queued = 0;
            for (int cb = cb0; cb < cb0 + ncb; ++cb) {
                const int p = 32 * cb + lane;
                const bool ok = p < L;
                int sid;
                const int q = ok ? locate(segs[warp], nseg, p, &sid) : b0;
                const unsigned valid = ok ? (cb == ra ? lanes_below : 0xffffffffu) & nrmask : 0u;
                const bool keep = valid != 0u && !apart_from_box_d(rbox, load_sorted(sorted, q), a.dt, gate_hi);
                const unsigned kept = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int slot = queued + __popc(kept & lanes_below);
                    qidx[warp][slot] = q;
                    qmask[warp][slot] = valid;
                }
                queued += __popc(kept);
                if (queued >= 32) {
                    drain(32);
                    if (lane < queued - 32) {
                        qidx[warp][lane] = qidx[warp][32 + lane];
                        qmask[warp][lane] = qmask[warp][32 + lane];
                    }
                    queued -= 32;
                }
            }
            if (queued > 0) drain(queued);
            __syncwarp();
            // The rows change with the next item: run the queued pairs now.
            if (fcount > 0) exact_flush<false>(fq[warp], fcount, sorted, orig, rows[warp], rorig[warp], a, surv, surv_cap, pc);
            fcount = 0;
            __syncwarp();
            continue;
        }
        for (int cb = cb0; cb < cb0 + ncb; cb += kCols) {
            SortedState col[kCols];
            int qs[kCols];
            unsigned valid[kCols];
            for (int h = 0; h < kCols; ++h) {
                const int p = 32 * (cb + h) + lane;
                const bool ok = (cb + h < cb0 + ncb) && p < L;
                int sid;
                const int q = ok ? locate(segs[warp], nseg, p, &sid) : b0;
                col[h] = load_sorted(sorted, q);
                qs[h] = q;
                // The block that starts at the row block's own columns keeps only column > row.
                valid[h] = ok ? (cb + h == ra ? ((1u << lane) - 1u) : 0xffffffffu) & nrmask : 0u;
            }
            unsigned need[kCols];
            for (int h = 0; h < kCols; ++h) need[h] = 0u;
#pragma unroll 4
            for (int r = 0; r < nr; ++r) {
                const double2 ra2 = rows[warp][r][0], rb2 = rows[warp][r][1], rc2 = rows[warp][r][2];
                for (int h = 0; h < kCols; ++h) need[h] |= gate_open(col[h], ra2, rb2, rc2, gate_hi2) << r;
            }
            for (int h = 0; h < kCols; ++h) {
                need[h] &= valid[h];
                if (__any_sync(0xffffffffu, need[h] != 0u))
                    exact_rows(need[h], col[h], qs[h], sorted, orig, rows[warp], rorig[warp], a, surv, surv_cap,
                               pc, fq[warp], fcount);
            }
        }
        __syncwarp();
        if (fcount > 0) exact_flush<false>(fq[warp], fcount, sorted, orig, rows[warp], rorig[warp], a, surv, surv_cap, pc);
        fcount = 0;
        __syncwarp();
    }
    pc.co = warp_sum(pc.co);
    pc.full = warp_sum(pc.full);
    if (lane == 0) {
        if (pc.co) atomicAdd(&a.ctrl->co_orbiting, pc.co);
        if (pc.full) atomicAdd(&a.ctrl->exact_evals, pc.full);
    }
}

// ---------------------------------------------------------------------------
// Split-precision pair kernel: same work items and the same exact decision
// (filter_pair on the FP64 states) for the pairs the FP32 tests cannot
// reject. Rows and columns are FP32 records relative to their own cell's
// corner; a column from forward neighbour o is moved into the row cell's
// frame by forward_offset(o) cell edges. Tiles whose row block and column block
// are provably apart over the whole step (position and velocity boxes) are
// skipped before the row loop.
// ---------------------------------------------------------------------------

__device__ __forceinline__ float warp_min_f(float v) {
    float r;
    asm("redux.sync.min.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ float warp_max_f(float v) {
    float r;
    asm("redux.sync.max.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(v));
    return r;
}

struct Box {
    float pmin[3], pmax[3], vmin[3], vmax[3];
};

__device__ __forceinline__ Box warp_box(float4 p, float4 v) {
    Box b;
    b.pmin[0] = warp_min_f(p.x); b.pmin[1] = warp_min_f(p.y); b.pmin[2] = warp_min_f(p.z);
    b.pmax[0] = warp_max_f(p.x); b.pmax[1] = warp_max_f(p.y); b.pmax[2] = warp_max_f(p.z);
    b.vmin[0] = warp_min_f(v.x); b.vmin[1] = warp_min_f(v.y); b.vmin[2] = warp_min_f(v.z);
    b.vmax[0] = warp_max_f(v.x); b.vmax[1] = warp_max_f(v.y); b.vmax[2] = warp_max_f(v.z);
    return b;
}

// True if every pair (row in box a, column in box b) stays farther apart than
// gate over [0, dt]: the box distance d exceeds gate + dt w, w the largest
// relative speed. gate already carries the FP32 record errors. The distance is
// compared squared; w takes one approximate square root (sqrt.approx.f32,
// error a few units in the last place), raised by 1e-4, some 800 times 2^-23;
// the other factors cover the FP32 rounding of this test, so that it is at
// least as strict as d (1 - 1e-5) - dt w (1 + 1e-5) > gate.
__device__ __forceinline__ bool boxes_apart(const Box& a, const Box& b, float dt, float gate) {
    float d2 = 0.f, w2 = 0.f;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float gap = fmaxf(0.f, fmaxf(b.pmin[q] - a.pmax[q], a.pmin[q] - b.pmax[q]));
        d2 = fmaf(gap, gap, d2);
        const float w = fmaxf(fabsf(b.vmax[q] - a.vmin[q]), fabsf(b.vmin[q] - a.vmax[q]));
        w2 = fmaf(w, w, w2);
    }
    float w;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(w) : "f"(w2));
    const float reach = fmaf(dt, w * (1.0f + 1e-4f), gate);
    return d2 * (1.0f - 4e-5f) > reach * reach * (1.0f + 1e-5f);
}

// Second FP32 stage for the pairs the gate lets through, on FP32 records whose
// dr, dv carry absolute errors up to er, ev (f32_pos_err, f32_vel_err): true
// only if filter_pair_exact certainly returns FILTER_REJECT, for one of two
// reasons. vmin2e is (vmin + ev)^2; gate2 is the squared FP32 gate (the
// exact filter's gate widened by e = er + ev dt, as gate_open_f32 takes it).
//  (1) Separating, fast and convex: the reference's convexity rejection
//      (src/core/collision_filter.hpp:63), FP32 version of
//      certainly_convex_reject; margins as derived in the comments below.
//  (2) Closest approach after the step: when -dr.dv > |dv|^2 dt the exact
//      filter clamps ts to dt (src/core/collision_filter.hpp:45-47) and
//      gates |dr + dv dt|. The true relative motion stays within e of the
//      records' over the step, which gate2 covers. For the records' values,
//      the FP32 rounding of dr + dv dt is below 3.1e-7 |dr| (|dv| dt <= |dr|
//      when -dr.dv > |dv|^2 dt), and a pair wrongly classed as "after" by the
//      rounding of dr.dv and |dv|^2 dt (a few ulps of |dr||dv|) has its true
//      minimum within 4.8e-7 |dr| of |dr + dv dt|. With b = 1e-6 |dr| >= both:
//      (g + b)^2 <= g^2 (1 + 1e-4) + 1.01e-8 |dr|^2, and the factors below add
//      room for the rounding of the squares. In the bench workload these are
//      two thirds of the pairs the convexity test leaves.
__device__ __forceinline__ bool certainly_reject_f32(float rx, float ry, float rz, float vx, float vy, float vz,
                                                     float vmin2e, float er, float ev, float dt, float gate2) {
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    const float dv2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
    const float rv = fmaf(rx, vx, fmaf(ry, vy, rz * vz));
    // |dv| >= |dv'| - ev > vmin.
    const bool fast = dv2 > 1.0001f * vmin2e + 1e-12f;
    // rv >= rv' - (|dr'| ev + |dv'| er + er ev + 2e-7 |dr'||dv'|); squared bound.
    const bool separating =
        rv > 0.f && rv * rv > 4.01f * (r2 * (ev * ev) + dv2 * (er * er) + (er * ev) * (er * ev) + 4e-14f * r2 * dv2);
    // With 2|x| <= x^2 + 1 and 1e-6 for the FP32 rounding of the sums:
    // dv2' >= dv2 (1 - ev - 1e-6) - ev - ev^2 and r2' <= r2 (1 + er + 1e-6) + er + er^2;
    // the factors below take about twice those margins.
    const bool convex = dv2 * (1.0f - 2.0f * ev - 4e-6f) - 1.25f * (ev + ev * ev) >
                        static_cast<float>(kGravityGradient * 1.0002) *
                            fmaf(r2, 1.0f + 2.0f * er + 2e-6f, 1.25f * (er + er * er));
    if (fast && separating && convex) return true;
    if (!(rv < 0.f) || !(-rv > dv2 * dt)) return false;
    const float px = fmaf(vx, dt, rx), py = fmaf(vy, dt, ry), pz = fmaf(vz, dt, rz);
    const float pe2 = fmaf(px, px, fmaf(py, py, pz * pz));
    return pe2 > fmaf(gate2, 1.00012f, 1.2e-8f * r2);
}

// Rows flagged by the FP32 gate for the lane's column q: the second FP32
// stage (certainly_reject_f32) drops the pairs it proves rejected, the rest
// join the warp's queue for the exact filter.
__device__ __forceinline__ void exact_rows_f32(unsigned need, float4 cp, float4 cv, int q, const double* __restrict__ before,
                                               const int* __restrict__ orig, const float4 (*rows32)[2],
                                               const int* rorig, float vmin2e, float er, float ev, float dt_f,
                                               float gate2, const StepArgs& a,
                                               int2* __restrict__ surv, int64_t surv_cap, PairCounters& pc, int2* fq,
                                               int& fcount, float4 (*ccol)[2], int* cidx, bool staged,
                                               unsigned short* pq) {
    const int lane = threadIdx.x & 31;
    unsigned todo = __reduce_or_sync(0xffffffffu, need);
    // When the flagged pairs are sparse (under half the lanes busy per row of
    // the loop below), they are queued one pair per lane instead and tested 32
    // at a time; the same test on the same pairs, so the same survivors.
    const int mode = a.tune.pair_stage2;
    if (mode == 2 || (mode == 1 && 2u * __reduce_add_sync(0xffffffffu, static_cast<unsigned>(__popc(need))) <
                                       32u * static_cast<unsigned>(__popc(todo)))) {
        if (!staged) {  // the lanes' columns into the (empty) column queue
            ccol[lane][0] = cp;
            ccol[lane][1] = cv;
            cidx[lane] = q;
        }
        __syncwarp();
        unsigned mine = need;
        int pn = 0;
        auto test = [&](int count) {
            __syncwarp();
            unsigned keep = 0u;
            int qs = 0;
            if (lane < count) {
                const unsigned e = pq[lane];
                const int src = static_cast<int>(e >> 8), r = static_cast<int>(e & 0xFFu);
                const float4 c0 = ccol[src][0], c1 = ccol[src][1];
                const float4 rp = rows32[r][0], rv = rows32[r][1];
                qs = cidx[src];
                if (!certainly_reject_f32(c0.x - rp.x, c0.y - rp.y, c0.z - rp.z, c1.x - rv.x, c1.y - rv.y,
                                          c1.z - rv.z, vmin2e, er, ev, dt_f, gate2))
                    keep = 1u << r;
            }
            __syncwarp();
            queue_exact<true>(keep, qs, fq, fcount, before, orig, nullptr, rorig, a, surv, surv_cap, pc);
        };
        while (__any_sync(0xffffffffu, mine != 0u)) {
            const bool have = mine != 0u;
            const unsigned bal = __ballot_sync(0xffffffffu, have);
            if (have) {
                pq[pn + __popc(bal & lanemask_lt())] = static_cast<unsigned short>((lane << 8) | (__ffs(mine) - 1));
                mine &= mine - 1;
            }
            pn += __popc(bal);
            if (pn >= 32) {
                test(32);
                __syncwarp();
                if (lane < pn - 32) pq[lane] = pq[32 + lane];
                pn -= 32;
            }
        }
        if (pn > 0) test(pn);
        __syncwarp();
        return;
    }
    // FP32 second stage, row by row: drop rows no lane still needs.
    unsigned still = 0u;
    while (todo) {
        const int r = __ffs(todo) - 1;
        todo &= todo - 1;
        if ((need >> r) & 1u) {
            const float4 rp = rows32[r][0], rv = rows32[r][1];
            if (!certainly_reject_f32(cp.x - rp.x, cp.y - rp.y, cp.z - rp.z, cv.x - rv.x, cv.y - rv.y,
                                      cv.z - rv.z, vmin2e, er, ev, dt_f, gate2))
                still |= 1u << r;
        }
    }
    queue_exact<true>(still, q, fq, fcount, before, orig, nullptr, rorig, a, surv, surv_cap, pc);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks) k_pairs_split(StepArgs a, const double* __restrict__ before,
                                                        const float4* __restrict__ sorted32,
                                                        const int* __restrict__ orig,
                                                        const int2* __restrict__ col_tab, const int4* __restrict__ items,
                                                        int64_t items_cap, int2* __restrict__ surv, int64_t surv_cap) {
    __shared__ float4 rows32[kWarps][32][2];
    // The same rows in pairs, components interleaved, for the packed gate.
    __shared__ float2 rows2[kWarps][16][6];
    __shared__ int rorig[kWarps][32];
    // Per-warp queue of columns that survived the row-box test, drained 32 at a time.
    __shared__ float4 qcol[kWarps][64][2];
    __shared__ int qidx[kWarps][64];
    __shared__ unsigned qmask[kWarps][64];
    // Per-warp queue of pairs for the exact filter (column's sorted position, row).
    // Per-warp queue of flagged (column lane, row) pairs for the compacted second stage.
    __shared__ unsigned short pq[kWarps][64];
    __shared__ int2 fq[kWarps][64];
    if (step_void(a.ctrl)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const int n_items = static_cast<int>(min(static_cast<int64_t>(a.ctrl->n_items), items_cap));
    const double vmax = __longlong_as_double(static_cast<long long>(a.ctrl->vmax_true));
    const double dt3 = a.dt * a.dt * a.dt;
    const double gate_hi = (a.threshold_km + kGravityGradient * (2.0 * vmax) * dt3 + 1e-3) * (1.0 + 1e-9);
    // Error bounds of the FP32 records for this grid and these speeds.
    const double er_d = f32_pos_err(a.ctrl->grid.cell), ev_d = f32_vel_err(vmax);
    const float er = static_cast<float>(er_d), ev = static_cast<float>(ev_d);
    const double gate_e = (gate_hi + er_d + ev_d * a.dt) * (1.0 + 1e-6);
    const float gate_f = static_cast<float>(gate_e);
    const float gate2 = gate_f * gate_f;
    const float2 gate2x2 = make_float2(gate2, gate2);
    const bool gate_x2 = a.tune.pair_gate_x2 != 0;
    const float dt_f = static_cast<float>(a.dt);
    const float cell_f = static_cast<float>(a.ctrl->grid.cell);
    const double vme = sqrt(a.vmin2) + ev_d;
    const float vmin2e = static_cast<float>(vme * vme * (1.0 + 1e-6));
    const int box_rows = a.tune.box_min_rows;
    const int last_record = max(0, a.ctrl->n_alive - 1);
    PairCounters pc;
    int fcount = 0;
    // Items are handed out dynamically: their costs differ by orders of magnitude.
    for (int it = next_item(a.ctrl); it < n_items; it = next_item(a.ctrl)) {
        const int4 item = items[it];
        const int c = item.x, ra = item.y & 0xFFFFFF, cb0 = item.z, b0 = item.w;
        const int ncb = static_cast<int>(static_cast<unsigned int>(item.y) >> 24);
        const int r0 = 32 * ra;
        // The cell's column table and its rows, loaded together (the rows of
        // lanes past the cell's end are replaced below).
        const int2 te = col_tab[16 * static_cast<int64_t>(c) + (lane & 15)];
        const int rl = min(b0 + r0 + lane, last_record);
        float4 my_rp = sorted32[2 * static_cast<int64_t>(rl)];
        float4 my_rv = sorted32[2 * static_cast<int64_t>(rl) + 1];
        const int my_orig = orig[rl];
        const int L = __shfl_sync(0xffffffffu, te.x, 15), nseg = __shfl_sync(0xffffffffu, te.y, 15);
        const unsigned id_lo = static_cast<unsigned>(__shfl_sync(0xffffffffu, te.x, 14));
        const unsigned id_hi = static_cast<unsigned>(__shfl_sync(0xffffffffu, te.y, 14));
        const int second = __shfl_sync(0xffffffffu, te.x, 1);
        const int k = nseg > 1 ? second : L;
        const int nr = min(32, k - r0);
        const unsigned nrmask = nr >= 32 ? 0xffffffffu : ((1u << nr) - 1u);
        {
            // Rows past nr repeat the first row (their bits are masked off).
            const float4 p0 = make_float4(__shfl_sync(0xffffffffu, my_rp.x, 0), __shfl_sync(0xffffffffu, my_rp.y, 0),
                                          __shfl_sync(0xffffffffu, my_rp.z, 0), my_rp.w);
            const float4 v0 = make_float4(__shfl_sync(0xffffffffu, my_rv.x, 0), __shfl_sync(0xffffffffu, my_rv.y, 0),
                                          __shfl_sync(0xffffffffu, my_rv.z, 0), my_rv.w);
            if (lane >= nr) {
                my_rp = p0;
                my_rv = v0;
            }
        }
        // Lane j < nseg holds segment j: its first column, the sorted position
        // minus that column, and its move into the row cell's frame (the
        // forward offset times the cell edge; none for the cell itself).
        const int seg_start = lane < nseg ? te.x : 0x7FFFFFFF;
        const int seg_base = lane < nseg ? te.y - te.x : 0;
        const unsigned seg_id = lane < nseg ? (((lane < 8 ? id_lo >> (4 * lane) : id_hi >> (4 * (lane - 8)))) & 15u) : 0u;
        float4 seg_off = make_float4(0.f, 0.f, 0.f, 0.f);
        if (seg_id > 0) {
            int dx, dy, dz;
            forward_offset(static_cast<int>(seg_id) - 1, dx, dy, dz);
            // dx cell_f is exact (dx in {-1, 0, 1}): adding it rounds once, as fma(dx, cell_f, x) would.
            seg_off = make_float4(static_cast<float>(dx) * cell_f, static_cast<float>(dy) * cell_f,
                                  static_cast<float>(dz) * cell_f, 0.0f);
        }
        __syncwarp();
        if (lane < nr) {
            rows32[warp][lane][0] = my_rp;
            rows32[warp][lane][1] = my_rv;
            rorig[warp][lane] = my_orig;
        }
        if (gate_x2) {
            // Lane l writes its row into pair l / 2, half l % 2 (rows past nr
            // repeat the first row; their bits are masked off).
            float* pr = reinterpret_cast<float*>(rows2[warp][lane >> 1]) + (lane & 1);
            pr[0] = my_rp.x; pr[2] = my_rp.y; pr[4] = my_rp.z;
            pr[6] = my_rv.x; pr[8] = my_rv.y; pr[10] = my_rv.z;
        }
        // Tiles of at least box_rows rows test each column against the rows'
        // position / velocity box first and keep only columns that could come
        // within the gate of some row, compacted into full warps.
        const bool use_box = box_rows > 0 && nr >= box_rows;
        Box rbox;
        if (use_box) rbox = warp_box(my_rp, my_rv);
        __syncwarp();
        // Columns held by the lanes (entry `lane` of a batch) against every row.
        auto gate_rows = [&](float4 cp, float4 cv, int q, unsigned valid, bool staged) {
            unsigned need = 0u;
            if (gate_x2) {
#pragma unroll 2
                for (int r = 0; r < nr; r += 2) need |= gate_open_f32x2(cp, cv, rows2[warp][r >> 1], gate2x2) << r;
            } else {
#pragma unroll 4
                for (int r = 0; r < nr; ++r)
                    need |= gate_open_f32(cp, cv, rows32[warp][r][0], rows32[warp][r][1], gate2) << r;
            }
            need &= valid;
            if (__any_sync(0xffffffffu, need != 0u))
                exact_rows_f32(need, cp, cv, q, before, orig, rows32[warp], rorig[warp], vmin2e, er, ev, dt_f, gate2,
                               a, surv, surv_cap, pc, fq[warp], fcount, qcol[warp], qidx[warp], staged, pq[warp]);
        };
        auto drain = [&](int count) {
            __syncwarp();
            const int e = lane < count ? lane : 0;
            gate_rows(qcol[warp][e][0], qcol[warp][e][1], qidx[warp][e], lane < count ? qmask[warp][e] : 0u, true);
            __syncwarp();
        };
        int queued = 0;
        // A column block's lanes find their segments by one ballot (the
        // segment of its first column) and one OR of the segment starts inside it.
        for (int cb = cb0; cb < cb0 + ncb; ++cb) {
            const int p0 = 32 * cb;
            const int p = p0 + lane;
            const bool ok = p < L;
            const unsigned at_or_before = __ballot_sync(0xffffffffu, seg_start <= p0);
            const int seg0 = 31 - __clz(at_or_before);
            const unsigned inside = __reduce_or_sync(
                0xffffffffu, (seg_start > p0 && seg_start - p0 < 32) ? (1u << (seg_start - p0)) : 0u);
            const int seg = seg0 + __popc(inside & ((2u << lane) - 1u));
            const int sb = __shfl_sync(0xffffffffu, seg_base, seg);  // every lane: a full-mask shuffle
            const int q = ok ? sb + p : b0;
            const float ox = __shfl_sync(0xffffffffu, seg_off.x, seg);
            const float oy = __shfl_sync(0xffffffffu, seg_off.y, seg);
            const float oz = __shfl_sync(0xffffffffu, seg_off.z, seg);
            float4 cp = sorted32[2 * static_cast<int64_t>(q)];
            const float4 cv = sorted32[2 * static_cast<int64_t>(q) + 1];
            if (seg > 0) {
                cp.x += ox;
                cp.y += oy;
                cp.z += oz;
            }
            const unsigned valid = ok ? (cb == ra ? lanes_below : 0xffffffffu) & nrmask : 0u;
            if (!use_box) {
                gate_rows(cp, cv, q, valid, false);
                continue;
            }
            Box cbox;
            cbox.pmin[0] = cbox.pmax[0] = cp.x; cbox.pmin[1] = cbox.pmax[1] = cp.y; cbox.pmin[2] = cbox.pmax[2] = cp.z;
            cbox.vmin[0] = cbox.vmax[0] = cv.x; cbox.vmin[1] = cbox.vmax[1] = cv.y; cbox.vmin[2] = cbox.vmax[2] = cv.z;
            const bool keep = valid != 0u && !boxes_apart(rbox, cbox, dt_f, gate_f);
            const unsigned kept = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int slot = queued + __popc(kept & lanes_below);
                qcol[warp][slot][0] = cp;
                qcol[warp][slot][1] = cv;
                qidx[warp][slot] = q;
                qmask[warp][slot] = valid;
            }
            queued += __popc(kept);
            if (queued >= 32) {
                drain(32);
                if (lane < queued - 32) {
                    qcol[warp][lane][0] = qcol[warp][32 + lane][0];
                    qcol[warp][lane][1] = qcol[warp][32 + lane][1];
                    qidx[warp][lane] = qidx[warp][32 + lane];
                    qmask[warp][lane] = qmask[warp][32 + lane];
                }
                queued -= 32;
            }
        }
        if (queued > 0) drain(queued);
        __syncwarp();
        // The rows change with the next item: run the queued pairs now.
        if (fcount > 0) exact_flush<true>(fq[warp], fcount, before, orig, nullptr, rorig[warp], a, surv, surv_cap, pc);
        fcount = 0;
        __syncwarp();
    }
    pc.co = warp_sum(pc.co);
    pc.full = warp_sum(pc.full);
    if (lane == 0) {
        if (pc.co) atomicAdd(&a.ctrl->co_orbiting, pc.co);
        if (pc.full) atomicAdd(&a.ctrl->exact_evals, pc.full);
    }
}

// ---------------------------------------------------------------------------
// Refinement
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_refine_exact(StepArgs a, const double* __restrict__ before,
                                                         const double* __restrict__ after,
                                                         const double* __restrict__ size_m,
                                                         const int2* __restrict__ surv, int64_t surv_cap,
                                                         ks_conjunction* __restrict__ out, int64_t cap,
                                                         ChunkCtrl* chunk) {
    if (step_void(a.ctrl)) return;
    const unsigned long long ns = min(a.ctrl->refined, static_cast<unsigned long long>(surv_cap));
    const double t0 = a.sp->t0;
    const double s_hi = xsub(1.0, 1e-9);
    for (unsigned long long w = blockIdx.x * blockDim.x + threadIdx.x; w < ns; w += gridDim.x * blockDim.x) {
        const int i = surv[w].x, j = surv[w].y;
        double bi[6], bj[6], ai[6], aj[6];
        ld6(before, i, bi);
        ld6(before, j, bj);
        ld6(after, i, ai);
        ld6(after, j, aj);
        Hermite h;
        for (int q = 0; q < 3; ++q) {
            h.p0[q] = xsub(bj[q], bi[q]);
            h.m0[q] = xmul(xsub(bj[3 + q], bi[3 + q]), a.dt);
            h.p1[q] = xsub(aj[q], ai[q]);
            h.m1[q] = xmul(xsub(aj[3 + q], ai[3 + q]), a.dt);
        }
        const double s = closest_approach_exact(h);
        if (s <= 1e-9 || s >= s_hi) continue;
        double pp[3], vv[3];
        h.pos(s, pp);
        const double miss = xsqrt(xdot3(pp[0], pp[1], pp[2]));
        if (miss > a.threshold_km) continue;
        h.vel(s, vv);
        ks_conjunction c;
        c.i = i;
        c.j = j;
        c.step = a.sp->step;
        c.t = xadd(t0, xmul(s, a.dt));
        c.miss_km = miss;
        c.v_rel_km_s = xdiv(xsqrt(xdot3(vv[0], vv[1], vv[2])), a.dt);
        const double ri = xmul(xmul(xmul(0.5, size_m[i]), 1e-3), a.radius_scale);
        const double rj = xmul(xmul(xmul(0.5, size_m[j]), 1e-3), a.radius_scale);
        c.collision = miss < xadd(ri, rj) ? 1 : 0;
        c.realisation = a.real_id ? a.real_id[i] : 0;
        if (c.collision && a.coll) {
            const unsigned int k = atomicAdd(&a.ctrl->n_coll, 1u);
            if (k < static_cast<unsigned int>(a.coll_cap)) a.coll[k] = CollisionRec{i, j, c.t};
            else atomicOr(&a.ctrl->flags, FLAG_COLL_OVERFLOW);
        }
        atomicAdd(&a.ctrl->conj, 1ull);
        const unsigned long long slot = atomicAdd(&chunk->conj_count, 1ull);
        if (slot < static_cast<unsigned long long>(cap)) out[slot] = c;
        else atomicOr(&chunk->flags, FLAG_CONJ_OVERFLOW);
    }
}

// ---------------------------------------------------------------------------
// FP64 issue-rate microbenchmark: 8 independent dependent chains per thread.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_fp64_addmul(double* out, int iters, double a, double b) {
    double x[8];
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-3 + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __dadd_rn(__dmul_rn(x[q], a), b);
    }
    double s = 0;
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 1.2345) out[0] = s;
}

__global__ void __launch_bounds__(256) k_fp64_fma(double* out, int iters, double a, double b) {
    double x[8];
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-3 + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __fma_rn(x[q], a, b);
    }
    double s = 0;
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 1.2345) out[0] = s;
}

__global__ void __launch_bounds__(256) k_fp32_addmul(float* out, int iters, float a, float b) {
    float x[8];
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-3f + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __fadd_rn(__fmul_rn(x[q], a), b);
    }
    float s = 0;
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 1.2345f) out[0] = s;
}

__global__ void __launch_bounds__(256) k_fp32_fma(float* out, int iters, float a, float b) {
    float x[8];
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-3f + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __fmaf_rn(x[q], a, b);
    }
    float s = 0;
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 1.2345f) out[0] = s;
}

// Packed FP32: 8 independent chains of FFMA2 (two FP32 FMAs per lane and instruction).
__global__ void __launch_bounds__(256) k_fp32x2_fma(float* out, int iters, float a, float b) {
    float2 x[8];
    for (int q = 0; q < 8; ++q) x[q] = make_float2(threadIdx.x * 1e-3f + q, threadIdx.x * 2e-3f + q);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __ffma2_rn(x[q], a2, b2);
    }
    float s = 0;
    for (int q = 0; q < 8; ++q) s += x[q].x + x[q].y;
    if (s == 1.2345f) out[0] = s;
}

// SM count per device index, looked up on first use from each device. The
// entries are atomics so that threads driving different devices (or the
// allocation-free entry point from any thread) neither race nor share a count.
constexpr int kMaxSmDevices = 64;
std::atomic<int> g_sm_count[kMaxSmDevices];

// ---------------------------------------------------------------------------
// Fused object sort and cell build: one cooperative launch
//
// One block of 1024 threads per SM. Block b owns the keys [b R, b R + R),
// R = ceil(n / G) over the G blocks, K per thread in registers: warp w holds
// the 32 K consecutive keys from 32 K w, its round r the 32 from 32 r. Grid
// barriers take the place of kernel boundaries and of k_sort_onesweep's
// look-back (whose chain of L2 round trips grows with the number of tiles).
// Per 8-bit radix pass:
//   rank     per-warp digit counters in shared memory place every key among
//            the block's keys of its digit (stable: warp, round, lane order);
//            the block's 256 digit counts go to `counts` and are added to the
//            pass's digit totals; barrier
//   starts   warp w of block b scans digit d = b + w G over the G blocks and
//            writes every block's first output position for d; barrier
//   scatter  keys staged in shared memory in digit order, stored run by run
//            from the block's starts; barrier
// Then the cells, over the same ranges of the sorted keys:
//   heads    a key whose cell differs from its predecessor's opens a cell;
//            per-block counts; the records are gathered in sorted order while
//            the barrier completes
//   cells    ranges, keys and hash entries of the block's cells; barrier
//   items    per cell of the block's share: its 13 forward neighbours (hash),
//            the length of its column list and its work items; heavy and
//            light totals per block; barrier
//   list     the work list, heavy cells' items first, each group in cell order
// Every barrier wait is bounded by the look-back poll limit: a block that
// gives up sets FLAG_TIMEOUT (the step is discarded) and goes on, every store
// kept in bounds, so the launch always ends. Data other blocks wrote during
// the launch is read through L2 (ld.global.cg), never through L1.
// ---------------------------------------------------------------------------

constexpr int kFusedThreads = 1024;
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kFusedMaxGrid = 256;              // the starts scan loads at most 8 counts per lane
constexpr int kFusedDigits = 2048;              // digits of a pass, at most (11-bit digits)
constexpr int kFusedZeroWords = 32 + 6 * kFusedDigits;  // barrier counter, per-pass digit totals: zeroed per launch

struct FusedArgs {
    unsigned long long* keys[2];
    unsigned int* scratch;
    int* cell_begin;
    unsigned long long* cell_key;
    unsigned long long* hk;
    int* hv;
    unsigned long long hmask;
    const double* before;
    double* sorted;          // FP64 states in sorted order (with FP32 records when sorted32), or null
    int* sorted_orig;
    float4* sorted32;
    const float4* rec32;     // FP32 records in object order (used when sorted is null)
    int* nbr;
    int* cell_len;
    int2* col_tab;
    int4* items;
    int64_t items_cap;
    int per;
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier over a counter zeroed before the launch: the k-th barrier of
// the launch waits for k G arrivals. Split in two so that work nobody else
// reads before the launch ends can run while the barrier completes.
__device__ __forceinline__ void grid_arrive(unsigned int* bar, unsigned int& target) {
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
    }
}
__device__ __forceinline__ void grid_wait(const unsigned int* bar, unsigned int target, int poll_limit, int* flags) {
    if (threadIdx.x == 0) {
        int polls = 0;
        while (ld_acquire(bar) < target) {
            if (++polls > poll_limit) {
                atomicOr(flags, FLAG_TIMEOUT);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
}
__device__ __forceinline__ void grid_sync(unsigned int* bar, unsigned int& target, int poll_limit, int* flags) {
    grid_arrive(bar, target);
    grid_wait(bar, target, poll_limit, flags);
}

// Whether a barrier of this launch gave up (read through L2, the same answer
// for the whole block): the later phases then skip their work, keeping only
// their barrier arrivals, since the step is discarded.
__device__ __forceinline__ bool launch_gave_up(const int* flags, int* sh) {
    __syncthreads();
    if (threadIdx.x == 0) *sh = __ldcg(flags) & FLAG_TIMEOUT;
    __syncthreads();
    return *sh != 0;
}

// Exclusive scan over the block's 1024 threads (wsum: 32 words of shared memory).
__device__ __forceinline__ unsigned int scan_1024(unsigned int v, unsigned int* total, unsigned int* wsum) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned int t = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;
    }
    __syncthreads();
    const unsigned int off = warp > 0 ? wsum[warp - 1] : 0u;
    *total = wsum[31];
    __syncthreads();
    return off + incl - v;
}

// One warp: the sum of v[j] over the blocks j < upto, and over all G blocks.
__device__ __forceinline__ void blocks_sum(const unsigned int* v, int G, int upto, unsigned long long* below,
                                           unsigned long long* all) {
    const int lane = threadIdx.x & 31;
    unsigned long long sb = 0, sa = 0;
#pragma unroll
    for (int i = 0; i < kFusedMaxGrid / 32; ++i) {
        const int j = i * 32 + lane;
        const unsigned int x = j < G ? __ldcg(v + j) : 0u;
        sa += x;
        if (j < upto) sb += x;
    }
    *below = warp_sum(sb);
    *all = warp_sum(sa);
}

// Cell indices of a batch of cell keys (kEmpty: no lookup, -1): the first
// probes of the whole batch in flight together, then the values of the hits,
// then the rare longer probe sequences one by one.
template <int B>
__device__ __forceinline__ void hash_find_batch(const unsigned long long* hk, const int* hv, unsigned long long mask,
                                                const unsigned long long (&want)[B], int (&found)[B]) {
    unsigned int slot[B];
    unsigned long long got[B];
#pragma unroll
    for (int i = 0; i < B; ++i) slot[i] = static_cast<unsigned int>(hash_slot(want[i], mask));
#pragma unroll
    for (int i = 0; i < B; ++i) got[i] = want[i] != kEmpty ? __ldcg(hk + slot[i]) : kEmpty;
#pragma unroll
    for (int i = 0; i < B; ++i) found[i] = (want[i] != kEmpty && got[i] == want[i]) ? __ldcg(hv + slot[i]) : -1;
#pragma unroll
    for (int i = 0; i < B; ++i) {
        if (want[i] == kEmpty || got[i] == want[i] || got[i] == kEmpty) continue;
        unsigned long long h = (slot[i] + 1ull) & mask;
        for (unsigned long long probe = 1; probe <= mask; ++probe) {
            const unsigned long long k = __ldcg(hk + h);
            if (k == want[i]) { found[i] = __ldcg(hv + h); break; }
            if (k == kEmpty) break;
            h = (h + 1) & mask;
        }
    }
}

// The fused launch's cell table where cell keys leave room (at most 40 bits,
// fewer than 2^24 - 1 cells): entries (cell key << 24 | cell index) in
// buckets of four slots, one 32-byte sector each, filled in slot order; a
// lookup reads its bucket in one sector and finds the cell or an empty slot
// (the key is absent), and moves to the next bucket only past four entries.
constexpr int kCellIdBits = 24;

__device__ __forceinline__ unsigned long long cell_entry(unsigned long long key, int cid) {
    return (key << kCellIdBits) | static_cast<unsigned long long>(cid);
}

__device__ __forceinline__ void cell_insert_packed(unsigned long long* hk, unsigned long long bmask,
                                                   unsigned long long key, int cid) {
    const unsigned long long e = cell_entry(key, cid);
    unsigned long long bk = hash_slot(key, bmask);
    for (unsigned long long probe = 0; probe <= bmask; ++probe) {
        for (int j = 0; j < 4; ++j)
            if (atomicCAS(&hk[4 * bk + j], kEmpty, e) == kEmpty) return;
        bk = (bk + 1) & bmask;
    }
}

template <int B>
__device__ __forceinline__ void cell_find_batch_packed(const unsigned long long* hk, unsigned long long bmask,
                                                       const unsigned long long (&want)[B], int (&found)[B]) {
    unsigned long long ent[B][4];
    unsigned long long bk[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        bk[i] = hash_slot(want[i], bmask);
        if (want[i] != kEmpty) ld_bucket_cg(hk + 4 * bk[i], ent[i]);
        else ent[i][0] = ent[i][1] = ent[i][2] = ent[i][3] = kEmpty;
    }
    const unsigned long long idmask = (1ull << kCellIdBits) - 1;
#pragma unroll
    for (int i = 0; i < B; ++i) {
        found[i] = -1;
        if (want[i] == kEmpty) continue;
        unsigned long long e[4] = {ent[i][0], ent[i][1], ent[i][2], ent[i][3]};
        for (unsigned long long probe = 0; probe <= bmask; ++probe) {
            bool done = false;
            for (int j = 0; j < 4 && !done; ++j) {
                if (e[j] == kEmpty) done = true;
                else if ((e[j] >> kCellIdBits) == want[i]) {
                    found[i] = static_cast<int>(e[j] & idmask);
                    done = true;
                }
            }
            if (done) break;
            bk[i] = (bk[i] + 1) & bmask;   // a full bucket without the key: the next one
            ld_bucket_cg(hk + 4 * bk[i], e);
        }
    }
}

// Key of forward neighbour o of the cell with key `key`, or kEmpty outside the grid.
__device__ __forceinline__ unsigned long long forward_key(const GridParams& g, unsigned long long key, int o) {
    int dx, dy, dz;
    forward_offset(o, dx, dy, dz);
    const int wyz = g.w[1] + g.w[2];
    const unsigned long long rid = key >> (g.w[0] + wyz);
    const long long x = static_cast<long long>((key >> wyz) & ((1ull << g.w[0]) - 1)) + dx;
    const long long y = static_cast<long long>((key >> g.w[2]) & ((1ull << g.w[1]) - 1)) + dy;
    const long long z = static_cast<long long>(key & ((1ull << g.w[2]) - 1)) + dz;
    if (x < 0 || x > g.span[0] || y < 0 || y > g.span[1] || z < 0 || z > g.span[2]) return kEmpty;
    return (rid << (g.w[0] + wyz)) | (static_cast<unsigned long long>(x) << wyz) |
           (static_cast<unsigned long long>(y) << g.w[2]) | static_cast<unsigned long long>(z);
}

// The cell phases both fused launches share, once the step's cell table
// (cell_begin, cell_key, n_cells) and hash are complete: each block's share of
// the cells gets its 13 forward neighbours (lookups spread over the threads),
// its column-list lengths and work-item counts (heavy and light totals per
// block; barrier), then the work list, heavy cells' items first, each group in
// cell order. `clear` runs once the hash is no longer read.
template <typename Clear>
__device__ __forceinline__ void fused_cells_tail(const StepArgs& a, const FusedArgs& f, Ctrl* ctrl, int n,
                                                 unsigned long long hmask, bool packed, const GridParams& g,
                                                 unsigned int* wsum,
                                                 unsigned long long* bsum, int* gave_up, unsigned int* iparts,
                                                 unsigned int* bar, unsigned int& target, int polls, int* flags,
                                                 Clear clear) {
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // Neighbours, column-list lengths and work-item counts of the block's share of the cells.
    const int nc = launch_gave_up(flags, gave_up) ? 0 : max(0, min(__ldcg(&ctrl->n_cells), n));
    const int Rc = (nc + G - 1) / G;
    const int c0 = min(nc, b * Rc), c1 = min(nc, c0 + Rc);
    const int per = f.per;
    unsigned long long cand = 0;
    int biggest = 0;
    unsigned int heavy_sum = 0, light_sum = 0;
    // Forward neighbours: the block's (cell, offset) lookups spread over its
    // threads, kLook at a time per thread with their probes in flight together.
    {
        constexpr int kLook = 6;
        const int total = 13 * (c1 - c0);
        for (int j0 = 0; j0 < total; j0 += kLook * kFusedThreads) {
            unsigned long long want[kLook];
            int found[kLook];
#pragma unroll
            for (int i = 0; i < kLook; ++i) {
                const int j = j0 + i * kFusedThreads + tid;
                want[i] = kEmpty;
                if (j < total) {
                    const int c = c0 + j / 13;
                    want[i] = forward_key(g, __ldcg(f.cell_key + c), j % 13);
                }
            }
            if (packed) {
                // Two halves: each bucket read holds four entries in registers.
                unsigned long long w0[kLook / 2], w1[kLook / 2];
                int f0[kLook / 2], f1[kLook / 2];
#pragma unroll
                for (int i = 0; i < kLook / 2; ++i) {
                    w0[i] = want[i];
                    w1[i] = want[kLook / 2 + i];
                }
                cell_find_batch_packed<kLook / 2>(f.hk, hmask >> 2, w0, f0);
                cell_find_batch_packed<kLook / 2>(f.hk, hmask >> 2, w1, f1);
#pragma unroll
                for (int i = 0; i < kLook / 2; ++i) {
                    found[i] = f0[i];
                    found[kLook / 2 + i] = f1[i];
                }
            } else {
                hash_find_batch<kLook>(f.hk, f.hv, hmask, want, found);
            }
#pragma unroll
            for (int i = 0; i < kLook; ++i) {
                const int j = j0 + i * kFusedThreads + tid;
                if (j < total) f.nbr[13 * static_cast<int64_t>(c0) + j] = (found[i] >= 0 && found[i] < nc) ? found[i] : -1;
            }
        }
    }
    __syncthreads();
    for (int c = c0 + tid; c < c1; c += kFusedThreads) {
        const int b0 = __ldcg(f.cell_begin + c);
        const int kc = __ldcg(f.cell_begin + c + 1) - b0;
        const int* nb = f.nbr + 13 * static_cast<int64_t>(c);
        int fo[13];
#pragma unroll
        for (int o = 0; o < 13; ++o) fo[o] = __ldcg(nb + o);
        int other = 0;
        int nb_begin[13], nb_len[13];
#pragma unroll
        for (int o = 0; o < 13; ++o) {
            nb_begin[o] = fo[o] >= 0 ? __ldcg(f.cell_begin + fo[o]) : 0;
            nb_len[o] = fo[o] >= 0 ? __ldcg(f.cell_begin + fo[o] + 1) - nb_begin[o] : 0;
            other += nb_len[o];
        }
        write_column_table(f.col_tab + 16 * static_cast<int64_t>(c), b0, kc, nb_begin, nb_len);
        const int L = kc + other;
        f.cell_len[c] = L;
        const unsigned int n_items = cell_items((kc + 31) >> 5, (L + 31) >> 5, per);
        if (heavy_cell(kc, L)) heavy_sum += n_items;
        else light_sum += n_items;
        cand += static_cast<unsigned long long>(kc) * (kc - 1) / 2 + static_cast<unsigned long long>(kc) * other;
        biggest = max(biggest, kc);
    }
    cand = warp_sum(cand);
    biggest = warp_max(biggest);
    if (lane == 0) {
        if (cand) atomicAdd(&ctrl->candidates, cand);
        if (biggest > 0) atomicMax(&ctrl->max_cell, biggest);
    }
    {
        unsigned int ht, lt;
        scan_1024(heavy_sum, &ht, wsum);
        scan_1024(light_sum, &lt, wsum);
        if (tid == 0) {
            iparts[b] = ht;
            iparts[G + b] = lt;
        }
    }
    grid_sync(bar, target, polls, flags);
    // Work list: heavy cells' items first, then the light cells', each in cell order.
    if (warp == 0) {
        // Heavy totals, then light: one copy of the code run twice. Code that
        // runs once per launch is fetched from DRAM (the step's traffic has
        // evicted it), so two inlined copies took ~4 us each, this loop ~1.
        unsigned long long hb = 0, ha = 0, lb = 0, la = 0;
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            unsigned long long x, y;
            blocks_sum(iparts + h * G, G, b, &x, &y);
            if (h == 0) {
                hb = x;
                ha = y;
            } else {
                lb = x;
                la = y;
            }
        }
        if (lane == 0) {
            bsum[1] = hb;
            bsum[2] = ha + lb;
            if (b == 0) ctrl->n_items = static_cast<unsigned int>(ha + la);
        }
    }
    __syncthreads();
    // The hash is no longer read in this step.
    clear();
    if (launch_gave_up(flags, gave_up)) return;
    int64_t heavy_base = static_cast<int64_t>(bsum[1]);
    int64_t light_base = static_cast<int64_t>(bsum[2]);
    bool over = false;
    for (int blk = c0; blk < c1; blk += kFusedThreads) {
        const int c = blk + tid;
        int kc = 0, L = 0;
        unsigned int n_items = 0;
        bool heavy = false;
        int b0 = 0;
        if (c < c1) {
            b0 = __ldcg(f.cell_begin + c);
            kc = __ldcg(f.cell_begin + c + 1) - b0;
            L = __ldcg(f.cell_len + c);
            heavy = heavy_cell(kc, L);
            n_items = cell_items((kc + 31) >> 5, (L + 31) >> 5, per);
        }
        unsigned int ht, lt;
        const int64_t hoff = heavy_base + scan_1024(heavy ? n_items : 0u, &ht, wsum);
        const int64_t loff = light_base + scan_1024(c < c1 && !heavy ? n_items : 0u, &lt, wsum);
        heavy_base += ht;
        light_base += lt;
        const bool small = c < c1 && n_items <= 32;
        if (small) {
            const int ta = (kc + 31) >> 5, tc = (L + 31) >> 5;
            int64_t w = heavy ? hoff : loff;
            for (int ra = 0; ra < ta; ++ra)
                for (int cb = ra; cb < tc; cb += per, ++w) {
                    if (w < f.items_cap) f.items[w] = work_item(c, ra, cb, min(per, tc - cb), b0);
                    else over = true;
                }
        }
        // Cells with more than 32 items (all heavy): the warp writes them together.
        unsigned big = __ballot_sync(0xffffffffu, c < c1 && !small);
        while (big) {
            const int src = __ffs(big) - 1;
            big &= big - 1;
            const int cc = blk + (tid & ~31) + src;
            const int kk = __shfl_sync(0xffffffffu, kc, src), LL = __shfl_sync(0xffffffffu, L, src);
            const int bb = __shfl_sync(0xffffffffu, b0, src);
            const int ta = (kk + 31) >> 5, tc = (LL + 31) >> 5;
            int64_t wbase = __shfl_sync(0xffffffffu, hoff, src);
            for (int a0 = 0; a0 < ta; a0 += 32) {
                const int ra = a0 + lane;
                const unsigned int mine = ra < ta ? row_block_items(ra, tc, per) : 0u;
                unsigned int incl = mine;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                int64_t w = wbase + (incl - mine);
                for (int cb = ra; ra < ta && cb < tc; cb += per, ++w) {
                    if (w < f.items_cap) f.items[w] = work_item(cc, ra, cb, min(per, tc - cb), bb);
                    else over = true;
                }
                wbase += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
    }
    if (over) atomicOr(flags, FLAG_ITEMS_OVERFLOW);
}

template <int K, int DB>
__global__ void __launch_bounds__(kFusedThreads, 1) k_sort_cells(StepArgs a, FusedArgs f) {
    constexpr int ND = 1 << DB;              // digits of a pass
    constexpr unsigned DM = ND - 1;
    constexpr int kPer = ND / kFusedThreads > 0 ? ND / kFusedThreads : 1;  // digits per thread in digit loops
    extern __shared__ __align__(16) unsigned char fused_smem[];
    // Per-warp digit counters (u16: a warp holds at most 32 K keys), then the
    // stage of the scatter, then per-digit starts.
    unsigned short* wcnt = reinterpret_cast<unsigned short*>(fused_smem);                              // [32][ND]
    unsigned long long* stage = reinterpret_cast<unsigned long long*>(fused_smem + 2 * 32 * ND);      // [1024 K]
    unsigned int* dstart = reinterpret_cast<unsigned int*>(stage + kFusedThreads * K);  // block-local start of each digit
    unsigned int* dglob = dstart + ND;     // start of each digit in the output
    int* gshift = reinterpret_cast<int*>(dglob + ND);   // output position minus block-local position
    __shared__ unsigned int wsum[32];
    __shared__ unsigned int whead[32];     // cell heads of each warp, then their exclusive prefix
    __shared__ unsigned long long bsum[4];
    __shared__ int gave_up;
    __shared__ unsigned int block_heads;
    __shared__ GridParams g;

    Ctrl* ctrl = a.ctrl;
    if (step_void(ctrl)) return;
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned int* bar = f.scratch;
    unsigned int* totals = f.scratch + 32;                 // [passes][ND]
    unsigned int* heads = f.scratch + kFusedZeroWords;     // [G]
    unsigned int* iparts = heads + G;                      // [2 G]: heavy, then light items per block
    unsigned int* counts = iparts + 2 * G;                 // [G][ND]
    unsigned int* offs = counts + kFusedDigits * G;        // [G][ND]
    int* flags = &ctrl->flags;
    const int polls = a.tune.lookback_polls;
    unsigned int target = 0;
    int n = a.n;
    if (a.n_live) n = min(n, *a.n_live);
    const int R = (n + G - 1) / G;
    const int lo = min(n, b * R);
    const int cnt = min(min(n, lo + R) - lo, K * kFusedThreads);
    // The key bits [pack_bits, pack_bits + 8 sort_passes) in passes of DB bits.
    const int passes = (8 * a.sort_passes + DB - 1) / DB;
    const bool by_ballot = a.tune.sort_rank_ballot != 0;

    unsigned long long k[K];
    for (int pass = 0; pass < passes; ++pass) {
        const unsigned long long* in = f.keys[pass & 1];
        unsigned long long* out = f.keys[(pass & 1) ^ 1];
        const int shift = a.pack_bits + DB * pass;
        for (int i = tid; i < 32 * ND / 2; i += kFusedThreads) reinterpret_cast<unsigned int*>(wcnt)[i] = 0u;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const int li = warp * 32 * K + r * 32 + lane;
            k[r] = li < cnt ? __ldcg(in + lo + li) : 0ull;
        }
        __syncthreads();
        // Rank: place of each key among the block's keys of its digit, by warp.
        unsigned int rk[K];
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const bool valid = warp * 32 * K + r * 32 + lane < cnt;
            const unsigned d = static_cast<unsigned>(k[r] >> shift) & DM;
            const unsigned peers = digit_peers<DB>(d, valid, by_ballot);
            const unsigned int prior = valid ? wcnt[warp * ND + d] : 0u;
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) wcnt[warp * ND + d] = static_cast<unsigned short>(prior + __popc(peers));
            __syncwarp();
            rk[r] = prior + __popc(peers & lanemask_lt());
        }
        __syncthreads();
        // Per digit: the warps' exclusive prefix (in place) and the block's
        // count; thread t owns digits kPer t .. kPer t + kPer - 1.
        unsigned int tot[kPer];
        unsigned int mine = 0;
#pragma unroll
        for (int e = 0; e < kPer; ++e) {
            const int d = kPer * tid + e;
            unsigned int run = 0;
            if (d < ND) {
                for (int w = 0; w < kFusedWarps; ++w) {
                    const unsigned int c = wcnt[w * ND + d];
                    wcnt[w * ND + d] = static_cast<unsigned short>(run);
                    run += c;
                }
            }
            tot[e] = run;
            mine += run;
        }
        unsigned int unused;
        unsigned int start = scan_1024(mine, &unused, wsum);
#pragma unroll
        for (int e = 0; e < kPer; ++e) {
            const int d = kPer * tid + e;
            if (d < ND) {
                dstart[d] = start;
                counts[b * ND + d] = tot[e];
                if (tot[e]) atomicAdd(&totals[pass * ND + d], tot[e]);
            }
            start += tot[e];
        }
        grid_sync(bar, target, polls, flags);
        // Starts: digit d's place in the output, then each block's within it.
        {
            unsigned int tv[kPer];
            unsigned int sum = 0;
#pragma unroll
            for (int e = 0; e < kPer; ++e) {
                const int d = kPer * tid + e;
                tv[e] = d < ND ? __ldcg(totals + pass * ND + d) : 0u;
                sum += tv[e];
            }
            unsigned int run = scan_1024(sum, &unused, wsum);
#pragma unroll
            for (int e = 0; e < kPer; ++e) {
                const int d = kPer * tid + e;
                if (d < ND) dglob[d] = run;
                run += tv[e];
            }
        }
        __syncthreads();
        if constexpr (4 * ND <= kFusedThreads) {
            // Each block its own starts, without a second barrier: digit d's
            // keys of the blocks below it are the column sum of the count
            // matrix over rows j < b, or, for the upper half of the blocks,
            // the digit's total minus the rows j >= b (at most G / 2 rows,
            // split over kFusedThreads / ND threads per digit, coalesced
            // across the digits of a row).
            constexpr int kParts = kFusedThreads / ND;
            unsigned int* psum = reinterpret_cast<unsigned int*>(stage);   // [kParts][ND]; the stage is free
            const int d = tid % ND, part = tid / ND;
            const bool upper = 2 * b >= G;
            const int j0 = upper ? b : 0, span = upper ? G - b : b;
            const int r0 = j0 + span * part / kParts, r1 = j0 + span * (part + 1) / kParts;
            unsigned int acc = 0;
#pragma unroll 4
            for (int j = r0; j < r1; ++j) acc += __ldcg(counts + j * ND + d);
            psum[part * ND + d] = acc;
            __syncthreads();
            if (tid < ND) {
                unsigned int sum = 0;
#pragma unroll
                for (int q = 0; q < kParts; ++q) sum += psum[q * ND + tid];
                const unsigned int below = upper ? __ldcg(totals + pass * ND + tid) - sum : sum;
                gshift[tid] = static_cast<int>(dglob[tid] + below) - static_cast<int>(dstart[tid]);
            }
            __syncthreads();
        } else {
            for (int d = b + warp * G; d < ND; d += kFusedWarps * G) {
                constexpr int kSeg = kFusedMaxGrid / 32;
                const int S = (G + 31) / 32;
                unsigned int c[kSeg];
                unsigned int seg = 0;
#pragma unroll
                for (int i = 0; i < kSeg; ++i) {
                    const int j = lane * S + i;
                    c[i] = (i < S && j < G) ? __ldcg(counts + j * ND + d) : 0u;
                    seg += c[i];
                }
                unsigned int incl = seg;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                unsigned int run = dglob[d] + incl - seg;
#pragma unroll
                for (int i = 0; i < kSeg; ++i) {
                    const int j = lane * S + i;
                    if (i < S && j < G) offs[j * ND + d] = run;
                    run += c[i];
                }
            }
            grid_sync(bar, target, polls, flags);
            for (int d = tid; d < ND; d += kFusedThreads)
                gshift[d] = static_cast<int>(__ldcg(offs + b * ND + d)) - static_cast<int>(dstart[d]);
        }
        // Scatter: stage in digit order, store each digit's run from the block's start.
#pragma unroll
        for (int r = 0; r < K; ++r) {
            if (warp * 32 * K + r * 32 + lane < cnt) {
                const unsigned d = static_cast<unsigned>(k[r] >> shift) & DM;
                stage[dstart[d] + wcnt[warp * ND + d] + rk[r]] = k[r];
            }
        }
        __syncthreads();
        for (int q = tid; q < cnt; q += kFusedThreads) {
            const unsigned long long kk = stage[q];
            const int dst = gshift[static_cast<unsigned>(kk >> shift) & DM] + q;
            if (dst >= 0 && dst < n) out[dst] = kk;
        }
        grid_sync(bar, target, polls, flags);
    }

    // ---- cells ----
    const unsigned long long* sk = f.keys[passes & 1];
    if (tid == 0) g = ctrl->grid;
    __syncthreads();
    const bool skip = launch_gave_up(flags, &gave_up);
    const int m = skip ? 0 : min(ctrl->n_alive, n);
    const int sh = 3 * g.sub + a.pack_bits;
    const unsigned long long idx_mask = (1ull << a.pack_bits) - 1;
    unsigned int bal[K];
    unsigned int warp_heads = 0;
#pragma unroll
    for (int r = 0; r < K; ++r) {
        const int li = warp * 32 * K + r * 32 + lane;
        const int p = lo + li;
        const bool valid = li < cnt && p < m;
        unsigned long long key = 0, prev = 0;
        if (valid) {
            key = __ldcg(sk + p);
            if (p > 0) prev = __ldcg(sk + p - 1);
        }
        k[r] = key;
        bal[r] = __ballot_sync(0xffffffffu, valid && (p == 0 || (key >> sh) != (prev >> sh)));
        warp_heads += __popc(bal[r]);
    }
    if (lane == 0) whead[warp] = warp_heads;
    __syncthreads();
    if (warp == 0) {
        const unsigned int x = whead[lane];
        unsigned int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        whead[lane] = incl - x;
        if (lane == 31) {
            heads[b] = incl;
            block_heads = incl;
        }
    }
    grid_sync(bar, target, polls, flags);
    // Cells opened by the block's keys: ranges, keys, hash entries.
    if (warp == 0) {
        unsigned long long below, all;
        blocks_sum(heads, G, b, &below, &all);
        if (lane == 0) {
            bsum[0] = below;
            bsum[3] = all;
        }
    }
    __syncthreads();
    // The table in use this step, the same in every block (all cell counts
    // are in): by default (hash_slots_per_cell 0), where the cell keys leave
    // room, the packed bucketed table with 4 slots per cell (at 1M objects 87k
    // cells in 512k slots, 4 MB, in L2); else (key, cell) pairs over
    // hash_slots_per_cell slots per cell, or over the whole table. Either way
    // a power of two of slots at most the table's, whose prefix in use is
    // cleared again at the end.
    const bool packed = a.tune.hash_slots_per_cell == 0 && g.bits - 3 * g.sub <= 64 - kCellIdBits &&
                        bsum[3] + 1 < (1ull << kCellIdBits);
    const unsigned long long per_cell = packed ? 4ull : static_cast<unsigned long long>(a.tune.hash_slots_per_cell);
    unsigned long long hmask = per_cell > 0 ? 63 : f.hmask;
    while (hmask < f.hmask && hmask + 1 < per_cell * bsum[3]) hmask = 2 * hmask + 1;
    {
        // The block's cells take consecutive indices from `first`: ranges and
        // keys stored from registers, keys listed in shared memory (the
        // stage of the sort is free now) for the hash inserts, one per thread.
        const unsigned int first = static_cast<unsigned int>(bsum[0]);
        const unsigned int base = whead[warp];
        unsigned int earlier = 0;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const int li = warp * 32 * K + r * 32 + lane;
            const int p = lo + li;
            const bool head = (bal[r] >> lane) & 1u;
            const unsigned int local = base + earlier + __popc(bal[r] & lanemask_lt()) + (head ? 1u : 0u) - 1u;
            const int cid = static_cast<int>(first + local);
            if (head && cid >= 0 && cid < n) {
                const unsigned long long key = k[r] >> sh;
                f.cell_begin[cid] = p;
                f.cell_key[cid] = key;
                stage[local] = key;
            }
            if (li < cnt && p == m - 1 && cid >= 0 && cid < n) {
                ctrl->n_cells = cid + 1;
                f.cell_begin[cid + 1] = m;
            }
            earlier += __popc(bal[r]);
        }
        if (m == 0 && !skip && b == 0 && tid == 0) {
            ctrl->n_cells = 0;
            f.cell_begin[0] = 0;
        }
        __syncthreads();
        const int nh = min(static_cast<int>(block_heads), cnt);
        for (int i = tid; i < nh; i += kFusedThreads) {
            const int cid = static_cast<int>(first) + i;
            if (cid >= n) break;
            const unsigned long long key = stage[i];
            if (packed) {
                cell_insert_packed(f.hk, hmask >> 2, key, cid);
                continue;
            }
            unsigned long long h = hash_slot(key, hmask);
            for (unsigned long long probe = 0; probe <= hmask; ++probe) {
                const unsigned long long prev = atomicCAS(&f.hk[h], kEmpty, key);
                if (prev == kEmpty || prev == key) {
                    f.hv[h] = cid;
                    break;
                }
                h = (h + 1) & hmask;
            }
        }
    }
    grid_arrive(bar, target);
    // Records in cell order (read only by the pair kernel, after this launch).
#pragma unroll
    for (int r0 = 0; r0 < K; r0 += 4) {
        int o[4];
        unsigned long long kk[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int li = (r0 + j) * kFusedThreads + tid;
            const int p = lo + li;
            kk[j] = (r0 + j < K && li < cnt && p < m) ? __ldcg(sk + p) : kEmpty;
            const unsigned long long oi = kk[j] & idx_mask;
            o[j] = (kk[j] != kEmpty && oi < static_cast<unsigned long long>(n)) ? static_cast<int>(oi) : -1;
        }
        if (!f.sorted) {
            Rec32 rr[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (o[j] < 0) continue;
                rr[j] = ld_rec32(f.rec32 + 2 * static_cast<int64_t>(o[j]));
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (o[j] < 0) continue;
                const int64_t p = lo + (r0 + j) * kFusedThreads + tid;
                f.sorted_orig[p] = o[j];
                st_rec32(f.sorted32 + 2 * p, rr[j]);
            }
        } else {
            double2 st[4][3];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (o[j] < 0) continue;
                const double2* src = reinterpret_cast<const double2*>(f.before + 6 * static_cast<int64_t>(o[j]));
                st[j][0] = src[0];
                st[j][1] = src[1];
                st[j][2] = src[2];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (o[j] < 0) continue;
                const int64_t p = lo + (r0 + j) * kFusedThreads + tid;
                f.sorted_orig[p] = o[j];
                double2* dst = reinterpret_cast<double2*>(f.sorted + 6 * p);
                dst[0] = st[j][0];
                dst[1] = st[j][1];
                dst[2] = st[j][2];
                if (f.sorted32)
                    f32_record(g, kk[j] >> a.pack_bits, st[j][0].x, st[j][0].y, st[j][1].x, st[j][1].y, st[j][2].x,
                               st[j][2].y, f.sorted32 + 2 * p);
            }
        }
    }
    grid_wait(bar, target, polls, flags);
    // Neighbours, column-list lengths and work-item counts, then the work list;
    // the hash is cleared for the next step once no longer read (a chunk also
    // clears it once before its first step).
    fused_cells_tail(a, f, ctrl, n, hmask, packed, g, wsum, bsum, &gave_up, iparts, bar, target, polls, flags, [&]() {
        ulonglong2* h2 = reinterpret_cast<ulonglong2*>(f.hk);
        const int64_t words = static_cast<int64_t>((hmask + 1) >> 1);
        for (int64_t i = static_cast<int64_t>(b) * kFusedThreads + tid; i < words;
             i += static_cast<int64_t>(G) * kFusedThreads)
            h2[i] = make_ulonglong2(kEmpty, kEmpty);
    });
}


// Blocks of the fused kernel per device (0: not available), set up on first use.
std::atomic<int> g_fused_grid[kMaxSmDevices];

// Dynamic shared memory of k_sort_cells<K, DB>: per-warp u16 digit counters,
// the stage of K keys per thread, three u32 per digit.
size_t fused_smem_bytes(int K, int DB) {
    const size_t nd = size_t(1) << DB;
    return 2 * 32 * nd + sizeof(unsigned long long) * kFusedThreads * K + 3 * 4 * nd;
}

int grid_for_block(int64_t n, int per_sm_blocks, int block) {
    const int sms = sm_count();
    const int64_t want = (n + block - 1) / block;
    const int64_t cap = static_cast<int64_t>(sms) * per_sm_blocks;
    return static_cast<int>(want < 1 ? 1 : (want < cap ? want : cap));
}

int grid_for(int64_t n, int per_sm_blocks) {
    const int sms = sm_count();
    const int64_t want = (n + kBlock - 1) / kBlock;
    const int64_t cap = static_cast<int64_t>(sms) * per_sm_blocks;
    return static_cast<int>(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
    if (dev >= kMaxSmDevices) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return sms > 0 ? sms : 1;
    }
    int sms = g_sm_count[dev].load(std::memory_order_relaxed);
    if (sms == 0) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
        g_sm_count[dev].store(sms, std::memory_order_relaxed);
    }
    return sms;
}

int fused_grid() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxSmDevices) return 0;
    const int known = g_fused_grid[dev].load(std::memory_order_relaxed);
    if (known != 0) return known > 0 ? known : 0;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    int blocks = coop ? sm_count() : 0;
    if (blocks > kFusedMaxGrid) blocks = 0;
    bool failed = false;
    auto setup = [&](auto kernel, int K, int DB) {
        if (blocks <= 0) return;
        const int smem = static_cast<int>(fused_smem_bytes(K, DB));
        int occ = 0;
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kFusedThreads, smem) != cudaSuccess) {
            failed = true;
            blocks = 0;
        } else if (occ < 1) {
            blocks = 0;
        }
    };
    setup(k_sort_cells<4, 8>, 4, 8);
    setup(k_sort_cells<8, 8>, 8, 8);
    setup(k_sort_cells<12, 8>, 12, 8);
    setup(k_sort_cells<4, 11>, 4, 11);
    setup(k_sort_cells<8, 11>, 8, 11);
    if (failed) cudaGetLastError();  // the attribute query's error, not a launch's
    g_fused_grid[dev].store(blocks > 0 ? blocks : -1, std::memory_order_relaxed);
    return blocks;
}

int64_t fused_scratch_words(int grid) {
    return kFusedZeroWords + 3 * static_cast<int64_t>(grid) + 2 * static_cast<int64_t>(kFusedDigits) * grid;
}

namespace {
int fused_keys_per_thread(int64_t n, int grid) {
    if (grid <= 0) return 0;
    const int64_t r = (n + grid - 1) / grid;
    for (int K : {4, 8, 12})
        if (r <= static_cast<int64_t>(K) * kFusedThreads) return K;
    return 0;
}
}  // namespace

bool sort_cells_fused(const DeviceBuffers& b, const StepArgs& a) {
    if (!a.tune.sort_fused || !b.fused || a.pack_bits <= 0 || a.n <= 0) return false;
    if (a.sort_passes < 1 || a.sort_passes > 8 || a.pack_bits + 8 * a.sort_passes > 64) return false;
    const int grid = fused_grid();
    return grid > 0 && grid <= b.fused_grid && fused_keys_per_thread(a.n, grid) > 0;
}

// Digit width of the fused sort: 8 bits, or with tuning "sort_digit_bits" 11,
// 11 bits (three passes where 8-bit digits take four) where its counters fit
// next to the keys (K <= 8) and it saves a pass. At 1M objects the 11-bit form
// is slower (173 vs 130 us a step): its 128 KB of per-warp counters leave L1
// a fifth of its room for the cell phases' gathers and probes.
int fused_digit_bits(const StepArgs& a, int K) {
    if (a.tune.sort_digit_bits != 11 || K > 8) return 8;
    return (8 * a.sort_passes + 10) / 11 < a.sort_passes ? 11 : 8;
}

void launch_sort_cells(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int grid = fused_grid();
    const int K = fused_keys_per_thread(a.n, grid);
    const int DB = fused_digit_bits(a, K);
    cudaMemsetAsync(b.fused, 0, sizeof(unsigned int) * kFusedZeroWords, stream);
    FusedArgs f{};
    f.keys[0] = b.keys[0];
    f.keys[1] = b.keys[1];
    f.scratch = b.fused;
    f.cell_begin = b.cell_begin;
    f.cell_key = b.cell_key;
    f.hk = b.hash_keys;
    f.hv = b.hash_vals;
    f.hmask = static_cast<unsigned long long>(b.hash_cap - 1);
    f.before = b.state[a.src];
    f.sorted = f32_records(a) ? nullptr : b.sorted;
    f.sorted_orig = b.sorted_orig;
    f.sorted32 = f32_records(a) ? b.sorted32 : nullptr;
    f.rec32 = b.rec32;
    f.nbr = b.nbr;
    f.cell_len = b.cell_len;
    f.col_tab = b.col_tab;
    f.items = b.items;
    f.items_cap = b.items_cap;
    f.per = a.tune.item_col_blocks;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = fused_smem_bytes(K, DB);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (DB == 11) {
        if (K == 4) cudaLaunchKernelEx(&cfg, k_sort_cells<4, 11>, a, f);
        else cudaLaunchKernelEx(&cfg, k_sort_cells<8, 11>, a, f);
    } else if (K == 4) {
        cudaLaunchKernelEx(&cfg, k_sort_cells<4, 8>, a, f);
    } else if (K == 8) {
        cudaLaunchKernelEx(&cfg, k_sort_cells<8, 8>, a, f);
    } else {
        cudaLaunchKernelEx(&cfg, k_sort_cells<12, 8>, a, f);
    }
}

void launch_chunk_init(const DeviceBuffers& b, int k_steps, cudaStream_t stream, bool checkpoint) {
    k_chunk_init<<<1, kBlock, 0, stream>>>(b.ctrl, k_steps, b.ctrl + b.ctrl_len - 2, b.chunk,
                                           checkpoint ? b.ctrl + b.ctrl_len - 1 : nullptr);
}

void launch_seed_ctrl(const DeviceBuffers& b, int n, int src, Ctrl* target, int use_alive_src, cudaStream_t stream) {
    k_ctrl_reset<<<1, 32, 0, stream>>>(target);
    k_seed_ctrl<<<grid_for(n, 4), kBlock, 0, stream>>>(b.state[src], use_alive_src ? b.alive[src] : b.alive[1 - src],
                                                        n, target);
}

void launch_propagate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    if (a.precision == KS_PRECISION_SPLIT) {
        k_propagate_split<<<grid_for_block(a.n, 5 * kPropBlock / a.tune.prop_block, a.tune.prop_block), a.tune.prop_block, 0, stream>>>(
            a, b.state[a.src], b.state[1 - a.src], b.alive[a.src], b.alive[1 - a.src], b.keys[0]);
        return;
    }
    // Resident blocks per SM of 128 threads: 4 (registers for the whole RK4
    // in flight) or, by the tuning knob, 5 or 6 (fewer registers, more warps).
    const int mb = a.tune.prop_min_blocks;
    const int grid = grid_for_block(a.n, mb * kPropBlock / a.tune.prop_block, a.tune.prop_block);
    if (mb >= 6)
        k_propagate_exact<6><<<grid, a.tune.prop_block, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src],
                                                                      b.alive[a.src], b.alive[1 - a.src], b.keys[0]);
    else if (mb == 5)
        k_propagate_exact<5><<<grid, a.tune.prop_block, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src],
                                                                      b.alive[a.src], b.alive[1 - a.src], b.keys[0]);
    else
        k_propagate_exact<4><<<grid, a.tune.prop_block, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src],
                                                                      b.alive[a.src], b.alive[1 - a.src], b.keys[0]);
}

void launch_advance_spans(const ForceConsts& fc, const FragSpan* spans, const int* row_span, int64_t first,
                          int count, double* state, uint8_t* alive, cudaStream_t stream) {
    if (count <= 0) return;
    k_advance_spans<<<(count + kPropBlock - 1) / kPropBlock, kPropBlock, 0, stream>>>(fc, spans, row_span, first,
                                                                                      count, state, alive);
}

void launch_gather_rows(const double* before, const double* after, const int64_t* idx, int count, double* rows,
                        cudaStream_t stream) {
    if (count <= 0) return;
    k_gather_rows<<<(12 * count + kBlock - 1) / kBlock, kBlock, 0, stream>>>(before, after, idx, count, rows);
}

void launch_clear_alive(uint8_t* alive, const int64_t* idx, int count, cudaStream_t stream) {
    if (count <= 0) return;
    k_clear_alive<<<(count + kBlock - 1) / kBlock, kBlock, 0, stream>>>(alive, idx, count);
}

void launch_screen_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_screen_keys<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a, b.state[a.src], b.alive[1 - a.src], b.keys[0]);
}

void launch_fix_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_fix_keys<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a, b.state[a.src], b.alive[1 - a.src], b.keys[0]);
}

void launch_sort(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int n = a.n;
    if (n <= 0) return;  // nothing alive: the cell build sees n_alive == 0
    const int ntiles = (n + kSortTile - 1) / kSortTile;
    const int passes = a.sort_passes;
    // With a.hist the propagation counted the digits (launch_propagate's
    // caller cleared the histogram before it); otherwise count them here.
    const bool counted = a.hist != nullptr;
    if (!counted) cudaMemsetAsync(b.sort_hist, 0, sizeof(unsigned int) * 8 * 256, stream);
    cudaMemsetAsync(b.sort_ctr, 0, sizeof(unsigned int) * 8, stream);
    cudaMemsetAsync(b.sort_status, 0, sizeof(unsigned int) * 256 * static_cast<size_t>(ntiles) * passes, stream);
    // Counted by the propagation (and, if it rebuilt the keys, by k_fix_keys):
    // no counting pass of its own.
    if (!counted)
        k_sort_upsweep<<<ntiles, kBlock, 0, stream>>>(b.keys[0], n, a.n_live, passes, b.sort_hist, a.ctrl, 0,
                                                      a.pack_bits);
    for (int pass = 0; pass < passes; ++pass) {
        const int in = pass & 1, outb = 1 - in;
        k_sort_onesweep<<<ntiles, kBlock, 0, stream>>>(
            b.keys[in], pass == 0 ? nullptr : b.idx[in], b.keys[outb], b.idx[outb], n, a.n_live,
            a.pack_bits + 8 * pass, b.sort_hist + 256 * pass, counted ? b.sort_hist + 8 * 256 + 256 * pass : nullptr,
            b.sort_status + 256 * static_cast<size_t>(ntiles) * pass,
            b.sort_ctr + pass, &a.ctrl->flags, a.pack_bits > 0 ? 1 : 0, a.tune.lookback_polls, a.tune.sort_rank_ballot);
    }
}

// Key of each of the chunk's records: floor(2^32 (t - t_start) / span),
// clamped, a non-decreasing function of t, above the record's index.
__global__ void __launch_bounds__(kBlock) k_conj_keys(const ks_conjunction* __restrict__ conj, int64_t cap,
                                                      ChunkCtrl* chunk, const double* __restrict__ t_start,
                                                      double span_s, unsigned long long* __restrict__ keys,
                                                      int pack_bits) {
    const int n = static_cast<int>(min(chunk->conj_count, static_cast<unsigned long long>(cap)));
    if (blockIdx.x == 0 && threadIdx.x == 0) chunk->sort_n = n;
    const double t0 = *t_start;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const double f = xmul(xdiv(xsub(conj[q].t, t0), span_s), 4294967296.0);
        const double c = fmin(fmax(floor(f), 0.0), 4294967295.0);
        keys[q] = (static_cast<unsigned long long>(c) << pack_bits) | static_cast<unsigned long long>(q);
    }
}

__global__ void __launch_bounds__(kBlock) k_conj_gather(const ks_conjunction* __restrict__ conj,
                                                        const unsigned long long* __restrict__ order,
                                                        unsigned long long mask, const ChunkCtrl* chunk,
                                                        ks_conjunction* __restrict__ out) {
    const int n = chunk->sort_n;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        out[q] = conj[static_cast<int>(order[q] & mask)];
}

// Up to kConjSmall records of a chunk ordered by one block: the keys of
// k_conj_keys (14 index bits here) sorted by a bitonic network in shared
// memory, then the records gathered. With more records it sets
// FLAG_CONJ_LARGE and leaves them to the multi-block sort.
// (t, i, j) order of records (src/core/collision.cpp:743-747).
__device__ __forceinline__ bool conj_before(const ks_conjunction& a, const ks_conjunction& b) {
    if (a.t != b.t) return a.t < b.t;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
}

// Records ordered by a key monotone in t keep, among those sharing a key, the
// order they were appended in: the thread at the start of such a run orders it
// by (t, i, j) in place (insertion sort; runs are a few records). A run longer
// than kTieRun is left to the host (FLAG_CONJ_TIES).
constexpr int kTieRun = 64;
template <typename KeyAt>
__device__ __forceinline__ void order_tie_run(int q, int n, KeyAt key_at, ks_conjunction* __restrict__ out,
                                              ChunkCtrl* chunk) {
    const unsigned long long k = key_at(q);
    if (q > 0 && key_at(q - 1) == k) return;
    int e = q + 1;
    while (e < n && e - q <= kTieRun && key_at(e) == k) ++e;
    if (e - q < 2) return;
    if (e - q > kTieRun) {
        atomicOr(&chunk->flags, FLAG_CONJ_TIES);
        return;
    }
    for (int u = q + 1; u < e; ++u) {
        const ks_conjunction v = out[u];
        int w = u;
        while (w > q && conj_before(v, out[w - 1])) {
            out[w] = out[w - 1];
            --w;
        }
        out[w] = v;
    }
}

__global__ void __launch_bounds__(kBlock) k_conj_ties(const unsigned long long* __restrict__ order, int pb,
                                                      ChunkCtrl* chunk, ks_conjunction* __restrict__ out) {
    const int n = chunk->sort_n;
    auto key_at = [&](int p) { return order[p] >> pb; };
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        order_tie_run(q, n, key_at, out, chunk);
}

__global__ void __launch_bounds__(1024) k_conj_sort_small(const ks_conjunction* __restrict__ conj, int64_t cap,
                                                          ChunkCtrl* chunk, const double* __restrict__ t_start,
                                                          double span_s, ks_conjunction* __restrict__ out) {
    extern __shared__ unsigned long long sk[];
    const int n = static_cast<int>(min(chunk->conj_count, static_cast<unsigned long long>(cap)));
    if (n > kConjSmall) {
        if (threadIdx.x == 0) {
            chunk->sort_n = 0;
            atomicOr(&chunk->flags, FLAG_CONJ_LARGE);
        }
        return;
    }
    if (threadIdx.x == 0) chunk->sort_n = n;
    int m = 2;
    while (m < n) m <<= 1;
    const double t0 = *t_start;
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        unsigned long long key = ~0ull;  // padding sorts last
        if (q < n) {
            const double f = xmul(xdiv(xsub(conj[q].t, t0), span_s), 4294967296.0);
            const double c = fmin(fmax(floor(f), 0.0), 4294967295.0);
            key = (static_cast<unsigned long long>(c) << 14) | static_cast<unsigned long long>(q);
        }
        sk[q] = key;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int p = i ^ j;
                if (p > i) {
                    const unsigned long long a = sk[i], b = sk[p];
                    if ((a > b) == ((i & k) == 0)) {
                        sk[i] = b;
                        sk[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int q = threadIdx.x; q < n; q += blockDim.x) out[q] = conj[static_cast<int>(sk[q] & 0x3FFFull)];
    __syncthreads();
    auto key_at = [&](int p) { return sk[p] >> 14; };
    for (int q = threadIdx.x; q < n; q += blockDim.x) order_tie_run(q, n, key_at, out, chunk);
}

void launch_conj_sort(const DeviceBuffers& b, ChunkCtrl* chunk, const double* t_start, double span_s, bool small,
                      cudaStream_t stream) {
    const int cap = static_cast<int>(b.conj_cap);
    if (cap <= 0) return;
    if (small) {
        constexpr int kBytes = kConjSmall * sizeof(unsigned long long);
        cudaFuncSetAttribute(k_conj_sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize, kBytes);
        k_conj_sort_small<<<1, 1024, kBytes, stream>>>(b.conj, b.conj_cap, chunk, t_start, span_s, b.conj_sorted);
        return;
    }
    constexpr int kPasses = 4;
    const int ntiles = (cap + kSortTile - 1) / kSortTile;
    int pb = 1;  // record index bits below the 32-bit key
    while ((1ll << pb) < cap) ++pb;
    cudaMemsetAsync(b.conj_hist, 0, sizeof(unsigned int) * 8 * 256, stream);
    cudaMemsetAsync(b.conj_ctr, 0, sizeof(unsigned int) * 8, stream);
    cudaMemsetAsync(b.conj_status, 0, sizeof(unsigned int) * 256 * static_cast<size_t>(ntiles) * kPasses, stream);
    k_conj_keys<<<sm_count() * 4, kBlock, 0, stream>>>(b.conj, b.conj_cap, chunk, t_start, span_s, b.conj_keys[0],
                                                       pb);
    k_sort_upsweep<<<ntiles, kBlock, 0, stream>>>(b.conj_keys[0], cap, &chunk->sort_n, kPasses, b.conj_hist, nullptr,
                                                  0, pb);
    for (int pass = 0; pass < kPasses; ++pass) {
        const int in = pass & 1, outb = 1 - in;
        k_sort_onesweep<<<ntiles, kBlock, 0, stream>>>(
            b.conj_keys[in], nullptr, b.conj_keys[outb], nullptr, cap, &chunk->sort_n, pb + 8 * pass,
            b.conj_hist + 256 * pass, nullptr, b.conj_status + 256 * static_cast<size_t>(ntiles) * pass, b.conj_ctr + pass,
            &chunk->flags, 1, kLookbackLimit, 0);
    }
    k_conj_gather<<<sm_count() * 4, kBlock, 0, stream>>>(b.conj, b.conj_keys[kPasses & 1], (1ull << pb) - 1, chunk,
                                                         b.conj_sorted);
    k_conj_ties<<<sm_count() * 4, kBlock, 0, stream>>>(b.conj_keys[kPasses & 1], pb, chunk, b.conj_sorted);
}

// The pair kernel gates on FP32 cell-relative records (and decides with the
// exact FP64 filter): always in split precision, and in FP64 precision with
// pair variant 2.
bool f32_records(const StepArgs& a) { return a.precision == KS_PRECISION_SPLIT || a.tune.pair_variant == 2; }

void launch_cells(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int sb = sorted_buffer(a.sort_passes);
    const int ntiles = a.n > 0 ? (a.n + kCellTile - 1) / kCellTile : 1;
    unsigned int* bc = reinterpret_cast<unsigned int*>(b.block_counts);
    k_cell_count<<<ntiles, kBlock, 0, stream>>>(b.keys[sb], a.ctrl, bc, a.pack_bits);
    k_scan_small<<<1, 1024, 0, stream>>>(bc, ntiles, nullptr, nullptr, 1);
    cudaMemsetAsync(b.hash_keys, 0xFF, sizeof(unsigned long long) * b.hash_cap, stream);
    k_cell_write<<<ntiles, kBlock, 0, stream>>>(b.keys[sb], b.idx[sb], bc, a.ctrl, b.cell_begin, b.cell_key,
                                               b.hash_keys, b.hash_vals,
                                               static_cast<unsigned long long>(b.hash_cap - 1), b.state[a.src],
                                               f32_records(a) ? nullptr : b.sorted, b.sorted_orig,
                                               f32_records(a) ? b.sorted32 : nullptr, b.rec32, a.pack_bits);
    k_neighbours<<<grid_for(13 * static_cast<int64_t>(a.n), 8), kBlock, 0, stream>>>(
        a.ctrl, b.cell_key, b.hash_keys, b.hash_vals, static_cast<unsigned long long>(b.hash_cap - 1), b.nbr);
    // Left empty for the fused launches, which take it so.
    cudaMemsetAsync(b.hash_keys, 0xFF, sizeof(unsigned long long) * b.hash_cap, stream);
    k_items_count<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a.ctrl, b.cell_begin, b.nbr, b.cell_len, b.col_tab, b.item_part,
                                                           a.tune.item_col_blocks);
    // Offsets of the heavy, then the light cells' items per chunk of cells, and their total.
    k_scan_small<<<1, 1024, 0, stream>>>(b.item_part, static_cast<int>(2 * ((b.cap + kBlock - 1) / kBlock)),
                                         &a.ctrl->n_items, &a.ctrl->n_cells, 2);
    k_items_write<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a.ctrl, b.cell_begin, b.cell_len, b.item_part, b.items,
                                                           b.items_cap, a.tune.item_col_blocks);
}

void launch_pairs(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    // Default: the resident block count of each kernel.
    if (f32_records(a)) {
        // Register budget for 3 resident blocks per SM (80 registers), for 4
        // (64; the default: the higher occupancy outweighs a few spilled
        // registers) or for 5 (48; the most its shared memory allows).
        const int bps = a.tune.pair_blocks_per_sm > 0 ? a.tune.pair_blocks_per_sm : 4;
        if (bps >= 5)
            k_pairs_split<5><<<sm_count() * bps, kBlock, 0, stream>>>(a, b.state[a.src], b.sorted32, b.sorted_orig,
                                                                     b.col_tab, b.items, b.items_cap,
                                                                     b.survivors, b.surv_cap);
        else if (bps == 4)
            k_pairs_split<4><<<sm_count() * bps, kBlock, 0, stream>>>(a, b.state[a.src], b.sorted32, b.sorted_orig,
                                                                     b.col_tab, b.items, b.items_cap,
                                                                     b.survivors, b.surv_cap);
        else
            k_pairs_split<3><<<sm_count() * bps, kBlock, 0, stream>>>(a, b.state[a.src], b.sorted32, b.sorted_orig,
                                                                     b.col_tab, b.items, b.items_cap,
                                                                     b.survivors, b.surv_cap);
        return;
    }
    const int bps = a.tune.pair_blocks_per_sm > 0 ? a.tune.pair_blocks_per_sm : (a.tune.pair_variant == 1 ? 3 : 2);
    if (a.tune.pair_variant == 1)
        k_pairs_tiles<1><<<sm_count() * bps, kBlock, 0, stream>>>(a, b.sorted, b.sorted_orig, b.cell_begin, b.nbr,
                                                                 b.items, b.items_cap, b.survivors, b.surv_cap);
    else
        k_pairs_tiles<2><<<sm_count() * bps, kBlock, 0, stream>>>(a, b.sorted, b.sorted_orig, b.cell_begin, b.nbr,
                                                                 b.items, b.items_cap, b.survivors, b.surv_cap);
}

void launch_refine(const DeviceBuffers& b, const StepArgs& a, ks_conjunction* conj_out, int64_t conj_cap,
                   ChunkCtrl* chunk, cudaStream_t stream) {
    k_refine_exact<<<sm_count() * 2, kBlock, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src], b.size_m,
                                                         b.survivors, b.surv_cap, conj_out, conj_cap, chunk);
}

cudaError_t measure_fp64(double* addmul_per_s, double* fma_per_s, cudaStream_t stream) {
    double* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(double));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm_count() * 8, threads = 256, iters = 4096;
    const double ops = static_cast<double>(blocks) * threads * iters * 8;
    float best_am = 1e30f, best_f = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        float ms = 0;
        cudaEventRecord(e0, stream);
        k_fp64_addmul<<<blocks, threads, 0, stream>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_am) best_am = ms;
        cudaEventRecord(e0, stream);
        k_fp64_fma<<<blocks, threads, 0, stream>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_f) best_f = ms;
    }
    e = cudaGetLastError();
    *addmul_per_s = 2.0 * ops / (best_am * 1e-3);  // one mul + one add per element-iteration
    *fma_per_s = ops / (best_f * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e;
}

cudaError_t measure_fp32(double* addmul_per_s, double* fma_per_s, cudaStream_t stream) {
    float* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(float));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm_count() * 8, threads = 256, iters = 8192;
    const double ops = static_cast<double>(blocks) * threads * iters * 8;
    float best_am = 1e30f, best_f = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        float ms = 0;
        cudaEventRecord(e0, stream);
        k_fp32_addmul<<<blocks, threads, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_am) best_am = ms;
        cudaEventRecord(e0, stream);
        k_fp32_fma<<<blocks, threads, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_f) best_f = ms;
    }
    e = cudaGetLastError();
    *addmul_per_s = 2.0 * ops / (best_am * 1e-3);
    *fma_per_s = ops / (best_f * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e;
}

cudaError_t measure_fp32x2(double* fma_ops_per_s, cudaStream_t stream) {
    float* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(float));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm_count() * 8, threads = 256, iters = 8192;
    const double ops = 2.0 * static_cast<double>(blocks) * threads * iters * 8;  // two lanes per FFMA2
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        float ms = 0;
        cudaEventRecord(e0, stream);
        k_fp32x2_fma<<<blocks, threads, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    e = cudaGetLastError();
    *fma_ops_per_s = ops / (best * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e;
}

}  // namespace ks
