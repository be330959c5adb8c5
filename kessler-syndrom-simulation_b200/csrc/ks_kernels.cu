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
#include <cstdio>

#include "ks_engine.h"

namespace ks {

namespace {

constexpr int kBlock = 256;
constexpr unsigned long long kEmpty = ~0ull;
constexpr int kSortTile = 2048;            // keys per radix tile (256 threads x 8)
constexpr int kSortItems = kSortTile / kBlock;
constexpr int kWarps = kBlock / 32;
constexpr int kCellTile = 1024;            // sorted entries per cell-build tile

// Forward neighbour offsets (src/core/collision_filter.hpp:137-140): with the
// pairs inside a cell they visit every pair of neighbouring cells once.
__constant__ int c_forward[13][3] = {{1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0},
                                      {1, 0, 1},   {1, 1, -1}, {1, 1, 0},  {1, 1, 1},  {0, 1, -1},
                                      {0, 1, 0},   {0, 1, 1},  {0, 0, 1}};

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
                          double dt, double threshold_km, GridParams& g) {
    const double vrel = xmul(2.0, vmax);
    const double c = xadd(xadd(xmul(vrel, dt), threshold_km),
                          xmul(xmul(xmul(xmul(kGravityGradient, vrel), dt), dt), dt));
    g.cell = c > 1.0 ? c : 1.0;
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
    g.bits = bits;
}

// Compact key of a start-of-step position; sets *bad if outside the bounds.
__device__ __forceinline__ unsigned long long cell_key(const GridParams& g, double x, double y, double z,
                                                       int* bad) {
    const long long cx = static_cast<long long>(floor(xdiv(x, g.cell))) - g.lo[0];
    const long long cy = static_cast<long long>(floor(xdiv(y, g.cell))) - g.lo[1];
    const long long cz = static_cast<long long>(floor(xdiv(z, g.cell))) - g.lo[2];
    if (cx < 0 || cx > g.span[0] || cy < 0 || cy > g.span[1] || cz < 0 || cz > g.span[2]) *bad = 1;
    return (static_cast<unsigned long long>(cx) << (g.w[1] + g.w[2])) |
           (static_cast<unsigned long long>(cy) << g.w[2]) | static_cast<unsigned long long>(cz);
}

__device__ __forceinline__ unsigned long long dead_key(const GridParams& g) { return 1ull << g.bits; }

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

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Reduces per-thread speculation values over the block and applies them with
// one atomic per quantity per block.
struct SpecAccum {
    double vtrue, vnext;
    unsigned long long mn[3], mx[3];
    int alive;
    unsigned long long props;
    int bad;
    __device__ void init() {
        vtrue = 0.0; vnext = 0.0;
        for (int a = 0; a < 3; ++a) { mn[a] = kEmpty; mx[a] = 0ull; }
        alive = 0; props = 0; bad = 0;
    }
};

__device__ void flush_spec(SpecAccum& s, Ctrl* cur, Ctrl* next, bool screening) {
    __shared__ unsigned long long sh[kWarps][10];
    __shared__ int sh_alive[kWarps], sh_bad[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long vals[10];
    vals[0] = warp_max(static_cast<unsigned long long>(__double_as_longlong(s.vtrue)));
    vals[1] = warp_max(static_cast<unsigned long long>(__double_as_longlong(s.vnext)));
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
    if (threadIdx.x == 0) {
        for (int w = 1; w < kWarps; ++w) {
            vals[0] = max(vals[0], sh[w][0]);
            vals[1] = max(vals[1], sh[w][1]);
            for (int a = 0; a < 3; ++a) { vals[2 + a] = min(vals[2 + a], sh[w][2 + a]); vals[5 + a] = max(vals[5 + a], sh[w][5 + a]); }
            vals[8] += sh[w][8];
        }
        int alive = 0, bad = 0;
        for (int w = 0; w < kWarps; ++w) { alive += sh_alive[w]; bad |= sh_bad[w]; }
        atomicAdd(&cur->n_alive, alive);
        atomicAdd(&cur->object_steps, vals[8]);
        if (screening) {
            atomicMax(&cur->vmax_true, vals[0]);
            atomicMax(&next->spec_vmax, vals[1]);
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
    c.grid = GridParams{};
}

// ctrl[0..k) reset; ctrl[0] takes the carried speculation, the carry slot is reset.
__global__ void k_chunk_init(Ctrl* ctrl, int k_steps, Ctrl* carry, ChunkCtrl* chunk) {
    __shared__ Ctrl saved;
    if (threadIdx.x == 0) saved = *carry;
    __syncthreads();
    for (int s = threadIdx.x; s < k_steps; s += blockDim.x) ctrl_reset(ctrl[s]);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctrl[0].spec_vmax = saved.spec_vmax;
        for (int a = 0; a < 3; ++a) { ctrl[0].bb_min[a] = saved.bb_min[a]; ctrl[0].bb_max[a] = saved.bb_max[a]; }
        ctrl_reset(*carry);
        chunk->conj_count = 0ull;
        chunk->flags = 0;
    }
}

__global__ void k_ctrl_reset(Ctrl* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctrl_reset(*c);
}

// Speed and position bounds over alive objects of one state buffer.
__global__ void k_seed_ctrl(const double* __restrict__ st, int64_t stride, const uint8_t* __restrict__ alive,
                            int n, Ctrl* target) {
    SpecAccum s;
    s.init();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!alive[i]) continue;
        const double vx = st[3 * stride + i], vy = st[4 * stride + i], vz = st[5 * stride + i];
        s.vnext = fmax(s.vnext, xsqrt(xdot3(vx, vy, vz)));
        for (int a = 0; a < 3; ++a) {
            const unsigned long long e = enc_double(st[a * stride + i]);
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

__global__ void __launch_bounds__(kBlock) k_propagate_exact(StepArgs a, const double* __restrict__ in,
                                                            double* __restrict__ out,
                                                            const uint8_t* __restrict__ alive_in,
                                                            uint8_t* __restrict__ alive_out,
                                                            unsigned long long* __restrict__ keys,
                                                            int64_t stride) {
    __shared__ GridParams g;
    __shared__ MoonStage moon[3];
    if (threadIdx.x == 0) {
        if (a.screening)
            make_grid(__longlong_as_double(static_cast<long long>(a.ctrl->spec_vmax)), a.ctrl->bb_min,
                      a.ctrl->bb_max, a.dt, a.threshold_km, g);
        for (int q = 0; q < 3; ++q) moon[q] = a.sp->m[q];
        if (blockIdx.x == 0 && a.screening) a.ctrl->grid = g;
    }
    __syncthreads();
    const ForceConsts fc = a.fc;
    SpecAccum acc;
    acc.init();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double s[6];
        for (int q = 0; q < 6; ++q) s[q] = in[q * stride + i];
        if (!alive_in[i]) {
            for (int q = 0; q < 6; ++q) out[q * stride + i] = s[q];
            alive_out[i] = 0;
            if (a.screening) keys[i] = dead_key(g);
            continue;
        }
        acc.props += 1;
        unsigned long long key = 0ull;
        double vb = 0.0;
        if (a.screening) {
            key = cell_key(g, s[0], s[1], s[2], &acc.bad);
            vb = xsqrt(xdot3(s[3], s[4], s[5]));
        }
        rk4_exact(fc, a.dt, moon[0], moon[1], moon[2], s);
        for (int q = 0; q < 6; ++q) out[q * stride + i] = s[q];
        // Re-entry (src/core/orbital.cpp:297).
        const bool alive = !(xsqrt(xdot3(s[0], s[1], s[2])) < fc.r_earth);
        alive_out[i] = alive ? 1 : 0;
        if (alive) {
            acc.alive += 1;
            if (a.screening) {
                acc.vtrue = fmax(acc.vtrue, vb);
                acc.vnext = fmax(acc.vnext, xsqrt(xdot3(s[3], s[4], s[5])));
                for (int q = 0; q < 3; ++q) {
                    const unsigned long long e = enc_double(s[q]);
                    acc.mn[q] = min(acc.mn[q], e);
                    acc.mx[q] = max(acc.mx[q], e);
                }
            }
        }
        if (a.screening) keys[i] = alive ? key : dead_key(g);
    }
    flush_spec(acc, a.ctrl, a.ctrl_next, a.screening != 0);
}

// Keys for one-shot screening of given states: alive_after selects the objects,
// positions come from the start-of-step buffer. ctrl->spec_* already hold the
// bounds of exactly these objects, so the speculation is the true grid.
__global__ void __launch_bounds__(kBlock) k_screen_keys(StepArgs a, const double* __restrict__ before,
                                                        const uint8_t* __restrict__ alive_after,
                                                        unsigned long long* __restrict__ keys, int64_t stride) {
    __shared__ GridParams g;
    if (threadIdx.x == 0) {
        make_grid(__longlong_as_double(static_cast<long long>(a.ctrl->spec_vmax)), a.ctrl->bb_min,
                  a.ctrl->bb_max, a.dt, a.threshold_km, g);
        if (blockIdx.x == 0) {
            a.ctrl->grid = g;
            a.ctrl->vmax_true = a.ctrl->spec_vmax;
        }
    }
    __syncthreads();
    int bad = 0, alive = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        if (alive_after[i]) {
            keys[i] = cell_key(g, before[i], before[stride + i], before[2 * stride + i], &bad);
            ++alive;
        } else {
            keys[i] = dead_key(g);
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
                                                     unsigned long long* __restrict__ keys, int64_t stride) {
    const unsigned long long vt = a.ctrl->vmax_true;
    if (vt == a.ctrl->spec_vmax) return;
    __shared__ GridParams g;
    if (threadIdx.x == 0) {
        make_grid(__longlong_as_double(static_cast<long long>(vt)), a.ctrl->bb_min, a.ctrl->bb_max, a.dt,
                  a.threshold_km, g);
        if (blockIdx.x == 0) a.ctrl->grid = g;
    }
    __syncthreads();
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
        keys[i] = alive_after[i] ? cell_key(g, before[i], before[stride + i], before[2 * stride + i], &bad)
                                 : dead_key(g);
    bad = warp_max(bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(&a.ctrl->flags, FLAG_KEY_RANGE);
}

// ---------------------------------------------------------------------------
// Radix sort (LSD, 8-bit digits, stable)
// ---------------------------------------------------------------------------

// Per-tile digit counts, stored digit-major: hist[d * ntiles + tile].
__global__ void __launch_bounds__(kBlock) k_sort_hist(const unsigned long long* __restrict__ keys, int n,
                                                      int shift, unsigned int* __restrict__ hist, int ntiles,
                                                      Ctrl* ctrl, int check_bits) {
    __shared__ unsigned int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    for (int j = 0; j < kSortItems; ++j) {
        const int p = base + j * kBlock + threadIdx.x;
        const bool valid = p < n;
        const unsigned d = valid ? static_cast<unsigned>((keys[p] >> shift) & 0xFF) : 256u + (threadIdx.x & 31);
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[d], __popc(peers));
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
    if (check_bits && blockIdx.x == 0 && threadIdx.x == 0 && ctrl->grid.bits + 1 > check_bits)
        atomicOr(&ctrl->flags, FLAG_SORT_BITS);
}

// Exclusive scan of `len` counters in place, one block.
__global__ void __launch_bounds__(1024) k_scan_exclusive(unsigned int* __restrict__ v, int len) {
    __shared__ unsigned int warp_tot[32];
    const int per = (len + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    const int b1 = min(len, b0 + per);
    unsigned int sum = 0;
    for (int k = b0; k < b1; ++k) sum += v[k];
    // Block-wide exclusive scan of the per-thread sums.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned int t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    unsigned int run = incl - sum + (warp > 0 ? warp_tot[warp - 1] : 0);
    for (int k = b0; k < b1; ++k) {
        const unsigned int c = v[k];
        v[k] = run;
        run += c;
    }
}

// Stable scatter of one tile: ranks inside each warp with __match_any_sync,
// orders the tile by digit in shared memory, then writes runs of equal digits
// to consecutive global addresses.
__global__ void __launch_bounds__(kBlock) k_sort_scatter(const unsigned long long* __restrict__ keys_in,
                                                         const int* __restrict__ idx_in,
                                                         unsigned long long* __restrict__ keys_out,
                                                         int* __restrict__ idx_out, int n, int shift,
                                                         const unsigned int* __restrict__ hist, int ntiles) {
    __shared__ unsigned int wcnt[kWarps][256];
    __shared__ int gbase[256];
    __shared__ unsigned long long skeys[kSortTile];
    __shared__ int sidx[kSortTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile0 = blockIdx.x * kSortTile;
    const int count = min(kSortTile, n - tile0);
    for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();

    // Each warp owns kSortTile / kWarps consecutive keys, read 32 at a time.
    constexpr int kPerWarp = kSortTile / kWarps;
    constexpr int kRounds = kPerWarp / 32;
    unsigned long long k[kRounds];
    int id[kRounds];
    unsigned d[kRounds];
    for (int r = 0; r < kRounds; ++r) {
        const int l = warp * kPerWarp + r * 32 + lane;
        const int p = tile0 + l;
        const bool valid = l < count;
        k[r] = valid ? keys_in[p] : 0ull;
        id[r] = valid ? (idx_in ? idx_in[p] : p) : 0;
        d[r] = valid ? static_cast<unsigned>((k[r] >> shift) & 0xFF) : 256u + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, d[r]);
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        // Thread t owns digit t: tile total, then exclusive scan across digits.
        const int t = threadIdx.x;
        unsigned int tot = 0;
        for (int w = 0; w < kWarps; ++w) tot += wcnt[w][t];
        __shared__ unsigned int wsum[kWarps];
        unsigned int incl = tot;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        unsigned int off = 0;
        for (int w = 0; w < warp; ++w) off += wsum[w];
        const unsigned int start = off + incl - tot;
        gbase[t] = static_cast<int>(hist[t * ntiles + blockIdx.x]) - static_cast<int>(start);
        unsigned int run = start;
        for (int w = 0; w < kWarps; ++w) {
            const unsigned int c = wcnt[w][t];
            wcnt[w][t] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int r = 0; r < kRounds; ++r) {
        const bool valid = (warp * kPerWarp + r * 32 + lane) < count;
        const unsigned peers = __match_any_sync(0xffffffffu, d[r]);
        if (valid) {
            const unsigned pos = wcnt[warp][d[r]] + __popc(peers & lanemask_lt());
            skeys[pos] = k[r];
            sidx[pos] = id[r];
        }
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int l = threadIdx.x; l < count; l += kBlock) {
        const unsigned long long kk = skeys[l];
        const unsigned dd = static_cast<unsigned>((kk >> shift) & 0xFF);
        const int dst = gbase[dd] + l;
        keys_out[dst] = kk;
        idx_out[dst] = sidx[l];
    }
}

// ---------------------------------------------------------------------------
// Cells
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_cell_count(const unsigned long long* __restrict__ keys,
                                                       const Ctrl* __restrict__ ctrl, unsigned int* __restrict__ counts) {
    const int m = ctrl->n_alive;
    const int base = blockIdx.x * kCellTile;
    int c = 0;
    for (int j = threadIdx.x; j < kCellTile; j += kBlock) {
        const int p = base + j;
        if (p < m && (p == 0 || keys[p] != keys[p - 1])) ++c;
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
                                                       int* __restrict__ cell_of,
                                                       unsigned long long* __restrict__ hk, int* __restrict__ hv,
                                                       unsigned long long hmask, const double* __restrict__ before,
                                                       int64_t stride, double* __restrict__ sorted,
                                                       int* __restrict__ sorted_orig) {
    constexpr int kPer = kCellTile / kBlock;  // consecutive entries per thread
    const int m = ctrl->n_alive;
    if (m == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { ctrl->n_cells = 0; cell_begin[0] = 0; }
        return;
    }
    const int p0 = blockIdx.x * kCellTile + threadIdx.x * kPer;
    int heads[kPer];
    int local = 0;
    for (int j = 0; j < kPer; ++j) {
        const int p = p0 + j;
        heads[j] = (p < m && (p == 0 || keys[p] != keys[p - 1])) ? 1 : 0;
        local += heads[j];
    }
    // Block exclusive scan of `local`.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ int wsum[kWarps];
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int off = static_cast<int>(offsets[blockIdx.x]);
    for (int w = 0; w < warp; ++w) off += wsum[w];
    int run = off + incl - local;  // heads before this thread's first entry
    for (int j = 0; j < kPer; ++j) {
        const int p = p0 + j;
        if (p >= m) break;
        run += heads[j];
        const int cid = run - 1;
        const unsigned long long key = keys[p];
        if (heads[j]) {
            cell_begin[cid] = p;
            cell_key_out[cid] = key;
            unsigned long long h = hash_slot(key, hmask);
            for (unsigned long long probe = 0; probe <= hmask; ++probe) {
                const unsigned long long prev = atomicCAS(&hk[h], kEmpty, key);
                if (prev == kEmpty || prev == key) { hv[h] = cid; break; }
                h = (h + 1) & hmask;
            }
        }
        cell_of[p] = cid;
        const int o = idx[p];
        sorted_orig[p] = o;
        for (int q = 0; q < 6; ++q) sorted[6 * static_cast<int64_t>(p) + q] = before[q * stride + o];
        if (p == m - 1) {
            ctrl->n_cells = cid + 1;
            cell_begin[cid + 1] = m;
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_neighbours(Ctrl* ctrl, const int* __restrict__ cell_begin,
                                                       const unsigned long long* __restrict__ cell_key_in,
                                                       const unsigned long long* __restrict__ hk,
                                                       const int* __restrict__ hv, unsigned long long hmask,
                                                       int* __restrict__ nbr) {
    const int nc = ctrl->n_cells;
    const GridParams g = ctrl->grid;
    const unsigned long long mz = (1ull << g.w[2]) - 1, my = (1ull << g.w[1]) - 1;
    int biggest = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        biggest = max(biggest, cell_begin[c + 1] - cell_begin[c]);
        const unsigned long long key = cell_key_in[c];
        const long long cz = static_cast<long long>(key & mz);
        const long long cy = static_cast<long long>((key >> g.w[2]) & my);
        const long long cx = static_cast<long long>(key >> (g.w[1] + g.w[2]));
        for (int o = 0; o < 13; ++o) {
            const long long x = cx + c_forward[o][0], y = cy + c_forward[o][1], z = cz + c_forward[o][2];
            int found = -1;
            if (x >= 0 && x <= g.span[0] && y >= 0 && y <= g.span[1] && z >= 0 && z <= g.span[2]) {
                const unsigned long long nk = (static_cast<unsigned long long>(x) << (g.w[1] + g.w[2])) |
                                              (static_cast<unsigned long long>(y) << g.w[2]) |
                                              static_cast<unsigned long long>(z);
                found = hash_find(hk, hv, hmask, nk);
            }
            nbr[13 * static_cast<int64_t>(c) + o] = found;
        }
    }
    biggest = warp_max(biggest);
    if ((threadIdx.x & 31) == 0 && biggest > 0) atomicMax(&ctrl->max_cell, biggest);
}

// ---------------------------------------------------------------------------
// Pairs
// ---------------------------------------------------------------------------

struct SortedState {
    double rx, ry, rz, vx, vy, vz;
};

__device__ __forceinline__ SortedState load_sorted(const double* __restrict__ sorted, int p) {
    const double2* s = reinterpret_cast<const double2*>(sorted + 6 * static_cast<int64_t>(p));
    const double2 a = s[0], b = s[1], c = s[2];
    return SortedState{a.x, a.y, b.x, b.y, c.x, c.y};
}

__global__ void __launch_bounds__(kBlock) k_pairs_exact(StepArgs a, const double* __restrict__ sorted,
                                                        const int* __restrict__ orig,
                                                        const int* __restrict__ cell_of,
                                                        const int* __restrict__ cell_begin,
                                                        const int* __restrict__ nbr, int2* __restrict__ surv,
                                                        int64_t surv_cap) {
    const int m = a.ctrl->n_alive;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long cand = 0, co = 0, full = 0;
    if (p < m) {
        // Conservative distance gate bound: |dv| <= 2 * max speed.
        const double vmax = __longlong_as_double(static_cast<long long>(a.ctrl->vmax_true));
        const double dt3 = a.dt * a.dt * a.dt;
        const double gate_hi = (a.threshold_km + kGravityGradient * (2.0 * vmax) * dt3 + 1e-3) * (1.0 + 1e-9);
        const double gate_hi2 = gate_hi * gate_hi;
        const SortedState me = load_sorted(sorted, p);
        const int my_orig = orig[p];
        auto visit = [&](int q) {
            ++cand;
            const SortedState o = load_sorted(sorted, q);
            const double rx = xsub(o.rx, me.rx), ry = xsub(o.ry, me.ry), rz = xsub(o.rz, me.rz);
            const double vx = xsub(o.vx, me.vx), vy = xsub(o.vy, me.vy), vz = xsub(o.vz, me.vz);
            const double r2 = xdot3(rx, ry, rz);
            const double dv2 = xdot3(vx, vy, vz);
            const double rv = xadd(xadd(xmul(rx, vx), xmul(ry, vy)), xmul(rz, vz));
            if (certainly_far(r2, dv2, rv, gate_hi2)) return;
            ++full;
            const int res = filter_pair_exact(rx, ry, rz, vx, vy, vz, a.dt, a.threshold_km, a.vmin2);
            if (res == FILTER_CO_ORBITING) ++co;
            const bool keep = res == FILTER_REFINE;
            const unsigned act = __activemask();
            const unsigned bal = __ballot_sync(act, keep);
            if (bal) {
                const int leader = __ffs(bal) - 1;
                unsigned long long base = 0;
                if ((threadIdx.x & 31) == leader) base = atomicAdd(&a.ctrl->refined, static_cast<unsigned long long>(__popc(bal)));
                base = __shfl_sync(act, base, leader);
                if (keep) {
                    const unsigned long long pos = base + __popc(bal & lanemask_lt());
                    const int oq = orig[q];
                    if (pos < static_cast<unsigned long long>(surv_cap))
                        surv[pos] = make_int2(min(my_orig, oq), max(my_orig, oq));
                }
            }
        };
        const int c = cell_of[p];
        const int b = cell_begin[c];
        const int k = cell_begin[c + 1] - b;
        const int u = p - b;
        // Pairs inside the cell, balanced: object u meets the (k-1)/2 objects
        // after it (cyclically), plus the opposite one when k is even and u < k/2.
        const int half = (k - 1) / 2;
        for (int mm = 1; mm <= half; ++mm) {
            int q = u + mm;
            if (q >= k) q -= k;
            visit(b + q);
        }
        if ((k & 1) == 0 && u < k / 2) visit(b + u + k / 2);
        for (int o = 0; o < 13; ++o) {
            const int nc = nbr[13 * static_cast<int64_t>(c) + o];
            if (nc < 0) continue;
            const int q1 = cell_begin[nc + 1];
            for (int q = cell_begin[nc]; q < q1; ++q) visit(q);
        }
    }
    cand = warp_sum(cand);
    co = warp_sum(co);
    full = warp_sum(full);
    if ((threadIdx.x & 31) == 0) {
        if (cand) atomicAdd(&a.ctrl->candidates, cand);
        if (co) atomicAdd(&a.ctrl->co_orbiting, co);
        if (full) atomicAdd(&a.ctrl->exact_evals, full);
    }
}

// ---------------------------------------------------------------------------
// Refinement
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_refine_exact(StepArgs a, const double* __restrict__ before,
                                                         const double* __restrict__ after, int64_t stride,
                                                         const double* __restrict__ size_m,
                                                         const int2* __restrict__ surv, int64_t surv_cap,
                                                         ks_conjunction* __restrict__ out, int64_t cap,
                                                         ChunkCtrl* chunk) {
    const unsigned long long ns = min(a.ctrl->refined, static_cast<unsigned long long>(surv_cap));
    const double t0 = a.sp->t0;
    const double s_hi = xsub(1.0, 1e-9);
    for (unsigned long long w = blockIdx.x * blockDim.x + threadIdx.x; w < ns; w += gridDim.x * blockDim.x) {
        const int i = surv[w].x, j = surv[w].y;
        Hermite h;
        for (int q = 0; q < 3; ++q) {
            h.p0[q] = xsub(before[q * stride + j], before[q * stride + i]);
            h.m0[q] = xmul(xsub(before[(3 + q) * stride + j], before[(3 + q) * stride + i]), a.dt);
            h.p1[q] = xsub(after[q * stride + j], after[q * stride + i]);
            h.m1[q] = xmul(xsub(after[(3 + q) * stride + j], after[(3 + q) * stride + i]), a.dt);
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
        c.reserved = 0;
        atomicAdd(&a.ctrl->conj, 1ull);
        const unsigned long long slot = atomicAdd(&chunk->conj_count, 1ull);
        if (slot < static_cast<unsigned long long>(cap)) out[slot] = c;
        else atomicOr(&chunk->flags, FLAG_CONJ_OVERFLOW);
    }
}

// ---------------------------------------------------------------------------
// Layout conversion
// ---------------------------------------------------------------------------

__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t n, int64_t stride) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < 6 * n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = e / 6, q = e % 6;
        soa[q * stride + i] = aos[e];
    }
}

__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t n, int64_t stride) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < 6 * n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = e / 6, q = e % 6;
        aos[e] = soa[q * stride + i];
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

int g_sm_count = 0;

int grid_for(int64_t n, int per_sm_blocks) {
    const int sms = sm_count();
    const int64_t want = (n + kBlock - 1) / kBlock;
    const int64_t cap = static_cast<int64_t>(sms) * per_sm_blocks;
    return static_cast<int>(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

int sm_count() {
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 1;
    }
    return g_sm_count;
}

void launch_chunk_init(const DeviceBuffers& b, int k_steps, cudaStream_t stream) {
    k_chunk_init<<<1, kBlock, 0, stream>>>(b.ctrl, k_steps, b.ctrl + b.ctrl_len - 2, b.chunk);
}

void launch_seed_ctrl(const DeviceBuffers& b, int n, int src, Ctrl* target, int use_alive_src, cudaStream_t stream) {
    k_ctrl_reset<<<1, 32, 0, stream>>>(target);
    k_seed_ctrl<<<grid_for(n, 4), kBlock, 0, stream>>>(b.state[src], b.cap,
                                                        use_alive_src ? b.alive[src] : b.alive[1 - src], n, target);
}

void launch_propagate(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_propagate_exact<<<grid_for(a.n, 4), kBlock, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src],
                                                                b.alive[a.src], b.alive[1 - a.src], b.keys[0], b.cap);
}

void launch_screen_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_screen_keys<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a, b.state[a.src], b.alive[1 - a.src], b.keys[0], b.cap);
}

void launch_fix_keys(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    k_fix_keys<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a, b.state[a.src], b.alive[1 - a.src], b.keys[0], b.cap);
}

void launch_sort(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int n = a.n;
    if (n <= 0) return;  // nothing alive: the cell build sees n_alive == 0
    const int ntiles = (n + kSortTile - 1) / kSortTile;
    for (int pass = 0; pass < a.sort_passes; ++pass) {
        const int in = pass & 1, outb = 1 - in;
        const int shift = 8 * pass;
        k_sort_hist<<<ntiles, kBlock, 0, stream>>>(b.keys[in], n, shift, b.tile_hist, ntiles, a.ctrl,
                                                  pass == 0 ? 8 * a.sort_passes : 0);
        k_scan_exclusive<<<1, 1024, 0, stream>>>(b.tile_hist, 256 * ntiles);
        k_sort_scatter<<<ntiles, kBlock, 0, stream>>>(b.keys[in], pass == 0 ? nullptr : b.idx[in], b.keys[outb],
                                                     b.idx[outb], n, shift, b.tile_hist, ntiles);
    }
}

void launch_cells(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int sb = sorted_buffer(a.sort_passes);
    const int ntiles = a.n > 0 ? (a.n + kCellTile - 1) / kCellTile : 1;
    k_cell_count<<<ntiles, kBlock, 0, stream>>>(b.keys[sb], a.ctrl, reinterpret_cast<unsigned int*>(b.block_counts));
    k_scan_exclusive<<<1, 1024, 0, stream>>>(reinterpret_cast<unsigned int*>(b.block_counts), ntiles);
    cudaMemsetAsync(b.hash_keys, 0xFF, sizeof(unsigned long long) * b.hash_cap, stream);
    k_cell_write<<<ntiles, kBlock, 0, stream>>>(b.keys[sb], b.idx[sb], reinterpret_cast<const unsigned int*>(b.block_counts),
                                               a.ctrl, b.cell_begin, b.cell_key, b.cell_of, b.hash_keys, b.hash_vals,
                                               static_cast<unsigned long long>(b.hash_cap - 1), b.state[a.src], b.cap,
                                               b.sorted, b.sorted_orig);
    k_neighbours<<<grid_for(a.n, 8), kBlock, 0, stream>>>(a.ctrl, b.cell_begin, b.cell_key, b.hash_keys, b.hash_vals,
                                                          static_cast<unsigned long long>(b.hash_cap - 1), b.nbr);
}

void launch_pairs(const DeviceBuffers& b, const StepArgs& a, cudaStream_t stream) {
    const int blocks = (a.n + kBlock - 1) / kBlock;
    k_pairs_exact<<<blocks > 0 ? blocks : 1, kBlock, 0, stream>>>(a, b.sorted, b.sorted_orig, b.cell_of, b.cell_begin,
                                                                  b.nbr, b.survivors, b.surv_cap);
}

void launch_refine(const DeviceBuffers& b, const StepArgs& a, ks_conjunction* conj_out, int64_t conj_cap,
                   ChunkCtrl* chunk, cudaStream_t stream) {
    k_refine_exact<<<sm_count() * 2, kBlock, 0, stream>>>(a, b.state[a.src], b.state[1 - a.src], b.cap, b.size_m,
                                                         b.survivors, b.surv_cap, conj_out, conj_cap, chunk);
}

void launch_aos_to_soa(const double* aos, double* soa, int64_t n, int64_t stride, cudaStream_t stream) {
    if (n <= 0) return;
    k_aos_to_soa<<<grid_for(6 * n, 8), kBlock, 0, stream>>>(aos, soa, n, stride);
}

void launch_soa_to_aos(const double* soa, double* aos, int64_t n, int64_t stride, cudaStream_t stream) {
    if (n <= 0) return;
    k_soa_to_aos<<<grid_for(6 * n, 8), kBlock, 0, stream>>>(soa, aos, n, stride);
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

}  // namespace ks
