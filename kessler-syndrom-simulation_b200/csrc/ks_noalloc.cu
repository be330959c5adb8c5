// Allocation-free one-shot screening: ks_screen_noalloc.
//
// Some callers cannot allocate GPU memory when they want to screen: an
// application that hands all device memory to its own pool up front, or a
// time-critical host loop that cannot afford cudaMalloc / cudaFree (they
// synchronise the device and stall every other stream). For them this entry
// point runs the same screening pipeline as ks_screen on device buffers carved
// from one fixed array that lives in the library's device image, so it calls
// no cudaMalloc, no cudaFree and no allocating library routine.
//
// Limits: at most kNoAllocMaxObjects objects per call and fixed capacities for
// pairs sent to refinement, work items and conjunctions; going beyond any of
// them is reported as an error, never as a partial result. Every GPU that
// loads the library holds the array until the process exits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "kessler_b200.h"
#include "ks_engine.h"
#include "ks_host.h"

namespace {

constexpr int64_t kNoAllocMaxObjects = 16384;
constexpr int64_t kNoAllocSurvivors = 1 << 17;
constexpr int64_t kNoAllocItems = 4 * kNoAllocMaxObjects;
constexpr int64_t kNoAllocConj = 1 << 15;
constexpr int64_t kNoAllocHash = 2 * kNoAllocMaxObjects;  // power of two >= 2 x objects
constexpr int kMaxDevices = 64;
constexpr int kMaxAttempts = 3;  // first run + replays with more radix passes

constexpr int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

// Byte size of every buffer, in carving order (see carve()).
constexpr int64_t scratch_bytes() {
    const int64_t n = kNoAllocMaxObjects;
    int64_t b = 0;
    b += 2 * align256(sizeof(double) * 6 * n);          // state[2]
    b += 2 * align256(n);                                // alive[2]
    b += align256(sizeof(double) * n);                   // size_m
    b += 2 * align256(sizeof(unsigned long long) * n);   // keys[2]
    b += 2 * align256(sizeof(int) * n);                  // idx[2]
    b += align256(sizeof(unsigned int) * 8 * 256);       // sort_hist
    b += align256(sizeof(unsigned int) * 8 * 256 * ((n + 2047) / 2048));  // sort_status
    b += align256(sizeof(unsigned int) * 8);             // sort_ctr
    b += align256(sizeof(int) * ((n + 1023) / 1024 + 1));                // block_counts
    b += align256(sizeof(int) * (n + 1));                // cell_begin
    b += align256(sizeof(unsigned long long) * n);       // cell_key
    b += align256(sizeof(int) * 13 * n);                 // nbr
    b += align256(sizeof(int) * n);                      // cell_len
    b += align256(sizeof(int2) * 16 * n);                // col_tab
    b += align256(sizeof(unsigned int) * 2 * ((n + 255) / 256 + 1));  // item_part
    b += align256(sizeof(int4) * kNoAllocItems);         // items
    b += align256(sizeof(unsigned long long) * kNoAllocHash);  // hash keys
    b += align256(sizeof(int) * kNoAllocHash);           // hash values
    b += align256(sizeof(double) * 6 * n);               // sorted
    b += align256(sizeof(float4) * 2 * n);               // sorted32
    b += align256(sizeof(float4) * 2 * n);               // rec32
    b += align256(sizeof(int) * n);                      // sorted_orig
    b += align256(sizeof(int2) * kNoAllocSurvivors);     // survivors
    b += align256(sizeof(ks_conjunction) * kNoAllocConj);  // conjunctions
    b += align256(sizeof(ks::Ctrl) * 3);                 // step, carry, carry checkpoint
    b += align256(sizeof(ks::ChunkCtrl));
    b += align256(sizeof(ks::StepParams));
    return b;
}

constexpr int64_t kScratchBytes = scratch_bytes();  // about 9.3 MB

// The scratch array. In host code this name is only a stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_screen_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Message of the current call, copied to the caller's buffer (if any) on return.
thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

template <typename T>
T* take(unsigned char*& p, int64_t bytes) {
    T* out = reinterpret_cast<T*>(p);
    p += align256(bytes);
    return out;
}

ks::DeviceBuffers carve(unsigned char* base) {
    const int64_t n = kNoAllocMaxObjects;
    ks::DeviceBuffers b;
    unsigned char* p = base;
    b.cap = n;
    for (int k = 0; k < 2; ++k) b.state[k] = take<double>(p, sizeof(double) * 6 * n);
    for (int k = 0; k < 2; ++k) b.alive[k] = take<uint8_t>(p, n);
    b.size_m = take<double>(p, sizeof(double) * n);
    for (int k = 0; k < 2; ++k) b.keys[k] = take<unsigned long long>(p, sizeof(unsigned long long) * n);
    for (int k = 0; k < 2; ++k) b.idx[k] = take<int>(p, sizeof(int) * n);
    b.sort_hist = take<unsigned int>(p, sizeof(unsigned int) * 8 * 256);
    b.sort_status_len = 8 * 256 * ((n + 2047) / 2048);
    b.sort_status = take<unsigned int>(p, sizeof(unsigned int) * b.sort_status_len);
    b.sort_ctr = take<unsigned int>(p, sizeof(unsigned int) * 8);
    b.block_counts = take<int>(p, sizeof(int) * ((n + 1023) / 1024 + 1));
    b.cell_begin = take<int>(p, sizeof(int) * (n + 1));
    b.cell_key = take<unsigned long long>(p, sizeof(unsigned long long) * n);
    b.nbr = take<int>(p, sizeof(int) * 13 * n);
    b.cell_len = take<int>(p, sizeof(int) * n);
    b.col_tab = take<int2>(p, sizeof(int2) * 16 * n);
    b.item_part = take<unsigned int>(p, sizeof(unsigned int) * 2 * ((n + 255) / 256 + 1));
    b.items = take<int4>(p, sizeof(int4) * kNoAllocItems);
    b.items_cap = kNoAllocItems;
    b.hash_keys = take<unsigned long long>(p, sizeof(unsigned long long) * kNoAllocHash);
    b.hash_vals = take<int>(p, sizeof(int) * kNoAllocHash);
    b.hash_cap = kNoAllocHash;
    b.sorted = take<double>(p, sizeof(double) * 6 * n);
    b.sorted32 = take<float4>(p, sizeof(float4) * 2 * n);
    b.rec32 = take<float4>(p, sizeof(float4) * 2 * n);
    b.sorted_orig = take<int>(p, sizeof(int) * n);
    b.survivors = take<int2>(p, sizeof(int2) * kNoAllocSurvivors);
    b.surv_cap = kNoAllocSurvivors;
    b.conj = take<ks_conjunction>(p, sizeof(ks_conjunction) * kNoAllocConj);
    b.conj_cap = kNoAllocConj;
    b.ctrl = take<ks::Ctrl>(p, sizeof(ks::Ctrl) * 3);
    b.ctrl_len = 3;
    b.chunk = take<ks::ChunkCtrl>(p, sizeof(ks::ChunkCtrl));
    b.params = take<ks::StepParams>(p, sizeof(ks::StepParams));
    return b;
}

// Device address of the scratch array on the current device, resolved once
// per device (the first call on each device does this set-up). The cached
// address belongs to the device's primary context: a cudaDeviceReset between
// calls would leave it stale, so the library does not support resetting a
// device it has screened on.
int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(KS_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(KS_ERR_RANGE, "device index beyond the scratch table");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_screen_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(KS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = ptr;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return KS_OK;
}

bool conj_less(const ks_conjunction& a, const ks_conjunction& b) {
    if (a.t != b.t) return a.t < b.t;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
}

#define NA_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(KS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

namespace {

int screen_noalloc(int64_t n, const double* before, const double* after, const uint8_t* alive_after,
                   const double* size_m, double t0, double dt, double threshold_km, double radius_scale,
                   double min_encounter_speed_km_s, ks_conjunction* out, int64_t cap, int64_t* count,
                   ks_step_stats* stats, void* stream) {
    if (n < 0 || !count || cap < 0 || (n > 0 && (!before || !after || !alive_after || !size_m)) || !(dt > 0.0) ||
        threshold_km < 0.0 || radius_scale < 0.0 || min_encounter_speed_km_s < 0.0)
        return fail(KS_ERR_ARG, "ks_screen_noalloc: bad arguments");
    *count = 0;
    if (n > kNoAllocMaxObjects)
        return fail(KS_ERR_RANGE, "ks_screen_noalloc: " + std::to_string(n) + " objects, at most " +
                                      std::to_string(kNoAllocMaxObjects) + " per call");
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ks::DeviceBuffers b = carve(base);

    if (n > 0) {
        NA_CUDA(cudaMemcpyAsync(b.state[0], before, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
        NA_CUDA(cudaMemcpyAsync(b.state[1], after, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
        NA_CUDA(cudaMemcpyAsync(b.alive[1], alive_after, n, cudaMemcpyHostToDevice, s));
        NA_CUDA(cudaMemcpyAsync(b.size_m, size_m, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    }
    ks::StepParams sp{};
    sp.t0 = t0;
    sp.step = 0;
    NA_CUDA(cudaMemcpyAsync(b.params, &sp, sizeof(sp), cudaMemcpyHostToDevice, s));

    ks::StepArgs a{};
    a.fc.neg_mu_earth = -ks::kMuEarth;
    a.fc.k_j2 = ks::j2_numerator();
    a.fc.mu_moon = ks::kMuMoon;
    a.fc.r_earth = ks::kREarth;
    a.dt = dt;
    a.threshold_km = threshold_km;
    a.vmin2 = min_encounter_speed_km_s * min_encounter_speed_km_s;
    a.radius_scale = radius_scale;
    a.n = static_cast<int>(n);
    a.screening = 1;
    a.sp = b.params;
    a.ctrl = b.ctrl;
    a.ctrl_next = b.ctrl + 1;
    a.src = 0;
    a.rec32 = b.rec32;

    // The array keeps the previous call's contents: the control blocks are
    // reset here, the sort and hash buffers by the launches that use them.
    ks::launch_chunk_init(b, 1, s);
    ks::launch_seed_ctrl(b, a.n, 0, a.ctrl, 0, s);
    ks::Ctrl c{};
    NA_CUDA(cudaMemcpyAsync(&c, a.ctrl, sizeof(ks::Ctrl), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    // Radix passes for the key width of this call (grid bits + the dead flag).
    {
        unsigned long long vb = c.spec_vmax;
        double vmax;
        std::memcpy(&vmax, &vb, sizeof(vmax));
        const double vrel = 2.0 * vmax;
        double cell = vrel * dt + threshold_km + ks::kGravityGradient * vrel * dt * dt * dt;
        if (cell < 1.0) cell = 1.0;
        int bits = 0;
        for (int ax = 0; ax < 3; ++ax) {
            auto dec = [](unsigned long long u) {
                unsigned long long v = (u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
                double d;
                std::memcpy(&d, &v, 8);
                return d;
            };
            const double mn = dec(c.bb_min[ax]), mx = dec(c.bb_max[ax]);
            if (!(mn <= mx)) continue;
            const long long span = static_cast<long long>(std::floor(mx / cell)) -
                                   static_cast<long long>(std::floor(mn / cell));
            int w = 0;
            while (w < 63 && (span >> w) > 0) ++w;
            bits += w;
        }
        a.sort_passes = std::max(1, (bits + 3 * a.tune.subcell_bits + 1 + 7) / 8);
    }
    for (int attempt = 0; attempt < kMaxAttempts; ++attempt) {
        if (attempt > 0) {
            ks::launch_chunk_init(b, 1, s);
            ks::launch_seed_ctrl(b, a.n, 0, a.ctrl, 0, s);
        }
        ks::launch_screen_keys(b, a, s);
        ks::launch_sort(b, a, s);
        ks::launch_cells(b, a, s);
        ks::launch_pairs(b, a, s);
        ks::launch_refine(b, a, b.conj, b.conj_cap, b.chunk, s);
        NA_CUDA(cudaGetLastError());
        ks::ChunkCtrl ch{};
        NA_CUDA(cudaMemcpyAsync(&c, a.ctrl, sizeof(ks::Ctrl), cudaMemcpyDeviceToHost, s));
        NA_CUDA(cudaMemcpyAsync(&ch, b.chunk, sizeof(ch), cudaMemcpyDeviceToHost, s));
        NA_CUDA(cudaStreamSynchronize(s));
        const int flags = c.flags | ch.flags;
        if (flags & ks::FLAG_KEY_RANGE) return fail(KS_ERR_RANGE, "ks_screen_noalloc: cell key outside its grid");
        if (flags & ks::FLAG_TIMEOUT) return fail(KS_ERR_TIMEOUT, "ks_screen_noalloc: radix sort wait gave up");
        if (flags & ks::FLAG_SORT_BITS) {
            // The keys needed more radix passes than launched: replay with
            // enough of them. Records of such a run are never returned.
            a.sort_passes = std::max(a.sort_passes, (c.grid.bits + 1 + 7) / 8);
            continue;
        }
        if (c.refined > static_cast<unsigned long long>(kNoAllocSurvivors))
            return fail(KS_ERR_OVERFLOW, "ks_screen_noalloc: " + std::to_string(c.refined) +
                                             " pairs to refine, fixed capacity " + std::to_string(kNoAllocSurvivors));
        if (ks::items_total(c) > kNoAllocItems)
            return fail(KS_ERR_OVERFLOW, "ks_screen_noalloc: pair work list beyond its fixed capacity");
        if ((flags & ks::FLAG_CONJ_OVERFLOW) || ch.conj_count > static_cast<unsigned long long>(kNoAllocConj)) {
            *count = static_cast<int64_t>(ch.conj_count);
            return fail(KS_ERR_OVERFLOW, "ks_screen_noalloc: more conjunctions than the fixed capacity " +
                                             std::to_string(kNoAllocConj));
        }
        const int64_t nc = static_cast<int64_t>(ch.conj_count);
        *count = nc;
        if (stats) {
            stats->step = 0;
            stats->candidate_pairs = static_cast<int64_t>(c.candidates);
            stats->refined_pairs = static_cast<int64_t>(c.refined);
            stats->co_orbiting = static_cast<int64_t>(c.co_orbiting);
            stats->conjunctions = static_cast<int64_t>(c.conj);
            stats->cell_km = c.grid.cell;
            stats->max_cell_objects = c.max_cell;
            stats->alive = c.n_alive;
        }
        if (nc > cap) return fail(KS_ERR_OVERFLOW, "ks_screen_noalloc: output holds " + std::to_string(cap) +
                                                       " records, " + std::to_string(nc) + " found");
        if (nc > 0) {
            if (!out) return fail(KS_ERR_ARG, "ks_screen_noalloc: null output buffer");
            NA_CUDA(cudaMemcpyAsync(out, b.conj, sizeof(ks_conjunction) * nc, cudaMemcpyDeviceToHost, s));
            NA_CUDA(cudaStreamSynchronize(s));
            std::sort(out, out + nc, conj_less);
        }
        return KS_OK;
    }
    return fail(KS_ERR_RANGE, "ks_screen_noalloc: cell keys still wider than the radix passes after " +
                                  std::to_string(kMaxAttempts) + " attempts");
}

}  // namespace

extern "C" int ks_screen_noalloc(int64_t n, const double* before, const double* after, const uint8_t* alive_after,
                                 const double* size_m, double t0, double dt, double threshold_km,
                                 double radius_scale, double min_encounter_speed_km_s, ks_conjunction* out,
                                 int64_t cap, int64_t* count, ks_step_stats* stats, void* stream, char* error,
                                 int64_t error_len) {
    g_error.clear();
    const int rc = screen_noalloc(n, before, after, alive_after, size_m, t0, dt, threshold_km, radius_scale,
                                  min_encounter_speed_km_s, out, cap, count, stats, stream);
    if (error && error_len > 0) {
        const size_t m = std::min(g_error.size(), static_cast<size_t>(error_len - 1));
        std::memcpy(error, g_error.data(), m);
        error[m] = '\0';
    }
    return rc;
}
