// C++ drop-in layer over the C ABI (include/kessler_b200.h).
//
// Mirrors the reference's hot-path interface (src/core/orbital.hpp,
// src/core/collision.hpp) so its call sites can switch with a few lines:
//
//   Reference                                   This header
//   -------------------------------------------------------------------------
//   Simulation::step() over std::vector<Object> kessler_b200::step_objects(...)
//   Screener::screen / screen_step              kessler_b200::Screener::screen(...)
//   Screener::set_gpu / gpu / gpu_compiled      kessler_b200::Screener::set_gpu(...)
//   CLI loop begin / step / finish (main.cpp)   kessler_b200::DeviceSimulation
//
// The template functions take the reference's own types by member name
// (State{r{x,y,z}, v{x,y,z}}, Object{s, alive, size_m}, Conjunction{i, j, t,
// miss_km, v_rel_km_s, collision}); nothing here includes the reference's
// headers. DeviceSimulation keeps the population on the GPU between steps,
// which is where the speed comes from; the host-buffer calls copy states in
// and out on every call, like the reference's own GPU backend did.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "kessler_b200.h"

namespace kessler_b200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code(code) {}
    int code;
};

inline void check(ks_ctx* ctx, int rc, const char* where) {
    if (rc != KS_OK) throw Error(rc, std::string(where) + ": " + ks_last_error(ctx));
}

// ScreeningConfig (src/core/collision.hpp:26-37).
struct ScreeningConfig {
    double threshold_km = 5.0;
    double radius_scale = 1.0;
    double min_encounter_speed_km_s = 0.01;
};

// Owning handle of one device context.
class Context {
public:
    explicit Context(int device = 0) {
        const int rc = ks_create(device, &ctx_);
        if (rc != KS_OK) throw Error(rc, "ks_create failed (no usable CUDA device?)");
    }
    ~Context() { ks_destroy(ctx_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ks_ctx* get() const { return ctx_; }
    std::string device_name() const { return ks_device_name(ctx_); }

private:
    ks_ctx* ctx_ = nullptr;
};

namespace detail {

template <class StateT>
void pack_state(const StateT& s, double* out) {
    out[0] = s.r.x; out[1] = s.r.y; out[2] = s.r.z;
    out[3] = s.v.x; out[4] = s.v.y; out[5] = s.v.z;
}

template <class StateT>
void unpack_state(const double* in, StateT& s) {
    s.r.x = in[0]; s.r.y = in[1]; s.r.z = in[2];
    s.v.x = in[3]; s.v.y = in[4]; s.v.z = in[5];
}

template <class ConjT>
ConjT to_conjunction(const ks_conjunction& c) {
    ConjT out{};
    out.i = c.i;
    out.j = c.j;
    out.t = c.t;
    out.miss_km = c.miss_km;
    out.v_rel_km_s = c.v_rel_km_s;
    out.collision = c.collision != 0;
    return out;
}

}  // namespace detail

// Screener (src/core/collision.hpp:75-120): one-shot screening of a step
// from host states, on the GPU. No CPU fallback: set_gpu(true) fails when no
// device is usable, and screen() throws.
class Screener {
public:
    explicit Screener(const ScreeningConfig& cfg = {}) : cfg_(cfg) {}
    ScreeningConfig& config() { return cfg_; }
    const ScreeningConfig& config() const { return cfg_; }

    static bool gpu_compiled() { return true; }

    bool set_gpu(bool on, std::string* message = nullptr) {
        if (!on) {
            ctx_.reset();
            return true;
        }
        if (ctx_) return true;
        try {
            ctx_.reset(new Context(0));
            if (message) *message = ctx_->device_name();
            return true;
        } catch (const Error& e) {
            if (message) *message = e.what();
            return false;
        }
    }
    bool gpu() const { return ctx_ != nullptr; }

    // Screener::screen(before, after, t0, dt, stats): conjunctions of the step
    // [t0, t0 + dt] ordered by (t, i, j). ObjectT needs members s, alive, size_m.
    template <class ConjT, class StateT, class ObjectT>
    std::vector<ConjT> screen(const std::vector<StateT>& before, const std::vector<ObjectT>& after, double t0,
                              double dt, ks_step_stats* stats = nullptr) {
        if (!ctx_ && !set_gpu(true)) throw Error(KS_ERR_NO_DEVICE, "no usable CUDA device");
        const size_t n = before.size();
        if (after.size() != n) throw Error(KS_ERR_ARG, "before/after sizes differ");
        b_.resize(6 * n);
        a_.resize(6 * n);
        alive_.resize(n);
        size_.resize(n);
        for (size_t i = 0; i < n; ++i) {
            detail::pack_state(before[i], &b_[6 * i]);
            detail::pack_state(after[i].s, &a_[6 * i]);
            alive_[i] = after[i].alive ? 1 : 0;
            size_[i] = after[i].size_m;
        }
        ks_ctx* c = ctx_->get();
        check(c, ks_set_screening(c, 1, cfg_.threshold_km, cfg_.radius_scale, cfg_.min_encounter_speed_km_s),
              "ks_set_screening");
        int64_t count = 0;
        out_.resize(1024);
        for (;;) {
            check(c, ks_screen(c, static_cast<int64_t>(n), b_.data(), a_.data(), alive_.data(), size_.data(), t0, dt,
                               out_.data(), static_cast<int64_t>(out_.size()), &count, stats),
                  "ks_screen");
            if (count <= static_cast<int64_t>(out_.size())) break;
            out_.resize(static_cast<size_t>(count));
        }
        std::vector<ConjT> res;
        res.reserve(static_cast<size_t>(count));
        for (int64_t k = 0; k < count; ++k) res.push_back(detail::to_conjunction<ConjT>(out_[k]));
        return res;
    }

private:
    ScreeningConfig cfg_;
    std::unique_ptr<Context> ctx_;
    std::vector<double> b_, a_, size_;
    std::vector<uint8_t> alive_;
    std::vector<ks_conjunction> out_;
};

// Simulation::step over host objects (src/core/orbital.cpp:286-300): `steps`
// steps of every alive object starting at time t, states and alive flags
// updated in place. Returns the new time (t advanced by repeated addition of
// dt, as Simulation::step does, src/core/orbital.cpp:299).
template <class ObjectT>
double step_objects(Context& ctx, std::vector<ObjectT>& objects, double epoch_jd, double t, double dt,
                    long steps = 1) {
    const size_t n = objects.size();
    std::vector<double> st(6 * n);
    std::vector<uint8_t> alive(n);
    for (size_t i = 0; i < n; ++i) {
        detail::pack_state(objects[i].s, &st[6 * i]);
        alive[i] = objects[i].alive ? 1 : 0;
    }
    check(ctx.get(), ks_propagate(ctx.get(), static_cast<int64_t>(n), st.data(), alive.data(), epoch_jd, t, dt, steps),
          "ks_propagate");
    for (size_t i = 0; i < n; ++i) {
        detail::unpack_state(&st[6 * i], objects[i].s);
        objects[i].alive = alive[i] != 0;
    }
    for (long k = 0; k < steps; ++k) t += dt;
    return t;
}

// The CLI step loop with the population resident on the GPU: each step is
// Screener::begin + Simulation::step + Screener::finish (src/main.cpp:352-373).
class DeviceSimulation {
public:
    explicit DeviceSimulation(int device = 0) : ctx_(device) {}

    Context& context() { return ctx_; }

    // states: n x 6 doubles {rx, ry, rz, vx, vy, vz}; size_m: characteristic sizes (m).
    void set_population(const std::vector<double>& states, const std::vector<double>& size_m,
                        const std::vector<uint8_t>& alive = {}) {
        const int64_t n = static_cast<int64_t>(size_m.size());
        if (static_cast<int64_t>(states.size()) != 6 * n) throw Error(KS_ERR_ARG, "states must hold 6 doubles per object");
        check(ctx_.get(), ks_set_population(ctx_.get(), n, states.data(), size_m.data(),
                                            alive.empty() ? nullptr : alive.data()),
              "ks_set_population");
    }
    void set_clock(double epoch_jd, double t, double dt) {
        check(ctx_.get(), ks_set_clock(ctx_.get(), epoch_jd, t, dt), "ks_set_clock");
    }
    void set_screening(bool enabled, const ScreeningConfig& cfg = {}) {
        check(ctx_.get(), ks_set_screening(ctx_.get(), enabled ? 1 : 0, cfg.threshold_km, cfg.radius_scale,
                                           cfg.min_encounter_speed_km_s),
              "ks_set_screening");
    }
    void set_precision(int precision) { check(ctx_.get(), ks_set_precision(ctx_.get(), precision), "ks_set_precision"); }
    void set_steps_per_graph(int k) { check(ctx_.get(), ks_set_steps_per_graph(ctx_.get(), k), "ks_set_steps_per_graph"); }

    // Simulation::advance(n) with screening of every step.
    void advance(long steps) { check(ctx_.get(), ks_run(ctx_.get(), steps), "ks_run"); }

    std::vector<ks_conjunction> take_conjunctions() {
        int64_t n = 0;
        check(ctx_.get(), ks_take_conjunctions(ctx_.get(), nullptr, 0, &n), "ks_take_conjunctions");
        std::vector<ks_conjunction> out(static_cast<size_t>(n));
        if (n) check(ctx_.get(), ks_take_conjunctions(ctx_.get(), out.data(), n, &n), "ks_take_conjunctions");
        out.resize(static_cast<size_t>(n));
        return out;
    }
    // The same records without a copy: f(const ks_conjunction&) is called on
    // each, in (t, i, j) order, where the engine holds them (ks_take_conjunctions_view).
    template <typename F>
    void for_each_conjunction(F&& f) {
        for (;;) {
            const ks_conjunction* first = nullptr;
            int64_t n = 0;
            check(ctx_.get(), ks_take_conjunctions_view(ctx_.get(), &first, &n), "ks_take_conjunctions_view");
            if (n <= 0) return;
            for (int64_t q = 0; q < n; ++q) f(first[q]);
        }
    }
    std::vector<ks_step_stats> take_step_stats() {
        int64_t n = 0;
        check(ctx_.get(), ks_take_step_stats(ctx_.get(), nullptr, 0, &n), "ks_take_step_stats");
        std::vector<ks_step_stats> out(static_cast<size_t>(n));
        if (n) check(ctx_.get(), ks_take_step_stats(ctx_.get(), out.data(), n, &n), "ks_take_step_stats");
        out.resize(static_cast<size_t>(n));
        return out;
    }
    void get_population(std::vector<double>& states, std::vector<uint8_t>& alive) {
        const int64_t n = ks_population_size(ctx_.get());
        states.resize(static_cast<size_t>(6 * n));
        alive.resize(static_cast<size_t>(n));
        check(ctx_.get(), ks_get_population(ctx_.get(), n, states.data(), alive.data()), "ks_get_population");
    }
    double time() const {
        double t = 0;
        int64_t k = 0;
        ks_get_clock(ctx_.get(), &t, &k);
        return t;
    }
    int64_t size() const { return ks_population_size(ctx_.get()); }

    // Fragmentation (BreakupConfig / Fragmentation, src/core/breakup.hpp:75-153).
    void set_breakup(bool on, double lc_m = 0.10, double catastrophic_j_per_g = 40.0, uint64_t seed = 1) {
        check(ctx_.get(), ks_set_breakup(ctx_.get(), on ? 1 : 0, lc_m, catastrophic_j_per_g, seed), "ks_set_breakup");
    }
    void set_masses(const std::vector<double>& mass_kg) {
        check(ctx_.get(), ks_set_masses(ctx_.get(), static_cast<int64_t>(mass_kg.size()), mass_kg.data()),
              "ks_set_masses");
    }
    void impact(int64_t target, double projectile_mass_kg, double v_rel_km_s) {
        check(ctx_.get(), ks_impact(ctx_.get(), target, projectile_mass_kg, v_rel_km_s), "ks_impact");
    }
    std::vector<ks_breakup_event> take_breakups() {
        int64_t n = 0;
        check(ctx_.get(), ks_take_breakups(ctx_.get(), nullptr, 0, &n), "ks_take_breakups");
        std::vector<ks_breakup_event> out(static_cast<size_t>(n));
        if (n) check(ctx_.get(), ks_take_breakups(ctx_.get(), out.data(), n, &n), "ks_take_breakups");
        out.resize(static_cast<size_t>(n));
        return out;
    }
    // Per-object originating event (-1 for the initial population).
    std::vector<int32_t> events_of_objects() {
        const int64_t n = size();
        std::vector<int32_t> ev(static_cast<size_t>(n));
        check(ctx_.get(), ks_get_objects(ctx_.get(), n, nullptr, nullptr, nullptr, ev.data(), nullptr), "ks_get_objects");
        return ev;
    }

private:
    Context ctx_;
};

}  // namespace kessler_b200
