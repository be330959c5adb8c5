"""B200 engine for the per-step hot path of Kessler_Sim.

Python view of the C ABI (include/kessler_b200.h), used by the tests and the
benchmark. The reference-facing C++ drop-in lives in host/kessler_b200.hpp.

    eng = Engine(device=0)
    eng.set_population(states, size_m)          # Simulation::objects
    eng.set_clock(epoch_jd, 0.0, 10.0)          # Simulation::{epoch_jd, t, dt}
    eng.set_screening(True, 5.0, 1.0, 0.01)     # ScreeningConfig
    eng.run(360)                                # 360 x (begin / step / finish)
    conj = eng.take_conjunctions()              # sorted by (t, i, j)
"""
import ctypes as C
import os

import numpy as np

from ._abi import (BREAKUP_DTYPE, CONJ_DTYPE, PRECISION_FP64, PRECISION_SPLIT, STATS_DTYPE, STATUS_NAMES, Timing,
                   TuningChoice, load_library, ptr)

__all__ = ["Engine", "KsError", "BREAKUP_DTYPE", "CONJ_DTYPE", "STATS_DTYPE", "PRECISION_FP64", "PRECISION_SPLIT",
           "moon_position", "generate_population", "sbm_impact", "load_library", "DEFAULT_EPOCH_JD"]

# src/core/orbital.hpp:30
DEFAULT_EPOCH_JD = 2461253.916666667
BREAKUP_HOST, BREAKUP_DEVICE = 0, 1


class KsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def _states(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 6:
        raise ValueError("states must have shape (n, 6): rx, ry, rz, vx, vy, vz")
    if n is not None and a.shape[0] != n:
        raise ValueError("states row count mismatch")
    return a


class Engine:
    """One device context: stream, device-resident population, clock, screening."""

    def __init__(self, device=0):
        self._lib = load_library()
        h = C.c_void_p()
        rc = self._lib.ks_create(int(device), C.byref(h))
        if rc != 0:
            raise KsError(rc, f"ks_create(device={device}) failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ks_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise KsError(rc, self._lib.ks_last_error(self._h).decode(errors="replace"))

    @property
    def device_name(self):
        return self._lib.ks_device_name(self._h).decode()

    @property
    def stream(self):
        """cudaStream_t of the context (int), e.g. for torch.cuda.ExternalStream."""
        return self._lib.ks_stream(self._h) or 0

    # --- population / clock / configuration ---
    def set_population(self, states, size_m, alive=None):
        st = _states(states)
        n = st.shape[0]
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        if sz.shape != (n,):
            raise ValueError("size_m must have shape (n,)")
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        if al is not None and al.shape != (n,):
            raise ValueError("alive must have shape (n,)")
        self._check(self._lib.ks_set_population(self._h, n, ptr(st), ptr(sz), ptr(al)))

    def set_population_batch(self, offsets, states, size_m, alive=None):
        """Independent realisations: realisation r owns rows offsets[r]:offsets[r+1]."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        st = _states(states, int(off[-1]))
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        self._check(self._lib.ks_set_population_batch(self._h, len(off) - 1, ptr(off), ptr(st), ptr(sz), ptr(al)))

    def population_size(self):
        return int(self._lib.ks_population_size(self._h))

    def get_population(self, states=None, alive=None):
        """(states (n, 6), alive (n,)); optional preallocated outputs (e.g. pinned host memory)."""
        n = self._lib.ks_population_size(self._h)
        st = np.empty((n, 6), dtype=np.float64) if states is None else states
        al = np.empty(n, dtype=np.uint8) if alive is None else alive
        if st.shape != (n, 6) or st.dtype != np.float64 or not st.flags.c_contiguous:
            raise ValueError("states must be a C-contiguous float64 array of shape (n, 6)")
        if al.shape != (n,) or al.dtype != np.uint8:
            raise ValueError("alive must be a uint8 array of shape (n,)")
        self._check(self._lib.ks_get_population(self._h, n, ptr(st), ptr(al)))
        return st, al

    def set_clock(self, epoch_jd=DEFAULT_EPOCH_JD, t=0.0, dt=10.0):
        self._check(self._lib.ks_set_clock(self._h, float(epoch_jd), float(t), float(dt)))

    def clock(self):
        t = C.c_double()
        k = C.c_int64()
        self._check(self._lib.ks_get_clock(self._h, C.byref(t), C.byref(k)))
        return t.value, k.value

    def set_screening(self, enabled=True, threshold_km=5.0, radius_scale=1.0, min_encounter_speed_km_s=0.01):
        self._check(self._lib.ks_set_screening(self._h, 1 if enabled else 0, float(threshold_km),
                                               float(radius_scale), float(min_encounter_speed_km_s)))

    def set_precision(self, precision):
        self._check(self._lib.ks_set_precision(self._h, int(precision)))

    def set_steps_per_graph(self, k):
        self._check(self._lib.ks_set_steps_per_graph(self._h, int(k)))

    def set_buffer_limits(self, survivor_pairs=0, conjunctions=0):
        self._check(self._lib.ks_set_buffer_limits(self._h, int(survivor_pairs), int(conjunctions)))

    def set_tuning(self, key, value):
        self._check(self._lib.ks_set_tuning(self._h, key.encode(), int(value)))

    def set_l2_flush(self, nbytes):
        self._check(self._lib.ks_set_l2_flush(self._h, int(nbytes)))

    def set_profiling(self, on):
        self._check(self._lib.ks_set_profiling(self._h, 1 if on else 0))

    # --- stepping ---
    def run(self, steps):
        self._check(self._lib.ks_run(self._h, int(steps)))

    def prepare_run(self):
        """Capture the chunk graphs the next run() calls launch, without running."""
        self._check(self._lib.ks_prepare_run(self._h))

    def take_conjunctions(self, out=None):
        """Records found since the last take, in (t, i, j) order. With `out` (a
        contiguous CONJ_DTYPE array, e.g. in pinned memory, reused from call to
        call) up to len(out) records are moved into it and out[:count] is
        returned; the rest stay for the next take."""
        cnt = C.c_int64()
        if out is not None:
            if out.dtype != CONJ_DTYPE or not out.flags["C_CONTIGUOUS"]:
                raise ValueError("out must be a contiguous CONJ_DTYPE array")
            self._check(self._lib.ks_take_conjunctions(self._h, ptr(out), len(out), C.byref(cnt)))
            return out[: cnt.value]
        self._check(self._lib.ks_take_conjunctions(self._h, None, 0, C.byref(cnt)))
        res = np.empty(cnt.value, dtype=CONJ_DTYPE)  # every record is written below
        if cnt.value:
            self._check(self._lib.ks_take_conjunctions(self._h, ptr(res), cnt.value, C.byref(cnt)))
        return res[: cnt.value]

    def take_conjunctions_view(self):
        """Zero-copy take: the oldest records not yet taken, as a CONJ_DTYPE array
        over the engine's own host memory (no copy), in (t, i, j) order; call
        until it returns an empty array. The array is valid only until the
        next run, population change or take on this engine: copy what must
        outlive that."""
        first = C.c_void_p()
        cnt = C.c_int64()
        self._check(self._lib.ks_take_conjunctions_view(self._h, C.byref(first), C.byref(cnt)))
        if cnt.value == 0 or not first.value:
            return np.empty(0, dtype=CONJ_DTYPE)
        buf = (C.c_char * (cnt.value * CONJ_DTYPE.itemsize)).from_address(first.value)
        return np.frombuffer(buf, dtype=CONJ_DTYPE, count=cnt.value)

    def take_step_stats(self):
        cnt = C.c_int64()
        self._check(self._lib.ks_take_step_stats(self._h, None, 0, C.byref(cnt)))
        out = np.empty(cnt.value, dtype=STATS_DTYPE)  # every row is written below
        if cnt.value:
            self._check(self._lib.ks_take_step_stats(self._h, ptr(out), cnt.value, C.byref(cnt)))
        return out[: cnt.value]

    def autotune(self, trial_steps=16):
        """Times candidate launch configurations on the resident population and keeps the fastest.

        The simulation is left exactly where it was; returns the chosen configuration."""
        ch = TuningChoice()
        self._check(self._lib.ks_autotune(self._h, int(trial_steps), C.byref(ch)))
        return {name: getattr(ch, name) for name, _ in TuningChoice._fields_}

    # --- fragmentation (NASA SBM) ---
    def set_breakup(self, on=True, lc_m=0.10, catastrophic_j_per_g=40.0, seed=1):
        self._check(self._lib.ks_set_breakup(self._h, 1 if on else 0, float(lc_m), float(catastrophic_j_per_g),
                                             int(seed)))

    def set_breakup_mode(self, mode, max_objects=0):
        """BREAKUP_HOST (the reference's draws, on the host) or BREAKUP_DEVICE
        (the SBM inside every step on the device, population budget max_objects).
        Call before set_population / set_population_batch."""
        self._check(self._lib.ks_set_breakup_mode(self._h, int(mode), int(max_objects)))

    def set_masses(self, mass_kg):
        m = np.ascontiguousarray(mass_kg, dtype=np.float64)
        self._check(self._lib.ks_set_masses(self._h, len(m), ptr(m)))

    def impact(self, target, projectile_mass_kg=10.0, v_rel_km_s=10.0):
        self._check(self._lib.ks_impact(self._h, int(target), float(projectile_mass_kg), float(v_rel_km_s)))

    def save_population(self, path):
        """Writes the resident population, clock and fragmentation streams to `path` (exact resume)."""
        self._check(self._lib.ks_save_population(self._h, os.fspath(path).encode()))

    def load_population(self, path):
        self._check(self._lib.ks_load_population(self._h, os.fspath(path).encode()))

    def take_breakups(self):
        cnt = C.c_int64()
        self._check(self._lib.ks_take_breakups(self._h, None, 0, C.byref(cnt)))
        out = np.zeros(cnt.value, dtype=BREAKUP_DTYPE)
        if cnt.value:
            self._check(self._lib.ks_take_breakups(self._h, ptr(out), cnt.value, C.byref(cnt)))
        return out[: cnt.value]

    def objects(self):
        """Per-object size_m, mass_kg, area_to_mass, event (-1: initial population) and realisation."""
        n = self._lib.ks_population_size(self._h)
        out = {"size_m": np.empty(n), "mass_kg": np.empty(n), "area_to_mass": np.empty(n),
               "event": np.empty(n, np.int32), "realisation": np.empty(n, np.int32)}
        self._check(self._lib.ks_get_objects(self._h, n, ptr(out["size_m"]), ptr(out["mass_kg"]),
                                             ptr(out["area_to_mass"]), ptr(out["event"]), ptr(out["realisation"])))
        return out

    def timing(self):
        t = Timing()
        self._check(self._lib.ks_get_timing(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in Timing._fields_}

    # --- one-shot calls on host buffers ---
    def screen(self, before, after, alive_after, size_m, t0, dt):
        """Screener::screen on given states; returns (conjunctions, stats)."""
        b = _states(before)
        n = b.shape[0]
        a = _states(after, n)
        al = np.ascontiguousarray(alive_after, dtype=np.uint8)
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        cap = 1024
        while True:
            out = np.zeros(cap, dtype=CONJ_DTYPE)
            stats = np.zeros(1, dtype=STATS_DTYPE)
            cnt = C.c_int64()
            self._check(self._lib.ks_screen(self._h, n, ptr(b), ptr(a), ptr(al), ptr(sz), float(t0), float(dt),
                                            ptr(out), cap, C.byref(cnt), ptr(stats)))
            if cnt.value <= cap:
                return out[: cnt.value], stats[0]
            cap = cnt.value

    def propagate(self, states, alive, epoch_jd, t, dt, steps):
        """`steps` x Simulation::step without screening, on host arrays (returns copies)."""
        st = _states(states).copy()
        al = np.ascontiguousarray(alive, dtype=np.uint8).copy()
        self._check(self._lib.ks_propagate(self._h, st.shape[0], ptr(st), ptr(al), float(epoch_jd), float(t),
                                           float(dt), int(steps)))
        return st, al

    def measure_fp64(self):
        """(add/mul, FMA) FP64 instructions per second of this device."""
        a = C.c_double()
        f = C.c_double()
        self._check(self._lib.ks_measure_fp64(self._h, C.byref(a), C.byref(f)))
        return a.value, f.value

    def measure_fp32(self):
        """(add/mul, FMA) FP32 instructions per second of this device."""
        a = C.c_double()
        f = C.c_double()
        self._check(self._lib.ks_measure_fp32(self._h, C.byref(a), C.byref(f)))
        return a.value, f.value

    def measure_fp32x2(self):
        """Packed FP32 FMA operations per second (FFMA2, two per lane and instruction)."""
        f = C.c_double()
        self._check(self._lib.ks_measure_fp32x2(self._h, C.byref(f)))
        return f.value


def moon_position(jd):
    lib = load_library()
    out = np.zeros(3)
    lib.ks_moon_position(float(jd), ptr(out))
    return out


def sbm_impact(state, target_mass_kg, target_size_m, projectile_mass_kg=10.0, v_rel_km_s=10.0, t=0.0, seed=1,
               lc_m=0.10, catastrophic_j_per_g=40.0):
    """NASA SBM forced impact on one object, on the host (no device).

    Returns (event record, fragment birth states (m, 6), sizes, masses, area-to-mass, [target alive, mass])."""
    lib = load_library()
    st = np.ascontiguousarray(state, dtype=np.float64).reshape(6)
    ev = np.zeros(1, dtype=BREAKUP_DTYPE)
    after = np.zeros(2)
    cap = 1024
    while True:
        fs, fz, fm, fa = np.zeros((cap, 6)), np.zeros(cap), np.zeros(cap), np.zeros(cap)
        m = lib.ks_sbm_impact(int(seed), float(lc_m), float(catastrophic_j_per_g), ptr(st), float(target_mass_kg),
                              float(target_size_m), float(projectile_mass_kg), float(v_rel_km_s), float(t), ptr(ev),
                              ptr(fs), ptr(fz), ptr(fm), ptr(fa), cap, ptr(after))
        if m < 0:
            raise KsError(1, "ks_sbm_impact: bad arguments")
        if m <= cap:
            return ev[0], fs[:m], fz[:m], fm[:m], fa[:m], after
        cap = int(m)


def generate_population(seed, n_base, n_total=None, n_parents=200, frag_age_max_s=0.0):
    """Seeded synthetic catalogue: (states (n, 6), size_m (n,), alive (n,))."""
    lib = load_library()
    n_total = n_base if n_total is None else n_total
    st = np.zeros((n_total, 6))
    sz = np.zeros(n_total)
    al = np.zeros(n_total, dtype=np.uint8)
    rc = lib.ks_generate_population(C.c_uint64(seed), n_base, n_total, int(n_parents), float(frag_age_max_s),
                                    ptr(st), ptr(sz), ptr(al))
    if rc != 0:
        raise KsError(rc, "ks_generate_population: bad arguments")
    return st, sz, al
