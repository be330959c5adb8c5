"""ORACLE - test infrastructure only.

ctypes front-end of the CPU checkers built by oracle/Makefile:
  - ``Oracle``    oracle/libks_oracle.so, the plain-C restatement (ks_oracle.c)
  - ``Reference`` oracle/_ref/libksref.so, the reference's own sources plus
                  ref_harness.cpp (present only where the reference tree was
                  available at build time)
Both expose the same calls (run / screen / step helpers) with the same record
layouts as the engine. Only tests/, the smoke check and bench.py's CPU-baseline
leg use this module; the product never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libks_oracle.so")
WORKLOAD_SO = os.path.join(HERE, "libks_workload.so")
REF_SO = os.path.join(HERE, "_ref", "libksref.so")
# Source tree of the reference, read only to build oracle/_ref and the golden
# fixtures. One environment variable names it everywhere.
REFERENCE_TREE = os.environ.get("KESSLER_REFERENCE", "/root/reference")


def reference_tree_present():
    return os.path.isdir(os.path.join(REFERENCE_TREE, "src"))

CONJ_DTYPE = np.dtype(
    [("i", "<i4"), ("j", "<i4"), ("step", "<i8"), ("t", "<f8"), ("miss_km", "<f8"),
     ("v_rel_km_s", "<f8"), ("collision", "<i4"), ("realisation", "<i4")], align=True)
BREAKUP_DTYPE = np.dtype(
    [("step", "<i8"), ("t", "<f8"), ("id", "<i4"), ("realisation", "<i4"), ("target", "<i8"), ("projectile", "<i8"),
     ("catastrophic", "<i4"), ("fragments", "<i4"), ("escaped", "<i4"), ("pad", "<i4"), ("first_fragment", "<i8"),
     ("v_rel_km_s", "<f8"), ("energy_j_per_g", "<f8"), ("target_mass_kg", "<f8"), ("projectile_mass_kg", "<f8"),
     ("sbm_mass_kg", "<f8"), ("expected_fragments", "<f8"), ("fragments_mass_kg", "<f8"), ("position", "<f8", (3,))],
    align=True)
STATS_DTYPE = np.dtype(
    [("step", "<i8"), ("candidate_pairs", "<i8"), ("refined_pairs", "<i8"), ("co_orbiting", "<i8"),
     ("conjunctions", "<i8"), ("cell_km", "<f8"), ("max_cell_objects", "<i4"), ("alive", "<i4")],
    align=True)

_P = C.c_void_p
_D = C.c_double
_L = C.c_long


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def build(ref=True):
    """Builds the checkers (ref=True also builds the reference when its tree exists)."""
    targets = ["oracle"]
    if ref and reference_tree_present():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + REFERENCE_TREE] + targets, check=True)


def generate_population(seed, n_base, n_total=None, n_parents=200, frag_age_max_s=0.0):
    """The seeded synthetic population, from oracle/libks_workload.so: the
    engine's own generator source built as a separate library, so that the
    CPU-baseline harness builds its inputs without loading the engine. Same
    arrays as the engine's ks_generate_population, bit for bit."""
    if not os.path.exists(WORKLOAD_SO):
        build(ref=False)
    lib = C.CDLL(WORKLOAD_SO)
    f = lib.ks_generate_population
    f.restype = C.c_int
    n_total = n_base if n_total is None else n_total
    st = np.zeros((n_total, 6))
    sz = np.zeros(n_total)
    al = np.zeros(n_total, dtype=np.uint8)
    rc = f(C.c_uint64(seed), C.c_int64(n_base), C.c_int64(n_total), C.c_int(int(n_parents)),
           _D(float(frag_age_max_s)), _p(st), _p(sz), _p(al))
    if rc != 0:
        raise ValueError("ks_generate_population: bad arguments")
    return st, sz, al


class _Checker:
    prefix = ""
    has_threads = False

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        pre = self.prefix
        run = getattr(self.lib, pre + "run")
        run.restype = _L
        scr = getattr(self.lib, pre + "screen")
        scr.restype = _L
        for name in ("moon_position", "acceleration", "rk4"):
            getattr(self.lib, pre + name).restype = None
        getattr(self.lib, pre + "filter_pair").restype = C.c_int
        getattr(self.lib, pre + "filter_pair").argtypes = [_D] * 9
        getattr(self.lib, pre + "prefilter_keep").restype = C.c_int
        getattr(self.lib, pre + "prefilter_keep").argtypes = [C.c_float] * 9

    def moon_position(self, jd):
        out = np.zeros(3)
        getattr(self.lib, self.prefix + "moon_position")(_D(jd), _p(out))
        return out

    def rk4(self, s, dt, m0, m1, m2):
        out = np.zeros(6)
        args = [np.ascontiguousarray(x, dtype=np.float64) for x in (s, m0, m1, m2)]
        getattr(self.lib, self.prefix + "rk4")(_p(args[0]), _D(dt), _p(args[1]), _p(args[2]), _p(args[3]),
                                               _p(out))
        return out

    def filter_pair(self, dr, dv, dt, thr, vmin2):
        return getattr(self.lib, self.prefix + "filter_pair")(*(list(map(float, dr)) + list(map(float, dv))
                                                               + [dt, thr, vmin2]))

    def prefilter_keep(self, dr, dv, dt, thr, vmin2):
        return getattr(self.lib, self.prefix + "prefilter_keep")(*(list(map(float, dr)) + list(map(float, dv))
                                                                  + [dt, thr, vmin2]))

    def run(self, states, size_m, alive=None, epoch_jd=2461253.916666667, t_start=0.0, dt=10.0, steps=1,
            screen=True, threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, threads=0, conj_cap=None):
        """The CLI step loop; returns (final states, alive, conjunctions, per-step stats[, timings])."""
        st = np.ascontiguousarray(states, dtype=np.float64).copy()
        n = st.shape[0]
        al = np.ones(n, np.uint8) if alive is None else np.ascontiguousarray(alive, dtype=np.uint8).copy()
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        cap = conj_cap if conj_cap is not None else max(1024, 64 * steps)
        stats = np.zeros(max(steps, 1), dtype=STATS_DTYPE)
        timings = np.zeros(5)
        while True:
            s2 = st.copy()
            a2 = al.copy()
            conj = np.zeros(cap, dtype=CONJ_DTYPE)
            args = [_L(n), _p(s2), _p(a2), _p(sz), _D(epoch_jd), _D(t_start), _D(dt), _L(steps),
                    C.c_int(1 if screen else 0), _D(threshold_km), _D(radius_scale), _D(min_vrel_km_s)]
            if self.has_threads:
                args.append(C.c_int(threads))
            args += [_p(conj), _L(cap), _p(stats)]
            if self.has_threads:
                args.append(_p(timings))
            total = getattr(self.lib, self.prefix + "run")(*args)
            if total < 0:
                raise RuntimeError("checker run failed")
            if total <= cap:
                self.last_timings = timings.copy()
                return s2, a2, conj[:total], stats[:steps]
            cap = int(total)

    def screen(self, before, after, alive_after, size_m, t0, dt, threshold_km=5.0, radius_scale=1.0,
               min_vrel_km_s=0.01, threads=0):
        b = np.ascontiguousarray(before, dtype=np.float64)
        a = np.ascontiguousarray(after, dtype=np.float64)
        al = np.ascontiguousarray(alive_after, dtype=np.uint8)
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        n = b.shape[0]
        cap = 1024
        while True:
            out = np.zeros(cap, dtype=CONJ_DTYPE)
            stats = np.zeros(1, dtype=STATS_DTYPE)
            args = [_L(n), _p(b), _p(a), _p(al), _p(sz), _D(t0), _D(dt), _D(threshold_km), _D(radius_scale),
                    _D(min_vrel_km_s)]
            if self.has_threads:
                args.append(C.c_int(threads))
            args += [_p(out), _L(cap), _p(stats)]
            k = getattr(self.lib, self.prefix + "screen")(*args)
            if k <= cap:
                return out[:k], stats[0]
            cap = int(k)


class Oracle(_Checker):
    """The plain-C restatement (oracle/ks_oracle.c)."""
    prefix = "kso_"
    has_threads = False

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)


class Reference(_Checker):
    """The reference compiled from its own sources (oracle/_ref/libksref.so)."""
    prefix = "ksref_"
    has_threads = True

    def __init__(self, path=REF_SO):
        super().__init__(path)
        self.lib.ksref_max_threads.restype = C.c_int
        self.lib.ksref_load_catalog.restype = _L
        self.lib.ksref_read_epoch_jd.restype = _D

    def max_threads(self):
        return self.lib.ksref_max_threads()

    def impact(self, state, mass_kg, size_m, projectile_mass_kg, v_rel_km_s, t=0.0, seed=1, lc_m=0.10,
               catastrophic_j_per_g=40.0, epoch_jd=2461253.916666667):
        """Fragmentation::impact on a one-object simulation: (event, states, sizes, masses, a2m, [alive, mass])."""
        f = self.lib.ksref_impact
        f.restype = _L
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(6)
        ev = np.zeros(1, dtype=BREAKUP_DTYPE)
        after = np.zeros(2)
        cap = 1024
        while True:
            fs, fz, fm, fa = np.zeros((cap, 6)), np.zeros(cap), np.zeros(cap), np.zeros(cap)
            m = f(C.c_uint64(seed), _D(lc_m), _D(catastrophic_j_per_g), _p(st), _D(mass_kg), _D(size_m),
                  _D(projectile_mass_kg), _D(v_rel_km_s), _D(epoch_jd), _D(t), _p(ev), _p(fs), _p(fz), _p(fm),
                  _p(fa), _L(cap), _p(after))
            if m <= cap:
                return ev[0], fs[:m], fz[:m], fm[:m], fa[:m], after
            cap = int(m)

    def run_breakup(self, states, size_m, mass_kg=None, alive=None, epoch_jd=2461253.916666667, dt=10.0, steps=1,
                    threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, threads=0, lc_m=0.10,
                    catastrophic_j_per_g=40.0, seed=1, impact=None):
        """The CLI loop with --breakup; impact = (index, mass_kg, v_rel_km_s, step) or None.

        Returns dict: states, alive, size_m, mass_kg, area_to_mass, event, conj, events, stats."""
        f = self.lib.ksref_run_breakup
        f.restype = C.c_int
        st = np.ascontiguousarray(states, dtype=np.float64)
        n = st.shape[0]
        al = np.ones(n, np.uint8) if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        sz = np.ascontiguousarray(size_m, dtype=np.float64)
        ms = np.zeros(n) if mass_kg is None else np.ascontiguousarray(mass_kg, dtype=np.float64)
        ii, im, iv, istep = impact if impact is not None else (-1, 0.0, 0.0, 0)
        obj_cap, conj_cap, ev_cap = 2 * n + 1024, 4096, 256
        while True:
            out = {"states": np.zeros((obj_cap, 6)), "alive": np.zeros(obj_cap, np.uint8),
                   "size_m": np.zeros(obj_cap), "mass_kg": np.zeros(obj_cap), "area_to_mass": np.zeros(obj_cap),
                   "event": np.zeros(obj_cap, np.int32), "conj": np.zeros(conj_cap, dtype=CONJ_DTYPE),
                   "events": np.zeros(ev_cap, dtype=BREAKUP_DTYPE), "stats": np.zeros(max(steps, 1), STATS_DTYPE)}
            counts = np.zeros(3, np.int64)
            rc = f(_L(n), _p(st), _p(al), _p(sz), _p(ms), _D(epoch_jd), _D(dt), _L(steps), _D(threshold_km),
                   _D(radius_scale), _D(min_vrel_km_s), C.c_int(threads), _D(lc_m), _D(catastrophic_j_per_g),
                   C.c_uint64(seed), _L(ii), _D(im), _D(iv), _L(istep), _L(obj_cap), _p(out["states"]),
                   _p(out["alive"]), _p(out["size_m"]), _p(out["mass_kg"]), _p(out["area_to_mass"]),
                   _p(out["event"]), _p(out["conj"]), _L(conj_cap), _p(out["events"]), _L(ev_cap),
                   _p(out["stats"]), _p(counts))
            if rc == 0:
                m, nc, ne = (int(x) for x in counts)
                for k in ("states", "alive", "size_m", "mass_kg", "area_to_mass", "event"):
                    out[k] = out[k][:m]
                out["conj"] = out["conj"][:nc]
                out["events"] = out["events"][:ne]
                out["stats"] = out["stats"][:steps]
                return out
            obj_cap, conj_cap, ev_cap = max(obj_cap, int(counts[0])), max(conj_cap, int(counts[1])), \
                max(ev_cap, int(counts[2]))

    def load_catalog(self, path):
        """(states, size_m, ids, epoch_jd) via the reference parser."""
        p = path.encode()
        n = self.lib.ksref_load_catalog(p, _L(0), None, None, None, None)
        st = np.zeros((n, 6))
        sz = np.zeros(n)
        ids = np.zeros(n, np.int32)
        dropped = C.c_int(0)
        self.lib.ksref_load_catalog(p, _L(n), _p(st), _p(sz), _p(ids), C.byref(dropped))
        return st, sz, ids, self.lib.ksref_read_epoch_jd(p)


def reference_available():
    return os.path.exists(REF_SO)
