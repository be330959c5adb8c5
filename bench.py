"""Benchmark of the per-step hot path: RK4 propagation + conjunction screening.

One step = one Simulation::step of the whole population followed by the
screening of that step (grid, pair filter, Hermite TCA refinement), i.e. one
iteration of the reference CLI loop (src/main.cpp:346-407) with --conj-km 5.

Workload (default): 1 000 000 objects = 28 340 seeded catalogue objects + 971 660
fragments in 200 clouds around random LEO parents (isotropic Delta-v, log-normal
magnitude, median 50 m/s, sigma_ln 0.8; radii 0.05-0.5 m, power law -1.6), each
cloud released at a random time within the day before the epoch; dt = 10 s,
threshold 5 km, radius scale 1, minimum encounter speed 10 m/s. Synthetic data.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--precision fp64]

Rank 0 prints one JSON line. With N > 1 (torchrun) every rank runs its own
independent realisation (seed + rank): weak scaling, no collective on the data
path; the timing is the max over ranks of the device time.
"""
import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "object-steps/s at 1M objs, split-prec vs FP64 at ≤1 m/24 h error; pairs/s"
L2_BYTES = 126 * 1024 * 1024
FLUSH_BYTES = 256 * 1024 * 1024

# Algorithmic FP64 operations per unit (as the reference writes them):
#   object-step: acceleration x 4 (33 mul + 21 add/sub + 5 div + 3 sqrt each)
#                + 78 RK4 combination ops = 294 mul/add + 20 div + 12 sqrt
#   candidate pair: 6 subtractions for dr, dv, then |dr|^2, |dv|^2, dr.dv (15)
#                   and the division-free distance gate (4) = 25 ops (FP64 in
#                   the plain path, FP32 in the split path); a pair that
#                   reaches the full filter adds its ts, p, |p|, gate and
#                   convexity terms: 30 mul/add + 1 div + 3 sqrt
FLOPS_OBJECT_STEP = 294 + 20 + 12
FLOPS_PAIR_CHEAP = 25
FLOPS_PAIR_FULL = 34


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=360)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="split", choices=["fp64", "split"],
                    help="path reported as the headline value (the other one is reported beside it)")
    ap.add_argument("--objects", type=int, default=1_000_000)
    ap.add_argument("--base", type=int, default=28_340)
    ap.add_argument("--parents", type=int, default=200)
    ap.add_argument("--frag-age-s", type=float, default=86400.0)
    ap.add_argument("--seed", type=int, default=20260801)
    ap.add_argument("--dt", type=float, default=10.0)
    ap.add_argument("--conj-km", type=float, default=5.0)
    ap.add_argument("--steps-per-graph", type=int, default=32)
    ap.add_argument("--cpu-steps", type=int, default=24, help="steps of the CPU baseline sample (~13 s on 16 cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-error-study", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=360,
                    help="steps of the end-to-end run (default 360: one simulated hour, a run long enough that the "
                         "population's upload and download weigh as in a real run; the line also reports an "
                         "end-to-end run of --steps steps)")
    ap.add_argument("--ens-realisations", type=int, default=64)
    ap.add_argument("--ens-steps", type=int, default=360)
    ap.add_argument("--ens-lc", type=float, default=0.05)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--cascade-realisations", type=int, default=16)
    ap.add_argument("--cascade-steps", type=int, default=360)
    ap.add_argument("--cascade-budget", type=float, default=1.25,
                    help="population budget of the cascade, as a multiple of its starting size")
    ap.add_argument("--no-cascade", action="store_true")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def config_of(a):
    return {"workload": f"{a.objects} objects ({a.base} catalogue + {a.objects - a.base} fragments in "
                        f"{a.parents} clouds released within {a.frag_age_s / 3600:g} h), dt {a.dt:g} s, "
                        f"--conj-km {a.conj_km:g}, radius scale 1, min-vrel 10 m/s",
            "objects": a.objects, "dt_s": a.dt, "threshold_km": a.conj_km, "precision": a.precision,
            "seed": a.seed, "steps_per_graph": a.steps_per_graph,
            "l2": f"flushed before every timed step ({FLUSH_BYTES >> 20} MiB write, outside the timed events)",
            "parallelism": "one independent realisation per GPU (seed + rank)"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0}, "fallback"


def _checkers():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import checkers
    return checkers


def cpu_checker():
    """The reference CPU path (oracle/_ref, built from the reference's sources)
    on all host threads, else the oracle port on one."""
    checkers = _checkers()
    if checkers.reference_available():
        return checkers.Reference(), "reference", os.cpu_count() or 1
    return checkers.Oracle(), "port", 1


def cpu_baseline(a, st, sz, al, steps):
    """The reference CPU path on this host: the first `steps` steps of the population."""
    chk, kind, threads = cpu_checker()
    t0 = time.perf_counter()
    fs, fa, conj, stats = chk.run(st, sz, al, epoch_jd=2461253.916666667, dt=a.dt, steps=steps, screen=True,
                                  threshold_km=a.conj_km, threads=threads)
    wall = time.perf_counter() - t0
    # objects propagated = alive at the start of each step
    alive_start = int(al.sum()) + int(np.sum(stats["alive"][:-1]))
    return {"value": alive_start / wall, "unit": "object-steps/s", "cores": threads, "kind": kind,
            "sample": f"first {steps} steps of the same {len(st)}-object population, screening included",
            "pairs_per_s": float(stats["candidate_pairs"].sum()) / wall, "wall_s": wall,
            "conjunctions": int(len(conj)), "_run": (fs, fa, conj, stats)}


def run_reference_arm(a):
    """The reference's own CPU implementation of the path (oracle/_ref) on the
    host's cores, on this arm's workload: W untimed steps, then K timed steps
    continuing from them. Its inputs come from oracle/libks_workload.so, so
    this arm loads nothing of the engine."""
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    checkers = _checkers()
    st, sz, al = checkers.generate_population(a.seed, a.base, a.objects, a.parents, a.frag_age_s)
    chk, kind, threads = cpu_checker()
    steps, warm = a.steps, a.warmup
    kw = dict(epoch_jd=2461253.916666667, dt=a.dt, screen=True, threshold_km=a.conj_km, threads=threads)
    if warm > 0:
        st, al, _, _ = chk.run(st, sz, al, t_start=0.0, steps=warm, **kw)
    t0 = time.perf_counter()
    _, _, conj, stats = chk.run(st, sz, al, t_start=warm * a.dt, steps=steps, **kw)
    wall = time.perf_counter() - t0
    alive_start = int(al.sum()) + int(np.sum(stats["alive"][:-1]))
    value = alive_start / wall
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "object-steps/s",
            "n_gpus": a.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * wall / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; no dataset)", "config": config_of(a),
            "pairs_per_s": float(stats["candidate_pairs"].sum()) / wall,
            "conjunctions_per_step": len(conj) / steps,
            "cpu_baseline": {"value": value, "unit": "object-steps/s", "cores": threads, "kind": kind,
                             "sample": f"all {steps} timed steps (after {warm} untimed) of the {a.objects}-object "
                                       f"workload, every host thread"},
            "e2e": {"value": value, "unit": "object-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def parity_vs_reference(ks, eng, a, st, sz, al, ref_run, steps):
    """The GPU FP64 path against the reference CPU path's own run of the first
    `steps` steps of the same population (the cpu_baseline sample): conjunction
    records and per-step counters compared bit for bit, final states too; and
    the split path's position error against the same reference states."""
    fs_ref, fa_ref, conj_ref, stats_ref = ref_run
    out = {"n_objects": int(len(st)), "steps": int(steps), "reference_conjunctions": int(len(conj_ref))}
    for name, prec in (("fp64", ks.PRECISION_FP64), ("split", ks.PRECISION_SPLIT)):
        eng.set_precision(prec)
        eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
        eng.set_screening(True, a.conj_km, 1.0, 0.01)
        eng.set_l2_flush(0)
        eng.set_profiling(False)
        eng.set_population(st, sz, al)
        eng.run(steps)
        fs, fa = eng.get_population()
        conj = eng.take_conjunctions()
        stats = eng.take_step_stats()
        recs = len(conj) == len(conj_ref) and all(np.array_equal(conj[f], conj_ref[f]) for f in
                                                  ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision"))
        ctrs = all(np.array_equal(stats[f], stats_ref[f]) for f in
                   ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km",
                    "max_cell_objects", "alive"))
        live = (fa == 1) & (fa_ref == 1)
        dr = np.linalg.norm(fs[live, :3] - fs_ref[live, :3], axis=1) * 1e3
        dv = np.linalg.norm(fs[live, 3:] - fs_ref[live, 3:], axis=1) * 1e6
        kg = set(zip(conj["i"].tolist(), conj["j"].tolist(), conj["step"].tolist()))
        kr = set(zip(conj_ref["i"].tolist(), conj_ref["j"].tolist(), conj_ref["step"].tolist()))
        out[name] = {"records_equal": bool(recs), "counters_equal": bool(ctrs),
                     "states_equal": bool(np.array_equal(fs, fs_ref) and np.array_equal(fa, fa_ref)),
                     "conjunctions": int(len(conj)), "pairs_only_here": len(kg - kr), "pairs_only_reference": len(kr - kg),
                     "max_pos_err_m": float(dr.max()) if dr.size else 0.0,
                     "max_vel_err_mm_s": float(dv.max()) if dv.size else 0.0}
    return out


def timed_chunk(steps, spg):
    """Steps per graph launch of a timed run of `steps` steps: the largest
    divisor of `steps` not above spg (every chunk then runs as one captured
    graph), or spg itself when that divisor would be under half of it."""
    spg = max(1, spg)
    d = max(k for k in range(1, min(steps, spg) + 1) if steps % k == 0) if steps > 0 else spg
    return d if 2 * d >= min(steps, spg) else spg


def timed_run(ks, eng, a, st, sz, al, precision, barrier):
    """W untimed warm-up steps, then K timed steps; per-step device time from
    CUDA events on the engine's stream, L2 flushed before each step outside
    the events."""
    eng.set_precision(precision)
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
    eng.set_screening(True, a.conj_km, 1.0, 0.01)
    eng.set_l2_flush(FLUSH_BYTES)
    eng.set_profiling(True)
    eng.set_population(st, sz, al)
    # The warm-up steps run as one graph: the process's first graph launch
    # carries a one-time set-up cost of tens of milliseconds.
    eng.set_steps_per_graph(a.warmup)
    eng.run(a.warmup)
    eng.set_steps_per_graph(timed_chunk(a.steps, a.steps_per_graph))
    eng.take_conjunctions()
    eng.take_step_stats()
    # The timed chunks' graphs are captured now, outside the timed region.
    eng.prepare_run()
    barrier()
    w0 = time.perf_counter()
    eng.run(a.steps)
    barrier()
    wall = time.perf_counter() - w0
    return eng.timing(), eng.take_conjunctions(), eng.take_step_stats(), wall


def _reduce(pg, x, op):
    if not pg:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    pg.all_reduce(t, op=op(pg))
    return float(t.item())


def max_over_ranks(pg, x):
    """Max over ranks (the slowest rank's device time bounds the job)."""
    return _reduce(pg, x, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(pg, x):
    """Sum over ranks (whole-job work: every rank runs its own realisation)."""
    return _reduce(pg, x, lambda d: d.ReduceOp.SUM)


def realisation_seed(seed, rank):
    """Seed of the population a rank simulates (independent realisations)."""
    return seed + rank


def roofline_of(tm, a, fp64_rate, fp32_rates, split):
    """Dominant kernel of the step and its achieved rate against the measured
    issue rate of the pipe that bounds it (algorithmic operations per launch
    divided by the launch's average CUDA-event duration). fp32_rates: the
    measured FP32 operation rates of this GPU (add/mul, FMA, packed FFMA2);
    the pair kernel is held to the highest of them (its gate runs on packed
    FMAs) and its fraction against each is listed."""
    if not isinstance(fp32_rates, dict):
        fp32_rates = {"addmul": fp32_rates}
    fp32_rate = max(fp32_rates.values())
    steps = max(1, tm["steps"])
    phases = {k: tm[k] / steps for k in ("propagate_ms", "sort_ms", "cells_ms", "pairs_ms", "refine_ms", "chunk_ms")}
    prop_ops = FLOPS_OBJECT_STEP * tm["object_steps"] / steps
    pair_ops = FLOPS_PAIR_CHEAP * tm["candidate_pairs"] / steps
    kernels = {
        "propagate": {"ms": phases["propagate_ms"], "ops": prop_ops, "pipe": "fp64", "peak": fp64_rate},
        # Both precisions gate pairs in FP32 (FP64 precision: pair variant 2,
        # the default) and decide with the exact FP64 filter.
        "pairs": {"ms": phases["pairs_ms"], "ops": pair_ops, "pipe": "fp32", "peak": fp32_rate},
    }
    for k in kernels.values():
        k["tflops"] = k["ops"] / (k["ms"] * 1e-3) / 1e12 if k["ms"] > 0 else None
        k["frac"] = (k["tflops"] * 1e12 / k["peak"]) if k["tflops"] else None
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    d = kernels[dom]
    # The memory-side phases against HBM: algorithmic bytes per step over the
    # phase's device time (the sort moves u64 keys that carry the object index).
    peaks, peak_src = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    n_obj = tm["object_steps"] / steps
    passes = tm["sort_passes"]
    hbm_phases = {
        "sort": (16.0 * passes * n_obj, phases["sort_ms"],
                 f"{passes} radix passes x (8 B key read + 8 B key written) per object"),
        "cells": (76.0 * n_obj, phases["cells_ms"],
                  "per object: 8 B key read, 32 B FP32 record gathered, 32 B record + 4 B index written"),
        "pairs": (32.0 * n_obj, phases["pairs_ms"], "per object: its 32 B FP32 record read once"),
    }
    if tm.get("sort_cells_fused"):
        # One launch sorts and builds the cells: its time is the sort phase's.
        hbm_phases = {
            "sort_cells": ((16.0 * passes + 76.0) * n_obj, phases["sort_ms"] + phases["cells_ms"],
                           f"{passes} radix passes x (8 B key read + 8 B key written) per object, then per "
                           "object 8 B key read, 32 B FP32 record gathered, 32 B record + 4 B index written"),
            "pairs": hbm_phases["pairs"],
        }
    hbm_kernels = {}
    for k, (nbytes, ms, what) in hbm_phases.items():
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
        hbm_kernels[k] = {"ms": ms, "algorithmic_bytes": nbytes, "gbs": gbs, "frac": gbs / hbm if gbs else None,
                          "what": what}
    fp32_fracs = {k: (kernels["pairs"]["tflops"] * 1e12 / v if kernels["pairs"]["tflops"] and v else None)
                  for k, v in fp32_rates.items()}
    return {"bound": d["pipe"], "kernel": dom, "achieved": d["tflops"], "peak": d["peak"] / 1e12,
            "unit": "TFLOP/s", "frac": d["frac"], "traffic": traffic_of(dom, split),
            # How busy the pipes really are (the pair kernel prunes most candidates
            # before its gate, so the algorithmic rate above can near the issue rate).
            "pipes_ncu": pipes_of(dom, split),
            "pipes_ncu_source": "ncu --set full of one launch at 400k objects (the committed profile summaries), "
                                "not measured in this run",
            "peak_source": "measured on this GPU by the project microbenchmarks (dependent chains of FP32 add/mul, "
                           "FMA and packed FFMA2, FP64 add/mul; the highest FP32 rate is the peak); "
                           "MEASURED_PEAKS.json has no FP64/FP32 SIMT figure",
            "pairs_fp32_rates_tops": {k: v / 1e12 for k, v in fp32_rates.items()},
            "pairs_frac_by_fp32_rate": fp32_fracs,
            "algorithmic_ops_per_launch": d["ops"], "phase_ms_per_step": phases,
            "kernels": {k: {"ms": v["ms"], "pipe": v["pipe"], "tflops": v["tflops"], "frac": v["frac"]}
                        for k, v in kernels.items()},
            "hbm": {"peak_gbs": hbm,
                    "peak_source": ("copy bandwidth measured on this pool (MEASURED_PEAKS.json hbm_gbs)"
                                    if peak_src == "measured" else "the profiling recipe's fallback (6.65 TB/s)"),
                    "phases": hbm_kernels}}


def pipes_of(kernel, split):
    """Pipe and issue utilisation of the kernel (fractions of peak, active
    cycles; DRAM of elapsed) from the committed ncu summaries, if present."""
    path = os.path.join(ROOT, "profiles", "pipes_per_kernel.txt")
    key = "pairs_split" if kernel == "pairs" else f"{kernel}_{'split' if split else 'exact'}"
    out = {}
    try:
        for line in open(path):
            f = line.split()
            if len(f) >= 3 and f[0] == key:
                out[f[1]] = float(f[2])
    except (OSError, ValueError):
        return None
    return out or None


def traffic_of(kernel, split):
    """DRAM bytes per launch of the kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    key = "pairs_split" if kernel == "pairs" else f"{kernel}_{'split' if split else 'exact'}"
    try:
        for line in open(path):
            f = line.split()
            if len(f) >= 2 and f[0] == key:
                return float(f[1])
    except OSError:
        pass
    return None


def launches_per_step(sort_passes, fused=False):
    # Fused: propagate, fix_keys, sort + cells (one cooperative launch), pairs,
    # refine. Otherwise: propagate, fix_keys, sort (one kernel per pass; the
    # propagation and, if it rebuilds keys, k_fix_keys count the digits), cells
    # (count, scan, write, neighbours, item count, scan, item write), pairs, refine.
    if fused:
        return 1 + 1 + 1 + 1 + 1
    return 1 + 1 + sort_passes + 7 + 1 + 1


# Per graph chunk of the timed run: chunk_init and the ordering of the chunk's
# conjunction records (keys, upsweep, 4 passes, gather; chunks this long take
# the multi-block sort).
LAUNCHES_PER_CHUNK = 8


BORDER_TOL_KM = 1e-5  # 1 cm: the agreement the plain form is held to after 24 h


def borderline_pairs(c_head, c_other, size_m, thr_km, head_is_split, tol_km=BORDER_TOL_KM, listed=20):
    """Conjunctions of either precision whose miss distance lies within tol of the
    threshold or of the pair's radius sum (where the two paths may decide
    differently), counted and listed separately with both miss distances; and
    every pair found by one precision only, with its miss distance and TCA
    fraction of the step (the refinement drops TCAs within 1e-9 of a step edge)."""
    split_c, fp64_c = (c_head, c_other) if head_is_split else (c_other, c_head)

    def near(c):
        rsum = 0.5e-3 * (size_m[c["i"]] + size_m[c["j"]])
        m = c["miss_km"]
        return (np.abs(m - thr_km) < tol_km) | (np.abs(m - rsum) < tol_km)

    keys = set()
    for c in (split_c, fp64_c):
        sel = c[near(c)]
        keys.update(zip(sel["i"].tolist(), sel["j"].tolist(), sel["step"].tolist()))

    def miss_of(c, key):
        hit = c[(c["i"] == key[0]) & (c["j"] == key[1]) & (c["step"] == key[2])]
        return float(hit["miss_km"][0]) if len(hit) else None

    rows = [{"i": k[0], "j": k[1], "step": k[2], "miss_km_split": miss_of(split_c, k), "miss_km_fp64": miss_of(fp64_c, k),
             "radius_sum_km": 0.5e-3 * float(size_m[k[0]] + size_m[k[1]])} for k in sorted(keys, key=lambda k: (k[2], k[0], k[1]))]
    only = [r for r in rows if r["miss_km_split"] is None or r["miss_km_fp64"] is None]
    ks_ = set(zip(split_c["i"].tolist(), split_c["j"].tolist(), split_c["step"].tolist()))
    kf_ = set(zip(fp64_c["i"].tolist(), fp64_c["j"].tolist(), fp64_c["step"].tolist()))
    one_set = []
    for name, c, keys_only in (("split", split_c, ks_ - kf_), ("fp64", fp64_c, kf_ - ks_)):
        for k in sorted(keys_only, key=lambda k: (k[2], k[0], k[1]))[:listed]:
            hit = c[(c["i"] == k[0]) & (c["j"] == k[1]) & (c["step"] == k[2])][0]
            one_set.append({"found_by": name, "i": k[0], "j": k[1], "step": k[2], "miss_km": float(hit["miss_km"]),
                            "t": float(hit["t"]), "radius_sum_km": 0.5e-3 * float(size_m[k[0]] + size_m[k[1]])})
    return {"borderline": {"tolerance_km": tol_km, "count": len(rows), "in_one_set_only": len(only),
                           "listed": (only + [r for r in rows if r not in only])[:listed]},
            "one_set_only": one_set}


def error_study(ks, eng, a, st, al):
    """Split vs FP64 propagation of the whole population: position and velocity
    differences at 1, 6 and 24 h (the FP64 path is bit-identical to the reference)."""
    out = {}
    s64, s32, a64, a32, t = st, st, al, al, 0.0
    for hours in (1, 6, 24):
        steps = int(round((hours * 3600.0 - t) / a.dt))
        eng.set_precision(ks.PRECISION_FP64)
        s64, a64 = eng.propagate(s64, a64, ks.DEFAULT_EPOCH_JD, t, a.dt, steps)
        eng.set_precision(ks.PRECISION_SPLIT)
        s32, a32 = eng.propagate(s32, a32, ks.DEFAULT_EPOCH_JD, t, a.dt, steps)
        t = hours * 3600.0
        live = (a64 == 1) & (a32 == 1)
        dr = np.linalg.norm(s32[live, :3] - s64[live, :3], axis=1) * 1e3
        dv = np.linalg.norm(s32[live, 3:] - s64[live, 3:], axis=1) * 1e6
        out[f"{hours}h"] = {"max_pos_m": float(dr.max()), "p99_pos_m": float(np.percentile(dr, 99)),
                            "median_pos_m": float(np.median(dr)), "max_vel_mm_s": float(dv.max()),
                            "alive_mismatch": int(((a64 == 1) != (a32 == 1)).sum())}
    return out


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference_arm(a)
    world, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    ks = importlib.import_module("kessler-syndrom-simulation_b200")
    st, sz, al = ks.generate_population(realisation_seed(a.seed, rank), a.base, a.objects, a.parents, a.frag_age_s)

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    eng = ks.Engine(local)
    fp64_rate, fp32_rate = eng.measure_fp64()[0], measure_fp32(eng)
    head = ks.PRECISION_SPLIT if a.precision == "split" else ks.PRECISION_FP64
    other = ks.PRECISION_FP64 if head == ks.PRECISION_SPLIT else ks.PRECISION_SPLIT
    runs = {}
    clk = None
    for prec in (other, head):  # headline last, with clocks sampled
        if prec == head:
            clocks = ClockSampler(local)
            clocks.start()
        runs[prec] = timed_run(ks, eng, a, st, sz, al, prec, barrier)
        if prec == head:
            clk = clocks.stop()

    def summary(prec):
        tm, conj, stats, wall = runs[prec]
        # Device time of the steps plus the chunks' own work (set-up,
        # checkpoint, ordering of the records); the L2 flushes are left out.
        dev_ms = max_over_ranks(pg, tm["total_ms"] + tm["chunk_ms"])
        obj = sum_over_ranks(pg, float(tm["object_steps"]))
        pairs = sum_over_ranks(pg, float(tm["candidate_pairs"]))
        steps = max(1, tm["steps"])
        return {"value": obj / (dev_ms * 1e-3), "ms_per_step": dev_ms / steps, "pairs_per_s": pairs / (dev_ms * 1e-3),
                "conjunctions_per_step": len(conj) / steps, "refined_pairs_per_step": tm["refined_pairs"] / steps,
                "exact_filter_pairs_per_step": tm["exact_filter_pairs"] / steps,
                "roofline": roofline_of(tm, a, fp64_rate, fp32_rate, prec == ks.PRECISION_SPLIT),
                "wall_s_timed_region": wall, "sort_passes": tm["sort_passes"],
                "sort_cells_fused": bool(tm.get("sort_cells_fused", 0))}

    main_s, other_s = summary(head), summary(other)
    c_head, c_other = runs[head][1], runs[other][1]
    kh = set(zip(c_head["i"].tolist(), c_head["j"].tolist(), c_head["step"].tolist()))
    ko = set(zip(c_other["i"].tolist(), c_other["j"].tolist(), c_other["step"].tolist()))
    split_set, fp64_set = (kh, ko) if head == ks.PRECISION_SPLIT else (ko, kh)
    tm_head = runs[head][0]
    line = {"metric": METRIC, "value": main_s["value"], "unit": "object-steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": main_s["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32 (split)" if head == ks.PRECISION_SPLIT else "f64",
            "data": "synthetic (seeded generator; no dataset)", "config": config_of(a),
            "pairs_per_s": main_s["pairs_per_s"], "conjunctions_per_step": main_s["conjunctions_per_step"],
            "gpu_launches": a.steps * launches_per_step(tm_head["sort_passes"], tm_head.get("sort_cells_fused", 0)) +
                            LAUNCHES_PER_CHUNK * -(-a.steps // max(1, a.steps_per_graph)),
            "roofline": main_s["roofline"], "clocks": clk,
            "fp64" if head == ks.PRECISION_SPLIT else "split": other_s,
            "conjunction_sets": dict(
                {"split_only": len(split_set - fp64_set), "fp64_only": len(fp64_set - split_set),
                 "common": len(split_set & fp64_set),
                 "over": f"the {a.steps} timed steps, pairs matched by (i, j, step)"},
                **borderline_pairs(c_head, c_other, sz, a.conj_km, head == ks.PRECISION_SPLIT)),
            "refined_pairs_per_step": main_s["refined_pairs_per_step"],
            "wall_s_timed_region": main_s["wall_s_timed_region"]}
    if not a.no_error_study:
        line["split_error_vs_fp64"] = error_study(ks, eng, a, st, al)
    if not a.no_e2e:
        line["e2e"] = e2e_run(ks, a, st, sz, al, local, barrier, pg, head)
        if line["e2e"]["steps"] != a.steps:
            line["e2e_at_timed_steps"] = e2e_run(ks, a, st, sz, al, local, barrier, pg, head, steps=a.steps)
    # Side workloads report a failure inside the line instead of losing it.
    if not a.no_ensemble:
        line["ensemble"] = side_run(ensemble_run, ks, a, local, barrier, pg, rank)
    if not a.no_cascade:
        line["cascade"] = side_run(cascade_run, ks, a, local, barrier, pg, rank, st, sz, al)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        base = cpu_baseline(a, st, sz, al, a.cpu_steps)
        line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"]["pairs_per_s"] = base["pairs_per_s"]
        line["parity_vs_reference"] = dict(parity_vs_reference(ks, eng, a, st, sz, al, base["_run"], a.cpu_steps),
                                           reference_kind=base["kind"])
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def side_run(fn, *args):
    try:
        return fn(*args)
    except Exception as e:  # noqa: BLE001 - reported in the JSON line
        return {"error": f"{type(e).__name__}: {e}"}


def ensemble_run(ks, a, device, barrier, pg, rank):
    """Batched Monte Carlo breakup ensemble: R realisations, each the seeded
    base catalogue plus one collision of a random LEO object (mass U[100, 2000]
    kg) with a projectile of mass U[100, 2000] kg at 10 km/s, fragmented by
    the NASA SBM at L_c = 5 cm (forced impacts through the engine), all resident
    as one batch. Split precision, 5 km screening, fragmentation on in the
    loop, configuration chosen by the engine's autotuner; then W untimed and K
    timed steps with the L2 flushed before each step."""
    R = a.ens_realisations
    st, sz, al = ks.generate_population(realisation_seed(a.seed, rank), a.base)
    n0 = len(sz)
    rng = np.random.default_rng(realisation_seed(a.seed, rank) + 7919)
    leo = np.flatnonzero(np.linalg.norm(st[:, :3], axis=1) - 6378.137 < 2000.0)
    targets = rng.choice(leo, size=R)
    m_target = rng.uniform(100.0, 2000.0, size=R)
    m_proj = rng.uniform(100.0, 2000.0, size=R)
    mass = np.zeros(R * n0)
    mass[np.arange(R) * n0 + targets] = m_target
    eng = ks.Engine(device)
    eng.set_precision(ks.PRECISION_SPLIT)
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
    eng.set_screening(True, a.conj_km, 1.0, 0.01)
    eng.set_population_batch(np.arange(R + 1) * n0, np.tile(st, (R, 1)), np.tile(sz, R), np.tile(al, R))
    eng.set_masses(mass)
    eng.set_breakup(True, a.ens_lc, 40.0, realisation_seed(a.seed, rank))
    for r in range(R):
        eng.impact(r * n0 + int(targets[r]), float(m_proj[r]), 10.0)
    events = eng.take_breakups()
    frags = events["fragments"].astype(np.int64)
    n_total = eng.population_size()
    eng.set_l2_flush(FLUSH_BYTES)
    t0 = time.perf_counter()
    choice = eng.autotune(32)
    tune_s = time.perf_counter() - t0
    eng.set_profiling(True)
    eng.run(a.warmup)
    eng.take_conjunctions()
    eng.take_step_stats()
    barrier()
    eng.run(a.ens_steps)
    barrier()
    tm = eng.timing()
    conj = eng.take_conjunctions()
    more = eng.take_breakups()
    eng.close()
    dev_ms = max_over_ranks(pg, tm["total_ms"] + tm["chunk_ms"])
    obj = sum_over_ranks(pg, float(tm["object_steps"]))
    return {"workload": f"{R} realisations x ({n0} seeded base objects + one SBM collision fragmented at "
                        f"L_c {a.ens_lc} m), one batch, split precision, dt {a.dt} s, {a.conj_km} km",
            "objects": int(n_total), "fragments_per_realisation": {"min": int(frags.min()), "max": int(frags.max()),
                                                                    "mean": float(frags.mean())},
            "value": obj / (dev_ms * 1e-3), "unit": "object-steps/s", "ms_per_step": dev_ms / max(1, tm["steps"]),
            "steps": a.ens_steps, "conjunctions": int(len(conj)), "breakups_in_loop": int(len(more)),
            "autotune": choice, "autotune_s": tune_s,
            "l2": "flushed before every step (256 MiB write)"}


def cascade_run(ks, a, device, barrier, pg, rank, st, sz, al):
    """Batched cascade: R realisations of the 1M-object population with collision
    radii x5 and fragmentation in the loop on the device (NASA SBM, L_c 10 cm,
    counter-based draws, one stream per realisation), split precision, 5 km,
    10 m/s, within a fixed population budget. Every collision fragments inside
    the step that found it, so chunks of steps run through collisions. Timed on
    the device (CUDA events) with the wall time beside it (chunks run by ks_run
    calls, their records taken after each call) and the host's share of it."""
    R = a.cascade_realisations
    n0 = len(sz)
    budget = int(R * n0 * a.cascade_budget)
    eng = ks.Engine(device)
    eng.set_breakup_mode(ks.BREAKUP_DEVICE, budget)
    eng.set_precision(ks.PRECISION_SPLIT)
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
    # Radii x5: a sustained cascade. At x50 the fragments of an event late in a
    # step (radii 2.5-12.5 m there) still overlap at the next step and collide
    # with each other, pairs by the hundred per event, past any per-step limit.
    eng.set_screening(True, a.conj_km, 5.0, 0.01)
    # Each ks_run call below is one chunk, run as one captured graph.
    chunk = timed_chunk(a.cascade_steps, a.steps_per_graph)
    eng.set_steps_per_graph(chunk)
    eng.set_population_batch(np.arange(R + 1) * n0, np.tile(st, (R, 1)), np.tile(sz, R), np.tile(al, R))
    eng.set_breakup(True, 0.10, 40.0, realisation_seed(a.seed, rank))
    eng.run(a.warmup)
    eng.take_conjunctions()
    eng.take_step_stats()
    warm_events = eng.take_breakups()
    n_start = eng.population_size()
    eng.set_profiling(True)
    # A caller streams the records out as the run goes: ks_run over chunks of
    # steps, each chunk's conjunction records taken with the zero-copy take
    # (counted, collisions tallied) and its breakup records and counters taken
    # after each call.
    tm = {k: 0.0 for k in ("total_ms", "chunk_ms", "object_steps", "steps", "host_chunk_ms", "host_prep_ms",
                           "host_launch_ms", "host_sync_ms")}
    n_conj = n_coll = 0
    evs, stats = [], []
    barrier()
    w0 = time.perf_counter()
    prep_calls = []
    for done in range(0, a.cascade_steps, chunk):
        eng.run(min(chunk, a.cascade_steps - done))
        t = eng.timing()
        for k in tm:
            tm[k] += t[k]
        prep_calls.append(round(t["host_prep_ms"], 2))
        while True:
            v = eng.take_conjunctions_view()
            if len(v) == 0:
                break
            n_conj += len(v)
            n_coll += int(v["collision"].sum())
        evs.append(eng.take_breakups())
        stats.append(eng.take_step_stats())
    barrier()
    wall = time.perf_counter() - w0
    ev = np.concatenate(evs)
    stats = np.concatenate(stats)
    n_end = eng.population_size()
    props = eng.objects()
    eng.close()
    frag = props["event"] >= 0
    size = props["size_m"][frag]
    dev_ms = max_over_ranks(pg, tm["total_ms"] + tm["chunk_ms"])
    obj = sum_over_ranks(pg, float(tm["object_steps"]))
    per_real = np.bincount(ev["realisation"], minlength=R) if len(ev) else np.zeros(R, int)
    return {"workload": f"{R} realisations x the {n0}-object population, collision radii x5, fragmentation "
                        f"in the loop on the device (SBM, L_c 0.1 m, counter-based draws), split precision, "
                        f"dt {a.dt} s, {a.conj_km} km, population budget {budget} objects",
            "value": obj / (dev_ms * 1e-3), "unit": "object-steps/s", "ms_per_step": dev_ms / max(1, tm["steps"]),
            "wall_s": wall, "wall_object_steps_per_s": obj / wall, "steps": a.cascade_steps,
            "simulated_hours": a.cascade_steps * a.dt / 3600.0,
            "objects_start": int(n_start), "objects_end": int(n_end), "events": int(len(ev)),
            "warmup_steps": a.warmup, "events_in_warmup": int(len(warm_events)), "catastrophic": int(ev["catastrophic"].sum()) if len(ev) else 0,
            "fragments_created": int(ev["fragments"].sum()) if len(ev) else 0,
            "escaped": int(ev["escaped"].sum()) if len(ev) else 0,
            "events_per_realisation": {"min": int(per_real.min()), "max": int(per_real.max())},
            "collisions": n_coll, "conjunctions": n_conj, "steps_per_call": chunk,
            "host_ms": {"runs": tm["host_chunk_ms"], "prep": tm["host_prep_ms"], "launch": tm["host_launch_ms"],
                        "wait_for_device": tm["host_sync_ms"],
                        "records_and_counters": tm["host_chunk_ms"] - tm["host_prep_ms"] - tm["host_launch_ms"] -
                        tm["host_sync_ms"], "prep_per_call": prep_calls},
            "fragment_sizes_m": {"n_gt_lc": int((size > 0.1).sum()), "ratio_n_gt_2lc": float((size > 0.2).sum() /
                                 max(1, (size > 0.1).sum())), "untruncated_power_law_ratio": 2 ** -1.71,
                                 "note": "SBM sizes are drawn from L^-1.71 truncated to [L_c, parent size] and "
                                         "skipped when the mass budget is spent; most parents here are fragments "
                                         "of 5-50 cm, so the ratio sits below the untruncated law"},
            "alive_end": int(stats["alive"][-1]) if len(stats) else None}


def measure_fp32(eng):
    """Measured FP32 operation rates: add/mul instructions, FMA instructions,
    and FMA lanes of packed FFMA2 instructions, per second."""
    am, fma = eng.measure_fp32()
    return {"addmul": am, "fma": fma, "fma_x2": eng.measure_fp32x2()}


def e2e_run(ks, a, st, sz, al, device, barrier, pg, precision, steps=None):
    """Through the C ABI with host buffers, the way a caller drives a run:
    upload the population from pinned host memory, then ks_run over chunks of
    steps (each chunk one graph launch that uploads every step's lunar rows
    and brings back every step's ordered conjunction records and counters),
    taking each chunk's records and counters as it ends, and finally read the
    population back into pinned host memory. Timed end to end on the host,
    max over ranks."""
    import torch
    steps = steps or a.e2e_steps or a.steps
    chunk = timed_chunk(steps, a.steps_per_graph)
    pin_st = torch.from_numpy(st).pin_memory().numpy()
    pin_sz = torch.from_numpy(sz).pin_memory().numpy()
    pin_al = torch.from_numpy(al).pin_memory().numpy()
    out_st = torch.empty(st.shape, dtype=torch.float64).pin_memory().numpy()
    out_al = torch.empty(al.shape, dtype=torch.uint8).pin_memory().numpy()
    eng = ks.Engine(device)
    eng.set_precision(precision)
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
    eng.set_screening(True, a.conj_km, 1.0, 0.01)
    eng.set_steps_per_graph(chunk)
    # Untimed warm-up on the same population: device buffers reach their
    # working sizes and the chunk graphs are built, as after a run's first chunk.
    eng.set_population(pin_st, pin_sz, pin_al)
    eng.run(min(steps, chunk))
    eng.take_conjunctions()
    eng.take_step_stats()
    eng.prepare_run()
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, a.dt)
    barrier()
    t0 = time.perf_counter()
    eng.set_population(pin_st, pin_sz, pin_al)
    t_up = time.perf_counter()
    nconj = nstats = 0
    last_t = 0.0
    run_s = take_s = 0.0
    host = {"prep_ms": 0.0, "launch_ms": 0.0, "sync_ms": 0.0, "after_ms": 0.0}
    for done in range(0, steps, chunk):
        r0 = time.perf_counter()
        eng.run(min(chunk, steps - done))
        r1 = time.perf_counter()
        tm = eng.timing()
        host["prep_ms"] += tm["host_prep_ms"]
        host["launch_ms"] += tm["host_launch_ms"]
        host["sync_ms"] += tm["host_sync_ms"]
        host["after_ms"] += tm["host_chunk_ms"] - tm["host_prep_ms"] - tm["host_launch_ms"] - tm["host_sync_ms"]
        # Zero-copy takes: the records where the device copied them (pinned
        # host memory), read before the next run reuses that memory.
        while True:
            v = eng.take_conjunctions_view()
            if len(v) == 0:
                break
            nconj += len(v)
            last_t = max(last_t, float(v["t"][-1]))
        nstats += len(eng.take_step_stats())
        run_s += r1 - r0
        take_s += time.perf_counter() - r1
    t_dn = time.perf_counter()
    fs, fa = eng.get_population(out_st, out_al)
    barrier()
    t1 = time.perf_counter()
    wall = max_over_ranks(pg, t1 - t0)
    world = pg.get_world_size() if pg else 1
    obj = float(al.sum()) * steps * world
    eng.close()
    assert nstats == steps
    phases = {"upload_ms": 1e3 * (t_up - t0), "runs_ms": 1e3 * run_s, "takes_ms": 1e3 * take_s,
              "download_ms": 1e3 * (t1 - t_dn), "runs_host_split": host}
    # Per step up: the step's start time, index and 3 lunar stages (position and
    # indirect term), 160 B; down: its 48 B conjunction records and its 216 B
    # control block (the counters).
    h2d = (st.nbytes + sz.nbytes + al.nbytes) / steps + 160
    d2h = (fs.nbytes + fa.nbytes) / steps + nconj * 48 / steps + 216
    return {"value": obj / wall, "unit": "object-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": steps, "steps_per_call": chunk, "phases_ms": phases,
            "what": f"ks_set_population from pinned host memory, then ks_run of {chunk}-step chunks (per step: "
                    "host->device lunar rows, device->host conjunction records in (t, i, j) order and counters, "
                    "taken after each call with the zero-copy take, ks_take_conjunctions_view, from the pinned "
                    "memory the device copied them into), then ks_get_population into pinned host memory; wall "
                    "clock, max over ranks"}


if __name__ == "__main__":
    sys.exit(main())
