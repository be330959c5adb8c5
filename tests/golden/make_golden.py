"""Generates the golden fixtures of tests/golden/ from the REFERENCE ITSELF.

Runs oracle/_ref/libksref.so (the reference's own src/core/orbital.cpp and
src/core/collision.cpp compiled in place by oracle/Makefile, driven like its
CLI step loop) and stores inputs and outputs, so that the tests can check the
oracle and the engine without the reference tree.

    python tests/golden/make_golden.py        # needs the reference tree

Fixtures:
  run_mixed.npz      1 500 catalogue objects + 1 500 fragments in 3 clouds
                     (released up to 2 h before the epoch), two planted
                     re-entries (one of them the fastest object, which forces
                     the grid to be rebuilt without it), 40 steps
  run_dense.npz      600 objects + 2 400 fragments in 2 clouds released at the
                     epoch: every cloud starts inside one cell, 12 steps
  screen_cases.npz   planted one-step encounters: crossing, co-orbiting,
                     separating, TCA at a step edge, collision, dead object
  ref_catalog_1h.json  counters of a 1 h run on the reference's shipped
                     catalogue (the README's own data), for the oracle
  cli_catalog.txt    a 2 500-object synthetic catalogue in the reference's
                     pipe format (with planted encounters), and
  cli_ref_*.csv      the conjunctions.csv / final_state.csv the reference CLI
                     (oracle/_ref/kessler_sim) writes for it over 15 minutes
  run_breakup.npz    the CLI loop with --breakup through the reference's
                     Fragmentation (planted collisions, a forced impact),
                     every object's final state and properties, events
  cli_snapshot_ref.json  SHA-256 of the reference CLI's periodic snapshots and
                     of its trajectories.csv / moon.csv for tracked ids
  cli_breakup_*      a 2 000-object catalogue of mixed object types and the
                     four files the reference CLI writes for it with --breakup
                     and --impact over 1.2 h
"""
import importlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import checkers  # noqa: E402

EPOCH = 2461253.916666667
CATALOG = os.path.join(checkers.REFERENCE_TREE, "data", "satellites_20260801_1000Z.txt")


def population(seed, n_base, n_total, n_parents, age):
    ks = importlib.import_module("kessler-syndrom-simulation_b200")
    return ks.generate_population(seed, n_base, n_total, n_parents, age)


def _accel(r):
    # Two-body + J2, only to plant encounters (the reference adds the Moon).
    mu, re, j2 = 398600.4418, 6378.137, 1.08262668e-3
    r2 = (r * r).sum()
    rn = np.sqrt(r2)
    a = -mu * r / (r2 * rn)
    k = 1.5 * j2 * mu * re * re / (r2 * r2 * rn)
    z2 = 5.0 * r[2] ** 2 / r2
    return a + k * r * np.array([z2 - 1.0, z2 - 1.0, z2 - 3.0])


def _propagate(s, t, h=1.0):
    s = np.array(s, float)
    n = int(round(abs(t) / h))
    h = t / n
    for _ in range(n):
        f = lambda y: np.concatenate([y[3:], _accel(y[:3])])
        k1 = f(s); k2 = f(s + k1 * h / 2); k3 = f(s + k2 * h / 2); k4 = f(s + k3 * h)
        s = s + (k1 + 2 * k2 + 2 * k3 + k4) * h / 6
    return s


def plant_encounters(st, first, count, steps, dt, seed):
    """Pairs (first + 2k, first + 2k + 1) that meet about mid-run: the same
    point with velocities rotated about the radius, carried back in time."""
    rng = np.random.default_rng(seed)
    for k in range(count):
        a = st[first + 2 * k].copy()
        r = a[:3]
        u = r / np.linalg.norm(r)
        ang = np.radians(20 + 140 * rng.random())
        v = a[3:]
        vb = v * np.cos(ang) + np.cross(u, v) * np.sin(ang) + u * np.dot(u, v) * (1 - np.cos(ang))
        off = rng.normal(size=3)
        off -= np.dot(off, vb) * vb / np.dot(vb, vb)
        off *= (0.05 + 3.0 * rng.random()) / np.linalg.norm(off)
        t_meet = (steps * (0.2 + 0.6 * rng.random()) + rng.random()) * dt
        st[first + 2 * k] = _propagate(a, -t_meet)
        st[first + 2 * k + 1] = _propagate(np.concatenate([r + off, vb]), -t_meet)


def plant_reentries(st, al):
    # Object 0: falling through the surface during step 0 at 15 km/s, the
    # fastest object of the population. Object 1: slower, dies a few steps later.
    st[0] = [6390.0, 0.0, 0.0, -15.0, 0.3, 0.0]
    st[1] = [0.0, 6700.0, 0.0, 0.0, -4.0, 1.0]


def save_run(name, st, sz, al, steps, dt=10.0, thr=5.0, rscale=1.0, vmin=0.01):
    ref = checkers.Reference()
    fs, fa, conj, stats = ref.run(st, sz, al, epoch_jd=EPOCH, t_start=0.0, dt=dt, steps=steps, screen=True,
                                  threshold_km=thr, radius_scale=rscale, min_vrel_km_s=vmin, threads=8)
    np.savez_compressed(os.path.join(HERE, name), states=st, size_m=sz, alive=al, epoch_jd=EPOCH, dt=dt,
                        steps=steps, threshold_km=thr, radius_scale=rscale, min_vrel_km_s=vmin,
                        final_states=fs, final_alive=fa, conj=conj, stats=stats)
    print(name, "conj", len(conj), "candidates/step", int(stats["candidate_pairs"].mean()),
          "dead", int((fa == 0).sum()))


def breakup_run(name="run_breakup.npz", steps=40, rscale=300.0, lc=0.1, seed=7):
    """The CLI loop with --breakup: planted encounters that end in collisions,
    a forced impact at step 3, the fragments screened from the next step on."""
    st, sz, al = population(4242, 1500, 2500, 3, 1800.0)
    plant_encounters(st, 100, 16, steps, 10.0, 17)
    rng = np.random.default_rng(9)
    mass = np.where(rng.random(len(sz)) < 0.5, 0.0, rng.uniform(1.0, 2000.0, len(sz)))
    mass[116], mass[117] = 0.5, 2000.0  # a cratering (non-catastrophic) collision
    impact = (50, 300.0, 10.0, 3)
    ref = checkers.Reference()
    out = ref.run_breakup(st, sz, mass, al, epoch_jd=EPOCH, dt=10.0, steps=steps, threshold_km=5.0,
                          radius_scale=rscale, min_vrel_km_s=0.01, threads=8, lc_m=lc, seed=seed, impact=impact)
    np.savez_compressed(os.path.join(HERE, name), states=st, size_m=sz, alive=al, mass_kg=mass, epoch_jd=EPOCH,
                        dt=10.0, steps=steps, threshold_km=5.0, radius_scale=rscale, min_vrel_km_s=0.01, lc_m=lc,
                        seed=seed, impact=np.array(impact), **{"out_" + k: v for k, v in out.items()})
    ev = out["events"]
    print(name, "objects", len(out["size_m"]), "events", len(ev), "catastrophic", int(ev["catastrophic"].sum()),
          "fragments", int(ev["fragments"].sum()), "conj", len(out["conj"]), "collisions",
          int(out["conj"]["collision"].sum()))


def screen_cases():
    """Hand-built before/after pairs for one Screener::screen call (dt = 10 s)."""
    dt = 10.0
    rng = np.random.default_rng(5)
    before, after, size = [], [], []

    def add(b, a, s=1.0):
        before.append(b)
        after.append(a)
        size.append(s)

    def straight(r, v):
        r = np.asarray(r, float)
        v = np.asarray(v, float)
        return list(r) + list(v), list(r + v * dt) + list(v)

    # Background objects far apart.
    for k in range(200):
        r = rng.normal(size=3)
        r = r / np.linalg.norm(r) * (7000 + 400 * rng.random())
        v = np.cross(r, [0, 0, 1.0])
        v = v / np.linalg.norm(v) * 7.5
        add(*straight(r, v))
    # 1. Crossings, TCA inside the step, misses from 50 m to just over 5 km.
    for k, miss in enumerate([0.05, 0.8, 2.5, 4.99, 5.02]):
        frac = 0.15 + 0.17 * k
        y = 7000.0 + 40.0 * k
        add(*straight([y, 0, 1000.0 * k], [0, 7.5, 0]))
        add(*straight([y, -3.5 * dt * frac, 1000.0 * k + miss], [0, 11.0, 0]))
    # 2. Co-orbiting pair 300 m apart, 2 m/s relative.
    add(*straight([0, 7100, 0], [-7.4, 0, 0]))
    add(*straight([0, 7100.3, 0], [-7.402, 0, 0]))
    # 3. Separating pair (closest at the start of the step).
    add(*straight([0, 0, 7200], [7.3, 0, 0]))
    add(*straight([0.5, 0, 7200], [7.3 + 3.0, 0, 0]))
    # 4. TCA at the very end of the step: approaching until t0 + dt.
    add(*straight([-7300, 0, 0], [0, 0, 7.3]))
    add(*straight([-7300, 0, -50.0], [0, 0, 12.3]))
    # 5. Collision: miss below the radius sum (sizes 30 m -> radius 15 m each).
    add(*straight([5000, 5000, 0], [0, 0, 7.0]), 30.0)
    add(*straight([5000.01, 4990.0, 35.0], [0, 2.0, 0.0]), 30.0)
    # 6. A close pair whose second object is dead after the step.
    add(*straight([-5000, -5000, 100], [0, 0, 7.0]))
    add(*straight([-5000, -5000.5, 130.0], [0, 0, 4.0]))
    b = np.array(before)
    a = np.array(after)
    alive = np.ones(len(b), np.uint8)
    alive[-1] = 0
    sz = np.array(size)
    ref = checkers.Reference()
    conj, stats = ref.screen(b, a, alive, sz, 1234.0, dt, threads=1)
    np.savez_compressed(os.path.join(HERE, "screen_cases.npz"), before=b, after=a, alive_after=alive, size_m=sz,
                        t0=1234.0, dt=dt, threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, conj=conj,
                        stats=np.array([stats]))
    print("screen_cases conj", len(conj), conj[["i", "j", "miss_km", "collision"]])


def catalogue_kat():
    ref = checkers.Reference()
    st, sz, ids, epoch = ref.load_catalog(CATALOG)
    fs, fa, conj, stats = ref.run(st, sz, None, epoch_jd=epoch, t_start=0.0, dt=10.0, steps=360, screen=True,
                                  threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, threads=8)
    k = int(np.argmin(conj["miss_km"]))
    out = {
        "source": "reference CLI step loop (oracle/_ref) on data/satellites_20260801_1000Z.txt",
        "objects": int(len(st)), "epoch_jd": epoch, "dt": 10.0, "steps": 360, "threshold_km": 5.0,
        "conjunctions": int(len(conj)),
        "below_km": {str(b): int((conj["miss_km"] < b).sum()) for b in (0.1, 1.0, 2.0, 5.0)},
        "collisions": int(conj["collision"].sum()),
        "closest": {"miss_m": float(conj["miss_km"][k] * 1000.0), "t_h": float(conj["t"][k] / 3600.0),
                    "id1": int(ids[conj["i"][k]]), "id2": int(ids[conj["j"][k]])},
        "candidate_pairs_total": int(stats["candidate_pairs"].sum()),
        "refined_pairs_total": int(stats["refined_pairs"].sum()),
        "max_co_orbiting": int(stats["co_orbiting"].max()),
        "final_state_sha_hint": float(np.abs(fs).sum()),
        "readme_24h": {"conjunctions": 38367, "below_1km": 1493, "below_100m": 14, "collisions": 0,
                       "closest_m": 7.2},
    }
    with open(os.path.join(HERE, "ref_catalog_1h.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("catalogue 1h", out["conjunctions"], out["closest"])


CONJ_FIELDS = ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision")
STAT_FIELDS = ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects",
               "alive")


def digest(arrays):
    """SHA-256 over the raw bytes of each array in turn (C order)."""
    import hashlib
    h = hashlib.sha256()
    for x in arrays:
        h.update(np.ascontiguousarray(x).tobytes())
    return h.hexdigest()


def catalogue_24h_kat():
    """24 h of the shipped catalogue (8 640 steps of 10 s, --conj-km 5): the
    README's own run. The reference's inputs (states, sizes and NORAD ids as
    its loader reads them) are kept as catalog_28340.npz so the check runs
    without the reference tree; its outputs are kept as SHA-256 digests of the
    final states, of every conjunction record field and of every per-step
    counter, plus the summary the README quotes."""
    ref = checkers.Reference()
    st, sz, ids, epoch = ref.load_catalog(CATALOG)
    np.savez_compressed(os.path.join(HERE, "catalog_28340.npz"), states=st, size_m=sz, ids=ids.astype(np.int32),
                        epoch_jd=epoch)
    steps = 8640
    fs, fa, conj, stats = ref.run(st, sz, None, epoch_jd=epoch, t_start=0.0, dt=10.0, steps=steps, screen=True,
                                  threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, threads=os.cpu_count())
    ps, pa, _, _ = ref.run(st, sz, None, epoch_jd=epoch, t_start=0.0, dt=10.0, steps=steps, screen=False,
                           threads=os.cpu_count())
    assert np.array_equal(ps, fs) and np.array_equal(pa, fa), "screening changed the states"
    k = int(np.argmin(conj["miss_km"]))
    out = {
        "source": "reference CLI step loop (oracle/_ref) on data/satellites_20260801_1000Z.txt, 24 h",
        "objects": int(len(st)), "epoch_jd": epoch, "dt": 10.0, "steps": steps, "threshold_km": 5.0,
        "radius_scale": 1.0, "min_vrel_km_s": 0.01,
        "conjunctions": int(len(conj)),
        "below_km": {str(b): int((conj["miss_km"] < b).sum()) for b in (0.1, 1.0, 5.0)},
        "collisions": int(conj["collision"].sum()),
        "closest": {"miss_m": float(conj["miss_km"][k] * 1000.0), "t_h": float(conj["t"][k] / 3600.0),
                    "id1": int(ids[conj["i"][k]]), "id2": int(ids[conj["j"][k]])},
        "alive_end": int(fa.sum()),
        "sha256_final_states": digest([fs, fa]),
        "sha256_conjunctions": digest([conj[f] for f in CONJ_FIELDS]),
        "sha256_step_counters": digest([stats[f] for f in STAT_FIELDS]),
        "readme": {"conjunctions": 38367, "below_1km": 1493, "below_100m": 14, "collisions": 0,
                   "closest_m": 7.2, "where": "README.md:179-186"},
    }
    with open(os.path.join(HERE, "ref_catalog_24h.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("catalogue 24h", out["conjunctions"], out["below_km"], out["closest"])


def million_kat(steps=24):
    """The bench workload (seed 20260801: 28 340 catalogue objects + 971 660
    fragments in 200 clouds released within the last day), dt 10 s, 5 km, run
    by the reference build for `steps` steps: SHA-256 digests of its final
    states, conjunction records and per-step counters. The population is the
    seeded generator's, so only the digests are kept."""
    st, sz, al = checkers.generate_population(20260801, 28340, 1_000_000, 200, 86400.0)
    ref = checkers.Reference()
    fs, fa, conj, stats = ref.run(st, sz, al, epoch_jd=EPOCH, t_start=0.0, dt=10.0, steps=steps, screen=True,
                                  threshold_km=5.0, radius_scale=1.0, min_vrel_km_s=0.01, threads=os.cpu_count())
    out = {
        "source": "reference CLI step loop (oracle/_ref) on the seeded 1M-object bench population",
        "population": {"seed": 20260801, "n_base": 28340, "n_total": 1000000, "parents": 200,
                       "frag_age_max_s": 86400.0},
        "epoch_jd": EPOCH, "dt": 10.0, "steps": steps, "threshold_km": 5.0, "radius_scale": 1.0,
        "min_vrel_km_s": 0.01,
        "conjunctions": int(len(conj)), "collisions": int(conj["collision"].sum()),
        "candidate_pairs_total": int(stats["candidate_pairs"].sum()),
        "refined_pairs_total": int(stats["refined_pairs"].sum()),
        "sha256_final_states": digest([fs, fa]),
        "sha256_conjunctions": digest([conj[f] for f in CONJ_FIELDS]),
        "sha256_step_counters": digest([stats[f] for f in STAT_FIELDS]),
    }
    with open(os.path.join(HERE, "ref_1M_24steps.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("1M kat", out["conjunctions"], out["candidate_pairs_total"])


CLI_ARGS = ["0.25", "10", "--conj-km", "5"]


def cli_golden():
    ks = importlib.import_module("kessler-syndrom-simulation_b200")
    cio = importlib.import_module("kessler-syndrom-simulation_b200.catalog_io")
    st, sz, al = ks.generate_population(99, 1500, 2500, 3, 1800.0)
    plant_encounters(st, 0, 20, 90, 10.0, 13)
    cat = os.path.join(HERE, "cli_catalog.txt")
    cio.write_catalog(cat, st, ids=np.arange(100001, 100001 + len(st)), rcs=cio.rcs_class_for_size(sz))
    exe = os.path.join(ROOT, "oracle", "_ref", "kessler_sim")
    with tempfile.TemporaryDirectory() as tmp:
        out = subprocess.run([exe, cat] + CLI_ARGS + ["--threads", "8"], cwd=tmp, capture_output=True, text=True,
                             check=True)
        shutil.copy(os.path.join(tmp, "output", "conjunctions.csv"), os.path.join(HERE, "cli_ref_conjunctions.csv"))
        shutil.copy(os.path.join(tmp, "output", "final_state.csv"), os.path.join(HERE, "cli_ref_final_state.csv"))
    n = sum(1 for _ in open(os.path.join(HERE, "cli_ref_conjunctions.csv"))) - 1
    print("cli golden: conjunctions", n)


CLI_BREAKUP_ARGS = ["1.2", "10", "--breakup", "--radius-scale", "500", "--lc", "0.1", "--seed", "3",
                    "--impact", "100051", "--impact-mass", "500", "--impact-vrel", "10", "--impact-at", "0.05"]


def cli_breakup_golden():
    """The reference CLI with --breakup and --impact on a catalogue of mixed
    object types (catalogue masses from the default mass table)."""
    ks = importlib.import_module("kessler-syndrom-simulation_b200")
    cio = importlib.import_module("kessler-syndrom-simulation_b200.catalog_io")
    st, sz, al = ks.generate_population(77, 1500, 2000, 2, 3600.0)
    plant_encounters(st, 100, 30, 432, 10.0, 29)
    rng = np.random.default_rng(31)
    rcs = cio.rcs_class_for_size(sz)
    rcs[100:160] = np.where(rng.random(60) < 0.5, "LARGE", "MEDIUM")
    types = np.where(rng.random(len(sz)) < 0.3, "PAYLOAD", np.where(rng.random(len(sz)) < 0.15, "ROCKET BODY",
                                                                     "DEBRIS"))
    types[50] = "PAYLOAD"
    rcs[50] = "LARGE"
    cat = os.path.join(HERE, "cli_breakup_catalog.txt")
    cio.write_catalog(cat, st, ids=np.arange(100001, 100001 + len(st)), rcs=rcs, types=types)
    exe = os.path.join(ROOT, "oracle", "_ref", "kessler_sim")
    with tempfile.TemporaryDirectory() as tmp:
        out = subprocess.run([exe, cat] + CLI_BREAKUP_ARGS + ["--threads", "8"], cwd=tmp, capture_output=True,
                             text=True, check=True)
        for name in ("conjunctions.csv", "final_state.csv", "breakups.csv", "population.csv"):
            shutil.copy(os.path.join(tmp, "output", name), os.path.join(HERE, "cli_breakup_ref_" + name))
    print("cli breakup golden:", open(os.path.join(HERE, "cli_breakup_ref_breakups.csv")).read().count("\n") - 1,
          "events,", open(os.path.join(HERE, "cli_breakup_ref_conjunctions.csv")).read().count("\n") - 1,
          "conjunctions")


CLI_SNAPSHOT_RUNS = {
    "snapshots": ["0.25", "10", "300", "--conj-km", "5"],
    "tracks": ["0.25", "10", "120", "100001,100007,100050,100399", "--conj-km", "5"],
}


def cli_snapshot_golden():
    """SHA-256 of the files the reference CLI writes with periodic snapshots
    (positional out_every) and with tracked ids (trajectories.csv, moon.csv)
    for cli_catalog.txt; the files themselves are not kept."""
    import hashlib
    cat = os.path.join(HERE, "cli_catalog.txt")
    exe = os.path.join(ROOT, "oracle", "_ref", "kessler_sim")
    out = {}
    for name, args in CLI_SNAPSHOT_RUNS.items():
        with tempfile.TemporaryDirectory() as tmp:
            subprocess.run([exe, cat] + args + ["--threads", "8"], cwd=tmp, capture_output=True, text=True,
                           check=True)
            files = sorted(f for f in os.listdir(os.path.join(tmp, "output"))
                           if f.startswith(("snapshot_", "trajectories", "moon")))
            out[name] = {"args": args, "sha256": {f: hashlib.sha256(open(os.path.join(tmp, "output", f), "rb").read())
                                                  .hexdigest() for f in files}}
    with open(os.path.join(HERE, "cli_snapshot_ref.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("cli snapshot golden:", {k: sorted(v["sha256"]) for k, v in out.items()})


def main():
    checkers.build(ref=True)
    if len(sys.argv) > 1:  # regenerate only the named fixtures, e.g. catalogue_24h_kat
        for name in sys.argv[1:]:
            globals()[name]()
        return
    st, sz, al = population(20260801, 1500, 3000, 3, 7200.0)
    plant_reentries(st, al)
    plant_encounters(st, 2, 12, 40, 10.0, 11)
    save_run("run_mixed.npz", st, sz, al, 40)
    st, sz, al = population(7, 600, 3000, 2, 0.0)
    plant_encounters(st, 0, 8, 12, 10.0, 12)
    save_run("run_dense.npz", st, sz, al, 12)
    screen_cases()
    cli_golden()
    cli_breakup_golden()
    cli_snapshot_golden()
    breakup_run()
    if os.path.exists(CATALOG):
        catalogue_kat()
        catalogue_24h_kat()
    million_kat()


if __name__ == "__main__":
    main()
