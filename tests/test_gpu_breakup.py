"""In-loop NASA SBM fragmentation on the engine against the reference's CLI loop.

tests/golden/run_breakup.npz was written by the reference itself
(oracle/_ref/libksref.so: Screener + Simulation::step + Fragmentation::apply,
with a forced Fragmentation::impact at the start of step 3): planted encounters
end in collisions (catastrophic and cratering), and the fragments join the
population. Bar: bit-exact final states, alive flags and per-object
properties (size, mass, area-to-mass, originating event) of every object,
fragments included; identical conjunction records, breakup events and per-step
counters — for any chunking of the run into graphs.
"""
import numpy as np
import pytest

from conftest import golden_path
from test_gpu_parity import STAT_FIELDS, assert_same_conj

pytestmark = pytest.mark.gpu

EVENT_FIELDS = ("step", "t", "id", "target", "projectile", "catastrophic", "fragments", "escaped", "first_fragment",
                "v_rel_km_s", "energy_j_per_g", "target_mass_kg", "projectile_mass_kg", "sbm_mass_kg",
                "expected_fragments", "fragments_mass_kg", "position")


def load():
    return dict(np.load(golden_path("run_breakup.npz")))


def run_with_breakup(eng, fx, spg, seed=None, precision=None):
    eng.set_steps_per_graph(spg)
    eng.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
    eng.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
    eng.set_population(fx["states"], fx["size_m"], fx["alive"])
    eng.set_masses(fx["mass_kg"])
    eng.set_breakup(True, float(fx["lc_m"]), 40.0, int(fx["seed"] if seed is None else seed))
    idx, mass, vrel, step = fx["impact"]
    steps = int(fx["steps"])
    eng.run(int(step))
    eng.impact(int(idx), float(mass), float(vrel))
    eng.run(steps - int(step))
    fs, fa = eng.get_population()
    out = dict(states=fs, alive=fa, conj=eng.take_conjunctions(), events=eng.take_breakups(),
               stats=eng.take_step_stats(), **eng.objects())
    eng.set_breakup(False)
    return out


@pytest.mark.parametrize("spg", [0, 7, 32])
def test_breakup_run_equals_reference(engine, spg):
    fx = load()
    got = run_with_breakup(engine, fx, spg)
    assert len(got["states"]) == len(fx["out_states"]) > len(fx["states"])
    assert np.array_equal(got["states"], fx["out_states"]), "states differ from the reference (bit level)"
    assert np.array_equal(got["alive"], fx["out_alive"])
    for k in ("size_m", "mass_kg", "area_to_mass", "event"):
        assert np.array_equal(got[k], fx["out_" + k]), k
    assert_same_conj(got["conj"], fx["out_conj"])
    ev, want = got["events"], fx["out_events"]
    assert len(ev) == len(want) >= 4
    for f in EVENT_FIELDS:
        assert np.array_equal(ev[f], want[f]), f
    for f in STAT_FIELDS:
        assert np.array_equal(got["stats"][f], fx["out_stats"][f]), f


def test_breakup_in_a_batch_equals_separate_runs(engine):
    # Two realisations of the same population: realisation r draws with seed + r.
    fx = load()
    seed = int(fx["seed"])
    singles = [run_with_breakup(engine, fx, 16, seed=seed + r) for r in range(2)]
    n0 = len(fx["states"])
    engine.set_steps_per_graph(16)
    engine.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
    engine.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
    engine.set_population_batch([0, n0, 2 * n0], np.concatenate([fx["states"]] * 2),
                                np.concatenate([fx["size_m"]] * 2), np.concatenate([fx["alive"]] * 2))
    engine.set_masses(np.concatenate([fx["mass_kg"]] * 2))
    engine.set_breakup(True, float(fx["lc_m"]), 40.0, seed)
    idx, mass, vrel, step = fx["impact"]
    engine.run(int(step))
    for r in range(2):
        engine.impact(int(idx) + r * n0, float(mass), float(vrel))
    engine.run(int(fx["steps"]) - int(step))
    fs, fa = engine.get_population()
    conj, events, props = engine.take_conjunctions(), engine.take_breakups(), engine.objects()
    engine.set_breakup(False)
    for r, one in enumerate(singles):
        rows = np.flatnonzero(props["realisation"] == r)
        local = np.full(len(fs), -1)
        local[rows] = np.arange(len(rows))
        assert np.array_equal(fs[rows], one["states"]), r
        assert np.array_equal(fa[rows], one["alive"]), r
        assert np.array_equal(props["event"][rows], one["event"]), r
        c = conj[conj["realisation"] == r].copy()
        c["i"], c["j"] = local[c["i"]], local[c["j"]]
        assert_same_conj(c, one["conj"])
        e = events[events["realisation"] == r]
        for f in ("step", "t", "id", "catastrophic", "fragments", "escaped", "sbm_mass_kg", "fragments_mass_kg"):
            assert np.array_equal(e[f], one["events"][f]), (r, f)


def test_breakup_off_leaves_collisions_alone(engine, oracle):
    fx = load()
    engine.set_steps_per_graph(32)
    engine.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
    engine.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
    engine.set_population(fx["states"], fx["size_m"], fx["alive"])
    engine.set_breakup(False)
    engine.run(20)
    conj = engine.take_conjunctions()
    want = oracle.run(fx["states"], fx["size_m"], fx["alive"], steps=20, threshold_km=float(fx["threshold_km"]),
                      radius_scale=float(fx["radius_scale"]))
    assert_same_conj(conj, want[2])
    assert conj["collision"].sum() > 0 and len(engine.take_breakups()) == 0
    assert engine.get_population()[0].shape[0] == len(fx["states"])


def test_population_file_resumes_the_run_exactly(engine, ks, tmp_path):
    # Save after 13 steps (fragments of the forced impact and of a planted
    # collision already in), resume in a fresh context, finish the 40 steps:
    # the same final population, properties and later events as the reference's
    # uninterrupted run.
    fx = load()
    engine.set_steps_per_graph(16)
    engine.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
    engine.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
    engine.set_population(fx["states"], fx["size_m"], fx["alive"])
    engine.set_masses(fx["mass_kg"])
    engine.set_breakup(True, float(fx["lc_m"]), 40.0, int(fx["seed"]))
    idx, mass, vrel, step = fx["impact"]
    engine.run(int(step))
    engine.impact(int(idx), float(mass), float(vrel))
    engine.run(13 - int(step))
    first = engine.take_breakups()
    engine.take_conjunctions()
    engine.take_step_stats()
    path = tmp_path / "mid.kspop"
    engine.save_population(path)
    engine.set_breakup(False)
    other = ks.Engine(0)
    try:
        other.set_steps_per_graph(7)
        other.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
        other.load_population(path)
        assert other.clock() == engine.clock()
        other.run(int(fx["steps"]) - 13)
        fs, fa = other.get_population()
        props = other.objects()
        events = np.concatenate([first, other.take_breakups()])
    finally:
        other.close()
    assert np.array_equal(fs, fx["out_states"]) and np.array_equal(fa, fx["out_alive"])
    for k in ("size_m", "mass_kg", "area_to_mass", "event"):
        assert np.array_equal(props[k], fx["out_" + k]), k
    for f in EVENT_FIELDS:
        assert np.array_equal(events[f], fx["out_events"][f]), f


def test_population_file_rejects_other_files(engine, tmp_path):
    bad = tmp_path / "bad.kspop"
    bad.write_bytes(b"not a population file")
    with pytest.raises(Exception):
        engine.load_population(bad)
