"""Pins the CPU oracle (oracle/ks_oracle.c) to the reference.

Two anchors: fixtures produced by the reference itself (tests/golden/, made by
make_golden.py from the reference's own sources) and, where the reference
build is present, live bit-for-bit comparisons on fresh seeded inputs.
"""
import json
import os

import numpy as np
import pytest

from conftest import REFERENCE_TREE, golden_path

CATALOG = os.path.join(REFERENCE_TREE, "data", "satellites_20260801_1000Z.txt")


def load(name):
    return dict(np.load(golden_path(name)))


def run_fixture(checker, fx, steps=None):
    return checker.run(fx["states"], fx["size_m"], fx["alive"], epoch_jd=float(fx["epoch_jd"]), t_start=0.0,
                       dt=float(fx["dt"]), steps=int(fx["steps"] if steps is None else steps), screen=True,
                       threshold_km=float(fx["threshold_km"]), radius_scale=float(fx["radius_scale"]),
                       min_vrel_km_s=float(fx["min_vrel_km_s"]))


@pytest.mark.parametrize("name", ["run_mixed.npz", "run_dense.npz"])
def test_oracle_reproduces_reference_run(oracle, name):
    fx = load(name)
    fs, fa, conj, stats = run_fixture(oracle, fx)
    assert np.array_equal(fs, fx["final_states"]), "final states differ from the reference (bit level)"
    assert np.array_equal(fa, fx["final_alive"])
    assert len(conj) == len(fx["conj"]) and len(conj) > 0
    assert np.array_equal(conj, fx["conj"]), "conjunction records differ"
    assert np.array_equal(stats, fx["stats"]), "per-step counters differ"


def test_oracle_reproduces_reference_screen_cases(oracle):
    fx = load("screen_cases.npz")
    conj, stats = oracle.screen(fx["before"], fx["after"], fx["alive_after"], fx["size_m"], float(fx["t0"]),
                                float(fx["dt"]))
    assert np.array_equal(conj, fx["conj"])
    ref = fx["stats"][0]
    for f in ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects"):
        assert stats[f] == ref[f], f
    assert stats["co_orbiting"] >= 1 and stats["conjunctions"] == 5


def test_fixtures_cover_the_edge_cases():
    mixed = load("run_mixed.npz")
    assert (mixed["final_alive"] == 0).sum() == 2, "planted re-entries"
    dense = load("run_dense.npz")
    assert dense["stats"]["max_cell_objects"].max() > 1000, "a fresh cloud inside one cell"
    sc = load("screen_cases.npz")
    assert sc["conj"]["collision"].sum() == 1
    assert (sc["alive_after"] == 0).sum() == 1


def test_planted_mistake_is_detected(oracle):
    """The comparison is sensitive at the bit level: one ulp on one input
    coordinate (planted here, in the oracle's input) changes the final state."""
    fx = load("run_mixed.npz")
    st = fx["states"].copy()
    st[100, 0] = np.nextafter(st[100, 0], np.inf)
    fs, _, _, _ = oracle.run(st, fx["size_m"], fx["alive"], epoch_jd=float(fx["epoch_jd"]), dt=10.0, steps=5,
                             screen=False)
    fs0, _, _, _ = oracle.run(fx["states"], fx["size_m"], fx["alive"], epoch_jd=float(fx["epoch_jd"]), dt=10.0,
                              steps=5, screen=False)
    assert not np.array_equal(fs[100], fs0[100])
    assert np.array_equal(np.delete(fs, 100, 0), np.delete(fs0, 100, 0))


def test_oracle_catalogue_kat(oracle, reference):
    """1 h on the reference's shipped catalogue: counters from the reference build."""
    if not os.path.exists(CATALOG):
        pytest.skip("shipped catalogue not present")
    with open(golden_path("ref_catalog_1h.json")) as f:
        kat = json.load(f)
    st, sz, ids, epoch = reference.load_catalog(CATALOG)
    fs, fa, conj, stats = oracle.run(st, sz, None, epoch_jd=epoch, dt=10.0, steps=kat["steps"],
                                     threshold_km=kat["threshold_km"])
    assert len(conj) == kat["conjunctions"] == 1493
    assert int(stats["candidate_pairs"].sum()) == kat["candidate_pairs_total"]
    assert int(stats["refined_pairs"].sum()) == kat["refined_pairs_total"]
    k = int(np.argmin(conj["miss_km"]))
    assert conj["miss_km"][k] * 1000.0 == kat["closest"]["miss_m"]
    assert (ids[conj["i"][k]], ids[conj["j"][k]]) == (kat["closest"]["id1"], kat["closest"]["id2"])
    for b, v in kat["below_km"].items():
        assert int((conj["miss_km"] < float(b)).sum()) == v


@pytest.mark.parametrize("seed,age", [(1, 0.0), (2, 1800.0), (3, 86400.0)])
def test_oracle_matches_reference_live(ks, oracle, reference, seed, age):
    st, sz, al = ks.generate_population(seed, 800, 2000, 4, age)
    a = reference.run(st, sz, al, steps=15, threads=4)
    b = oracle.run(st, sz, al, steps=15)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_elementary_functions_match_reference(oracle, reference):
    rng = np.random.default_rng(3)
    for jd in 2461253.9 + rng.random(50) * 400.0:
        assert np.array_equal(oracle.moon_position(jd), reference.moon_position(jd))
    for _ in range(200):
        r = rng.normal(size=3)
        r *= (6600 + 40000 * rng.random()) / np.linalg.norm(r)
        s = np.concatenate([r, rng.normal(size=3) * 4.0])
        m = [rng.normal(size=3) * 384000.0 for _ in range(3)]
        dt = float(rng.choice([1.0, 10.0, 30.0, -10.0]))
        assert np.array_equal(oracle.rk4(s, dt, *m), reference.rk4(s, dt, *m))


def test_filter_edge_cases_match_reference(oracle, reference):
    rng = np.random.default_rng(4)
    cases = [((0, 0, 0), (0, 0, 0)), ((1.0, 0, 0), (0, 0, 0)), ((3.0, 0, 0), (-0.3, 0, 0)),
             ((3.0, 0, 0), (0.3, 0, 0)), ((0.0, 4.9, 0), (1e-3, 0, 0)), ((0, 0, 5.0009), (0, 0, 0)),
             ((0, 0, 5.0011), (0, 0, 0)), ((100.0, 0, 0), (-10.0, 0, 0)), ((-0.0, 0.0, 0.0), (-0.0, 0.0, 0.0))]
    for _ in range(2000):
        dr = rng.normal(size=3) * rng.choice([0.01, 1.0, 10.0, 300.0])
        dv = rng.normal(size=3) * rng.choice([1e-4, 0.01, 1.0, 10.0])
        cases.append((dr, dv))
    for dr, dv in cases:
        for dt in (10.0, 60.0):
            assert oracle.filter_pair(dr, dv, dt, 5.0, 1e-4) == reference.filter_pair(dr, dv, dt, 5.0, 1e-4)
            assert oracle.prefilter_keep(dr, dv, dt, 5.0, 1e-4) == reference.prefilter_keep(dr, dv, dt, 5.0, 1e-4)
