"""24 steps of the 1M-object bench workload against the reference build.

The seeded population (seed 20260801: 28 340 catalogue-like objects plus
971 660 fragments in 200 clouds released within the last day), dt 10 s,
5 km threshold, radius scale 1, minimum encounter speed 10 m/s.
tests/golden/ref_1M_24steps.json holds SHA-256 digests of what the
reference's step loop (oracle/_ref, tests/golden/make_golden.py million_kat)
produced on it: final states, every field of every conjunction record and
every per-step counter. The FP64 form reproduces all of them bit for bit; the
split form finds the same pairs up to those within centimetres of the
threshold.
"""
import hashlib
import json

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

CONJ_FIELDS = ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision")
STAT_FIELDS = ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects",
               "alive")


def digest(arrays):
    h = hashlib.sha256()
    for x in arrays:
        h.update(np.ascontiguousarray(x).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def million(ks):
    with open(golden_path("ref_1M_24steps.json")) as f:
        kat = json.load(f)
    p = kat["population"]
    st, sz, al = ks.generate_population(p["seed"], p["n_base"], p["n_total"], p["parents"], p["frag_age_max_s"])
    return kat, st, sz, al


def run(ks, kat, st, sz, al, precision):
    with ks.Engine(0) as eng:
        eng.set_precision(precision)
        eng.set_clock(kat["epoch_jd"], 0.0, kat["dt"])
        eng.set_screening(True, kat["threshold_km"], kat["radius_scale"], kat["min_vrel_km_s"])
        eng.set_population(st, sz, al)
        eng.run(kat["steps"])
        fs, fa = eng.get_population()
        return fs, fa, eng.take_conjunctions(), eng.take_step_stats()


def test_million_fp64_equals_reference(ks, million):
    kat, st, sz, al = million
    fs, fa, conj, stats = run(ks, kat, st, sz, al, ks.PRECISION_FP64)
    assert len(conj) == kat["conjunctions"]
    assert int(conj["collision"].sum()) == kat["collisions"]
    assert int(stats["candidate_pairs"].sum()) == kat["candidate_pairs_total"]
    assert int(stats["refined_pairs"].sum()) == kat["refined_pairs_total"]
    assert digest([stats[f] for f in STAT_FIELDS]) == kat["sha256_step_counters"]
    assert digest([conj[f] for f in CONJ_FIELDS]) == kat["sha256_conjunctions"]
    assert digest([fs, fa]) == kat["sha256_final_states"]


def test_million_split_finds_the_reference_pairs(ks, million):
    kat, st, sz, al = million
    fs, fa, conj, stats = run(ks, kat, st, sz, al, ks.PRECISION_SPLIT)
    # Candidate pairs depend only on cell membership; a position a few
    # millimetres off can move an object across a cell face, so the totals
    # agree to a relative 1e-6, not exactly.
    assert abs(int(stats["candidate_pairs"].sum()) - kat["candidate_pairs_total"]) <= 1e-6 * kat["candidate_pairs_total"]
    assert abs(len(conj) - kat["conjunctions"]) <= 1e-4 * kat["conjunctions"] + 2
    assert int(conj["collision"].sum()) == kat["collisions"]
