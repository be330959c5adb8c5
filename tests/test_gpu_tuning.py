"""The autotuner: it changes launch shapes only, never results.

After ks_autotune the resident simulation is where it was (clock, step count,
population), and a run gives the oracle's states, conjunctions and counters
bit for bit (candidate counts and the cell edge excepted when it chose a
larger cell).
"""
import numpy as np
import pytest

from test_gpu_parity import assert_same_conj, run_engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_autotune_keeps_results(engine, oracle, ks, precision):
    st, sz, al = ks.generate_population(501, 6000, 40000, 10, 1800.0)
    engine.set_precision(ks.PRECISION_SPLIT if precision == "split" else ks.PRECISION_FP64)
    engine.set_steps_per_graph(32)
    engine.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
    engine.set_screening(True, 5.0, 1.0, 0.01)
    engine.set_population(st, sz, al)
    try:
        choice = engine.autotune(8)
        assert choice["trials"] >= 10
        assert choice["ms_per_step_best"] <= choice["ms_per_step_start"] * 1.1
        assert choice["steps_per_graph"] in (8, 16, 32, 64)
        assert engine.clock() == (0.0, 0)
        fs0, fa0 = engine.get_population()
        assert np.array_equal(fs0, st) and np.array_equal(fa0, al)
        assert len(engine.take_conjunctions()) == 0 and len(engine.take_step_stats()) == 0
        engine.run(6)
        fs, fa = engine.get_population()
        conj, stats = engine.take_conjunctions(), engine.take_step_stats()
        if precision == "fp64":
            want = oracle.run(st, sz, al, steps=6)
            assert np.array_equal(fs, want[0]) and np.array_equal(fa, want[1])
            assert_same_conj(conj, want[2])
            for f in ("refined_pairs", "co_orbiting", "conjunctions", "alive"):
                assert np.array_equal(stats[f], want[3][f]), f
        else:
            # the same split run with the default configuration
            for key, val in (("pair_variant", 2), ("pair_blocks_per_sm", 0), ("subcell_bits", 1),
                             ("box_min_rows", 4), ("cell_scale_permille", 1000), ("prop_block", 128)):
                engine.set_tuning(key, val)
            engine.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
            engine.set_population(st, sz, al)
            engine.run(6)
            f2, a2 = engine.get_population()
            d = np.abs(fs - f2).max(axis=1)
            assert np.array_equal(fs, f2), (choice, int((d > 0).sum()), float(d.max()), np.flatnonzero(d > 0)[:10])
            assert np.array_equal(fa, a2)
            assert_same_conj(conj, engine.take_conjunctions())
            engine.take_step_stats()
    finally:
        for key, val in (("pair_variant", 2), ("pair_blocks_per_sm", 0), ("subcell_bits", 1), ("box_min_rows", 4),
                         ("cell_scale_permille", 1000), ("prop_block", 128)):
            engine.set_tuning(key, val)
        engine.set_steps_per_graph(32)
        engine.set_precision(ks.PRECISION_FP64)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_unpacked_sort_keys_give_the_same_results(engine, oracle, ks, precision):
    # Sort keys without the packed object index (the path taken when cell keys
    # are too wide to leave room for it) against the default packed keys.
    st, sz, al = ks.generate_population(502, 5000, 30000, 8, 3600.0)
    prec = ks.PRECISION_SPLIT if precision == "split" else ks.PRECISION_FP64

    def run(pack):
        engine.set_tuning("pack_keys", pack)
        engine.set_precision(prec)
        engine.set_steps_per_graph(16)
        engine.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
        engine.set_screening(True, 5.0, 1.0, 0.01)
        engine.set_population(st, sz, al)
        engine.run(20)
        return engine.get_population(), engine.take_conjunctions(), engine.take_step_stats()

    try:
        packed, unpacked = run(1), run(0)
    finally:
        engine.set_tuning("pack_keys", 1)
        engine.set_precision(ks.PRECISION_FP64)
    assert np.array_equal(packed[0][0], unpacked[0][0]) and np.array_equal(packed[0][1], unpacked[0][1])
    assert_same_conj(packed[1], unpacked[1])
    for f in ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects"):
        assert np.array_equal(packed[2][f], unpacked[2][f]), f
    if precision == "fp64":
        want = oracle.run(st, sz, al, steps=20)
        assert np.array_equal(unpacked[0][0], want[0])
        assert_same_conj(unpacked[1], want[2])


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_fp64_pair_variants_equal_the_oracle(engine, oracle, ks, variant):
    # FP64 precision with each pair kernel: FP64 gate (two columns or one per
    # lane) or the FP32 gate on cell-relative records; the exact FP64 filter
    # decides in every case, so states, conjunctions and counters are the
    # reference's bit for bit.
    st, sz, al = ks.generate_population(503, 5000, 30000, 8, 3600.0)
    engine.set_tuning("pair_variant", variant)
    try:
        got = run_engine(engine, st, sz, al, 12)
    finally:
        engine.set_tuning("pair_variant", 2)
    want = oracle.run(st, sz, al, steps=12)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    assert_same_conj(got[2], want[2])
    for f in ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "alive"):
        assert np.array_equal(got[3][f], want[3][f]), f


def test_record_ordering_falls_back_when_a_chunk_holds_many(engine, oracle, ks):
    # One-step chunks after a step with few records order them in one block;
    # a step with more records than that takes (16 384) falls back to the
    # multi-block sort. Its records equal the oracle's for that step.
    st, sz, al = ks.generate_population(504, 28340, 150000, 30, 86400.0)
    engine.set_steps_per_graph(1)
    engine.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
    engine.set_screening(True, 1.0, 1.0, 0.01)
    engine.set_population(st, sz, al)
    try:
        engine.run(1)
        few = engine.take_conjunctions()
        s1, a1 = engine.get_population()
        engine.set_screening(True, 90.0, 1.0, 0.01)
        engine.run(1)
        many = engine.take_conjunctions()
        engine.take_step_stats()
    finally:
        engine.set_screening(True, 5.0, 1.0, 0.01)
        engine.set_steps_per_graph(32)
    want = oracle.run(s1, sz, a1, t_start=10.0, steps=1, threshold_km=90.0)[2]
    assert 0 < len(few) < 1000 and len(many) > 16384
    many = many.copy()
    many["step"] -= 1
    assert_same_conj(many, want)
