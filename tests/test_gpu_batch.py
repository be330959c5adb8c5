"""Batched realisations (one resident population of independent Monte Carlo runs).

Bar: each realisation of a batch gives, bit for bit, what a run on its objects
alone gives: final states and alive flags, conjunction records (indices offset
by the realisation's first row) and the refined / co-orbiting / conjunction
counters, summed over realisations. The batch shares one cell edge (at least
every realisation's own), so only candidate_pairs, cell_km and the fullest
cell may differ from the per-realisation runs. The grid cell edge knob
(cell_scale_permille) has the same contract on a single population.
"""
import numpy as np
import pytest

from test_gpu_parity import assert_same_conj, run_engine

pytestmark = pytest.mark.gpu

EPOCH = 2461253.916666667


def make_batch(ks, specs):
    """specs: (seed, n_base, n_total, parents, age) per realisation; (0, 0, ...) is an empty one."""
    parts = []
    for seed, n_base, n_total, parents, age in specs:
        if n_total == 0:
            parts.append((np.zeros((0, 6)), np.zeros(0), np.zeros(0, np.uint8)))
        else:
            parts.append(ks.generate_population(seed, n_base, n_total, parents, age))
    offsets = np.zeros(len(parts) + 1, np.int64)
    offsets[1:] = np.cumsum([len(p[1]) for p in parts])
    st = np.concatenate([p[0] for p in parts])
    sz = np.concatenate([p[1] for p in parts])
    al = np.concatenate([p[2] for p in parts])
    return parts, offsets, st, sz, al


def run_batch(eng, offsets, st, sz, al, steps, spg=16):
    eng.set_steps_per_graph(spg)
    eng.set_clock(EPOCH, 0.0, 10.0)
    eng.set_screening(True, 5.0, 1.0, 0.01)
    eng.set_population_batch(offsets, st, sz, al)
    eng.run(steps)
    fs, fa = eng.get_population()
    return fs, fa, eng.take_conjunctions(), eng.take_step_stats()


def per_realisation(conj, offsets, r):
    c = conj[conj["realisation"] == r].copy()
    c["i"] -= offsets[r]
    c["j"] -= offsets[r]
    return c


SPECS = [
    (101, 3000, 9000, 4, 0.0),        # fresh clouds
    (0, 0, 0, 0, 0.0),                # empty realisation
    (102, 1, 1, 0, 0.0),              # one object
    (103, 2500, 12000, 6, 3600.0),    # aged clouds, different size
    (104, 6000, 6000, 0, 0.0),        # catalogue only
]


def test_batch_equals_separate_oracle_runs(engine, oracle, ks):
    steps = 10
    parts, offsets, st, sz, al = make_batch(ks, SPECS)
    fs, fa, conj, stats = run_batch(engine, offsets, st, sz, al, steps)
    assert set(np.unique(conj["realisation"])) <= set(range(len(parts)))
    assert np.all(conj["i"] < conj["j"])
    sums = {f: np.zeros(steps, np.int64) for f in ("refined_pairs", "co_orbiting", "conjunctions", "alive")}
    for r, (pst, psz, pal) in enumerate(parts):
        lo, hi = offsets[r], offsets[r + 1]
        if hi == lo:
            assert not np.any(conj["realisation"] == r)
            continue
        want = oracle.run(pst, psz, pal, steps=steps)
        assert np.array_equal(fs[lo:hi], want[0]), r
        assert np.array_equal(fa[lo:hi], want[1]), r
        assert_same_conj(per_realisation(conj, offsets, r), want[2])
        for f in sums:
            sums[f] += want[3][f]
    assert len(conj) > 0
    for f in sums:
        assert np.array_equal(stats[f], sums[f]), f


def test_batch_split_equals_separate_split_runs(engine, ks):
    steps = 8
    parts, offsets, st, sz, al = make_batch(ks, [SPECS[0], SPECS[3], SPECS[4]])
    engine.set_precision(ks.PRECISION_SPLIT)
    try:
        fs, fa, conj, stats = run_batch(engine, offsets, st, sz, al, steps)
        for r, (pst, psz, pal) in enumerate(parts):
            lo, hi = offsets[r], offsets[r + 1]
            one = run_engine(engine, pst, psz, pal, steps)
            assert np.array_equal(fs[lo:hi], one[0]), r
            assert np.array_equal(fa[lo:hi], one[1]), r
            assert_same_conj(per_realisation(conj, offsets, r), one[2])
    finally:
        engine.set_precision(ks.PRECISION_FP64)


def test_batch_many_small_realisations(engine, oracle, ks):
    # 40 realisations (6 key bits) of uneven sizes, all in one grid
    specs = [(200 + r, 300 + 37 * r, 300 + 37 * r + (r % 5) * 400, r % 5, 0.0) for r in range(40)]
    parts, offsets, st, sz, al = make_batch(ks, specs)
    fs, fa, conj, stats = run_batch(engine, offsets, st, sz, al, 4)
    for r in (0, 7, 19, 39):
        pst, psz, pal = parts[r]
        want = oracle.run(pst, psz, pal, steps=4)
        lo, hi = offsets[r], offsets[r + 1]
        assert np.array_equal(fs[lo:hi], want[0]), r
        assert_same_conj(per_realisation(conj, offsets, r), want[2])


def test_single_population_resets_batch(engine, oracle, ks):
    parts, offsets, st, sz, al = make_batch(ks, [SPECS[0], SPECS[3]])
    run_batch(engine, offsets, st, sz, al, 2)
    pst, psz, pal = parts[1]
    got = run_engine(engine, pst, psz, pal, 5)
    want = oracle.run(pst, psz, pal, steps=5)
    assert np.array_equal(got[0], want[0])
    assert_same_conj(got[2], want[2])
    assert np.all(got[2]["realisation"] == 0)


@pytest.mark.parametrize("permille", [1000, 1500, 2500])
def test_cell_scale_changes_only_candidates(engine, oracle, ks, permille):
    st, sz, al = ks.generate_population(111, 4000, 20000, 8, 0.0)
    want = oracle.run(st, sz, al, steps=6)
    engine.set_tuning("cell_scale_permille", permille)
    try:
        got = run_engine(engine, st, sz, al, 6)
    finally:
        engine.set_tuning("cell_scale_permille", 1000)
    assert np.array_equal(got[0], want[0])
    assert_same_conj(got[2], want[2])
    for f in ("refined_pairs", "co_orbiting", "conjunctions", "alive"):
        assert np.array_equal(got[3][f], want[3][f]), f
    if permille == 1000:
        assert np.array_equal(got[3]["candidate_pairs"], want[3]["candidate_pairs"])
        assert np.array_equal(got[3]["cell_km"], want[3]["cell_km"])
    else:
        assert np.all(got[3]["cell_km"] > want[3]["cell_km"])
