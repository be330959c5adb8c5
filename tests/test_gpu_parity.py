"""Parity of the B200 engine (through the C ABI) with the reference and the oracle.

Bar: bit-exact. Final states, alive flags, conjunction records (pair ids, step,
TCA, miss distance, relative speed, collision flag) and per-step counters
(candidate pairs, refined pairs, co-orbiting pairs, cell edge, fullest cell)
must equal the reference's, which the golden fixtures hold, and the oracle's on
fresh inputs.
"""
import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

STAT_FIELDS = ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects",
               "alive")


def load(name):
    return dict(np.load(golden_path(name)))


def run_engine(eng, states, size_m, alive, steps, epoch_jd=2461253.916666667, dt=10.0, thr=5.0, rscale=1.0,
               vmin=0.01, spg=32, chunks=None):
    eng.set_steps_per_graph(spg)
    eng.set_clock(epoch_jd, 0.0, dt)
    eng.set_screening(True, thr, rscale, vmin)
    eng.set_population(states, size_m, alive)
    for k in (chunks or [steps]):
        eng.run(k)
    fs, fa = eng.get_population()
    return fs, fa, eng.take_conjunctions(), eng.take_step_stats()


def assert_same_stats(got, want):
    assert len(got) == len(want)
    for f in STAT_FIELDS:
        assert np.array_equal(got[f], want[f]), f


def assert_same_conj(got, want):
    assert len(got) == len(want), (len(got), len(want))
    for f in ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision"):
        assert np.array_equal(got[f], want[f]), f


@pytest.mark.parametrize("name", ["run_mixed.npz", "run_dense.npz"])
@pytest.mark.parametrize("spg", [0, 32])
def test_engine_reproduces_reference_run(engine, name, spg):
    fx = load(name)
    fs, fa, conj, stats = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], int(fx["steps"]),
                                     float(fx["epoch_jd"]), float(fx["dt"]), float(fx["threshold_km"]),
                                     float(fx["radius_scale"]), float(fx["min_vrel_km_s"]), spg=spg)
    assert np.array_equal(fs, fx["final_states"]), "states differ from the reference"
    assert np.array_equal(fa, fx["final_alive"])
    assert_same_conj(conj, fx["conj"])
    assert_same_stats(stats, fx["stats"])


def test_chunking_and_graph_parity_do_not_change_results(engine):
    fx = load("run_mixed.npz")
    base = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], 40, spg=0)
    for spg, chunks in ((7, [13, 27]), (1, [40]), (5, [3, 3, 34])):
        got = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], 40, spg=spg, chunks=chunks)
        assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
        assert_same_conj(got[2], base[2])
        assert_same_stats(got[3], base[3])


@pytest.mark.parametrize("variant,bps,x2,s2", [(0, 0, 1, 1), (0, 1, 1, 1), (1, 5, 1, 1), (1, 0, 1, 1), (2, 3, 1, 1),
                                               (2, 5, 1, 1),
                                               (2, 1, 1, 1), (2, 0, 0, 1), (2, 3, 0, 0), (2, 0, 1, 0), (2, 0, 1, 2),
                                               (2, 3, 0, 2)])
def test_tuning_knobs_do_not_change_results(engine, variant, bps, x2, s2):
    fx = load("run_dense.npz")
    engine.set_tuning("pair_variant", variant)
    engine.set_tuning("pair_blocks_per_sm", bps)
    engine.set_tuning("pair_gate_x2", x2)
    engine.set_tuning("pair_stage2", s2)
    try:
        fs, fa, conj, stats = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], int(fx["steps"]))
    finally:
        engine.set_tuning("pair_variant", 2)
        engine.set_tuning("pair_blocks_per_sm", 0)
        engine.set_tuning("pair_gate_x2", 1)
        engine.set_tuning("pair_stage2", 1)
    assert np.array_equal(fs, fx["final_states"])
    assert_same_conj(conj, fx["conj"])
    assert_same_stats(stats, fx["stats"])


def test_buffer_overflow_replays_to_the_same_result(engine):
    fx = load("run_mixed.npz")
    base = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], 40)
    engine.set_buffer_limits(survivor_pairs=1, conjunctions=1)
    got = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], 40)
    engine.set_buffer_limits(survivor_pairs=1 << 20, conjunctions=1 << 16)
    assert np.array_equal(got[0], base[0])
    assert_same_conj(got[2], base[2])
    assert_same_stats(got[3], base[3])


def test_screen_matches_reference_cases(engine):
    fx = load("screen_cases.npz")
    conj, stats = engine.screen(fx["before"], fx["after"], fx["alive_after"], fx["size_m"], float(fx["t0"]),
                                float(fx["dt"]))
    want = fx["stats"][0]
    assert_same_conj(conj, fx["conj"])
    for f in STAT_FIELDS[:-1]:
        assert stats[f] == want[f], f


@pytest.mark.parametrize("seed,n_base,n_total,parents,age,steps", [
    (11, 3000, 20000, 8, 0.0, 6),        # fresh clouds: thousands of objects per cell
    (12, 5000, 30000, 20, 6 * 3600.0, 8),  # aged clouds
    (13, 28340, 28340, 1, 0.0, 12),      # catalogue-sized, no fragments
])
def test_engine_matches_oracle_fresh_inputs(engine, oracle, ks, seed, n_base, n_total, parents, age, steps):
    st, sz, al = ks.generate_population(seed, n_base, n_total, parents, age)
    want = oracle.run(st, sz, al, steps=steps)
    got = run_engine(engine, st, sz, al, steps)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[1], want[1])
    assert_same_conj(got[2], want[2])
    assert_same_stats(got[3], want[3])


def test_engine_screen_matches_oracle_wide_threshold(engine, oracle, ks):
    st, sz, al = ks.generate_population(21, 4000, 9000, 5, 3600.0)
    after, alive_after = engine.propagate(st, al, 2461253.916666667, 0.0, 10.0, 1)
    for thr in (0.5, 5.0, 40.0):
        want, ws = oracle.screen(st, after, alive_after, sz, 0.0, 10.0, threshold_km=thr)
        engine.set_screening(True, thr, 1.0, 0.01)
        got, gs = engine.screen(st, after, alive_after, sz, 0.0, 10.0)
        assert_same_conj(got, want)
        for f in STAT_FIELDS:
            assert gs[f] == ws[f], (thr, f)
    engine.set_screening(True, 5.0, 1.0, 0.01)


def test_propagate_matches_oracle(engine, oracle, ks):
    st, sz, al = ks.generate_population(31, 5000)
    st[:3] = [[6390.0, 0, 0, -15.0, 0.3, 0], [0, 6700.0, 0, 0, -4.0, 1.0], [7000.0, 0, 0, 0, 7.5, 0]]
    al[2] = 0  # dead objects keep their state
    want = oracle.run(st, sz, al, steps=30, screen=False)
    got = engine.propagate(st, al, 2461253.916666667, 0.0, 10.0, 30)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[1], want[1])
    assert np.array_equal(got[0][2], st[2])


def test_edge_populations(engine, oracle):
    # empty
    conj, stats = engine.screen(np.zeros((0, 6)), np.zeros((0, 6)), np.zeros(0, np.uint8), np.zeros(0), 0.0, 10.0)
    assert len(conj) == 0 and stats["candidate_pairs"] == 0
    # one object; two objects at the same point; all dead
    one = np.array([[7000.0, 0, 0, 0, 7.5, 0]])
    fs, fa, conj, stats = run_engine(engine, one, np.ones(1), None, 5)
    want = oracle.run(one, np.ones(1), None, steps=5)
    assert np.array_equal(fs, want[0]) and len(conj) == 0 and stats["candidate_pairs"].sum() == 0
    two = np.array([[7000.0, 0, 0, 0, 7.5, 0], [7000.0, 0, 0, 0, 7.5, 0]])
    got = run_engine(engine, two, np.ones(2), None, 3)
    want = oracle.run(two, np.ones(2), None, steps=3)
    assert_same_stats(got[3], want[3])
    assert got[3]["candidate_pairs"].sum() == 3
    dead = np.zeros(4, np.uint8)
    got = run_engine(engine, np.tile(one, (4, 1)), np.ones(4), dead, 3)
    assert got[3]["alive"].max() == 0 and got[3]["candidate_pairs"].sum() == 0


def test_partial_takes_return_records_in_order(engine, ks):
    # Records taken a few at a time, between chunks and across them, come out
    # in the same (t, i, j) order as one take after the whole run.
    import ctypes as C
    from importlib import import_module
    ptr = import_module(ks.__name__ + "._abi").ptr
    st, sz, al = ks.generate_population(505, 5000, 30000, 8, 3600.0)
    want = run_engine(engine, st, sz, al, 24, spg=8)[2]
    assert len(want) > 40

    def take(cap):
        out = np.empty(cap, dtype=ks.CONJ_DTYPE)
        cnt = C.c_int64()
        assert engine._lib.ks_take_conjunctions(engine._h, ptr(out), cap, C.byref(cnt)) == 0
        return out[: cnt.value]

    engine.set_steps_per_graph(8)
    engine.set_clock(2461253.916666667, 0.0, 10.0)
    engine.set_screening(True, 5.0, 1.0, 0.01)
    engine.set_population(st, sz, al)
    parts = []
    engine.run(8)
    parts.append(take(3))          # from the last chunk's records
    engine.run(8)                  # the rest of the first chunk moves behind
    parts.append(take(5))
    parts.append(take(1))
    engine.run(8)
    parts.append(take(len(want)))  # everything left, older records first
    parts.append(take(10))         # nothing left
    engine.take_step_stats()
    got = np.concatenate(parts)
    assert len(parts[-1]) == 0
    assert_same_conj(got, want)


def test_ballot_ranking_of_the_radix_sort_changes_nothing(engine):
    """The radix sort's warp ranking by eight ballots orders the keys exactly
    as the hardware match does: the same run, bit for bit."""
    fx = load("run_mixed.npz")
    engine.set_tuning("sort_rank_ballot", 1)
    try:
        fs, fa, conj, stats = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], 40, spg=7)
    finally:
        engine.set_tuning("sort_rank_ballot", 0)
    assert np.array_equal(fs, fx["final_states"]) and np.array_equal(fa, fx["final_alive"])
    assert_same_conj(conj, fx["conj"])
    assert_same_stats(stats, fx["stats"])


@pytest.mark.parametrize("name,steps,spg,ballot", [("run_mixed.npz", 40, 7, 0), ("run_dense.npz", 0, 32, 0),
                                                    ("run_mixed.npz", 40, 32, 1)])
def test_fused_sort_and_cell_build_reproduce_the_reference(engine, name, steps, spg, ballot):
    """The object sort and cell build in one cooperative launch (the default
    where it fits) give the reference's run bit for bit, and so does the path
    of separate kernels; the timing block says which path ran."""
    fx = load(name)
    steps = steps or int(fx["steps"])
    engine.set_tuning("sort_rank_ballot", ballot)
    try:
        for fused in (1, 0):
            engine.set_tuning("sort_fused", fused)
            fs, fa, conj, stats = run_engine(engine, fx["states"], fx["size_m"], fx["alive"], steps, spg=spg,
                                             epoch_jd=float(fx["epoch_jd"]), dt=float(fx["dt"]),
                                             thr=float(fx["threshold_km"]), rscale=float(fx["radius_scale"]),
                                             vmin=float(fx["min_vrel_km_s"]))
            assert engine.timing()["sort_cells_fused"] == fused
            if steps == int(fx["steps"]):
                assert np.array_equal(fs, fx["final_states"]) and np.array_equal(fa, fx["final_alive"])
                assert_same_conj(conj, fx["conj"])
                assert_same_stats(stats, fx["stats"])
            elif fused:
                base = (fs, fa, conj, stats)
            else:
                assert np.array_equal(fs, base[0]) and np.array_equal(fa, base[1])
                assert_same_conj(conj, base[2])
                assert_same_stats(stats, base[3])
    finally:
        engine.set_tuning("sort_fused", 1)
        engine.set_tuning("sort_rank_ballot", 0)


@pytest.mark.parametrize("n_total,age", [(300_000, 3600.0), (1_100_000, 86400.0), (1_500_000, 86400.0)])
def test_fused_sort_and_cell_build_equal_the_separate_kernels(engine, ks, n_total, age):
    """Larger populations (4, 8 and 12 keys per thread of the fused kernel;
    the second near its 8-key limit), with 8-bit and 11-bit digits and with
    the whole hash or a crowded part of it (2 slots per cell: longer probe
    sequences): every record, counter and state equal with the fused launch and
    with the separate kernels."""
    st, sz, al = ks.generate_population(77, 20000, n_total, 60, age)
    runs = []
    try:
        for fused, bits, slots in ((1, 8, 0), (1, 11, 4), (1, 8, 2), (0, 8, 0)):
            engine.set_tuning("sort_fused", fused)
            engine.set_tuning("sort_digit_bits", bits)
            engine.set_tuning("hash_slots_per_cell", slots)
            runs.append(run_engine(engine, st, sz, al, 6, spg=3))
            assert engine.timing()["sort_cells_fused"] == fused
    finally:
        engine.set_tuning("sort_fused", 1)
        engine.set_tuning("sort_digit_bits", 8)
        engine.set_tuning("hash_slots_per_cell", 0)
    fs0, fa0, c0, s0 = runs[-1]
    assert len(c0) > 0
    for fs1, fa1, c1, s1 in runs[:-1]:
        assert np.array_equal(fs1, fs0) and np.array_equal(fa1, fa0)
        assert_same_conj(c1, c0)
        assert_same_stats(s1, s0)


def test_prepared_graphs_give_the_same_run(engine):
    """ks_prepare_run captures the chunk graphs (both parities) before the
    run: the run that launches them equals the reference's."""
    fx = load("run_mixed.npz")
    engine.set_steps_per_graph(5)
    engine.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
    engine.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
    engine.set_population(fx["states"], fx["size_m"], fx["alive"])
    engine.prepare_run()
    engine.run(int(fx["steps"]))
    fs, fa = engine.get_population()
    assert np.array_equal(fs, fx["final_states"]) and np.array_equal(fa, fx["final_alive"])
    assert_same_conj(engine.take_conjunctions(), fx["conj"])
    assert_same_stats(engine.take_step_stats(), fx["stats"])


def test_zero_copy_take_returns_the_same_records(engine, ks):
    """ks_take_conjunctions_view hands out the records where the engine holds
    them, older chunks' first, in the order of one copying take after the run;
    each view stays readable until the next run."""
    st, sz, al = ks.generate_population(505, 5000, 30000, 8, 3600.0)
    want = run_engine(engine, st, sz, al, 24, spg=8)[2]
    assert len(want) > 40
    engine.set_steps_per_graph(8)
    engine.set_clock(2461253.916666667, 0.0, 10.0)
    engine.set_screening(True, 5.0, 1.0, 0.01)
    engine.set_population(st, sz, al)
    parts = []
    engine.run(8)
    parts.append(engine.take_conjunctions_view().copy())   # the chunk's records in pinned memory
    assert len(engine.take_conjunctions_view()) == 0
    engine.run(8)
    engine.run(8)                                          # the second chunk's records move behind
    while True:
        v = engine.take_conjunctions_view()
        if len(v) == 0:
            break
        parts.append(v.copy())
    assert len(engine.take_conjunctions()) == 0
    engine.take_step_stats()
    got = np.concatenate(parts)
    assert_same_conj(got, want)
