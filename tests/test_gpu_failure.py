"""Failure detection on the device: a bounded wait that runs out.

The device-side waits of the engine are the radix sort's look-backs, where a
tile polls its predecessors' published digit counts, and the grid barriers of
the fused sort and cell build, where a block polls the count of blocks that
arrived. Each wait gives up after "lookback_polls" polls, sets a flag and goes
on with its stores kept in bounds; the host turns the flag into
KS_ERR_TIMEOUT and puts the simulation back where the chunk began. The
reference's counterpart is its CUDA-error path, which abandons the GPU for the
CPU for good (src/core/collision.cpp:706-714); the engine reports the error
instead and stays usable. Here the limit is set to zero, so that a tile gives
up at its first poll of a predecessor that has not published yet (a block at
its first poll of a barrier not every block has reached): no wait can hang,
and nothing faults. Both paths are run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KS_ERR_TIMEOUT = 7


def run_steps(ks, eng, st, sz, al, steps):
    eng.set_population(st, sz, al)
    eng.run(steps)
    fs, fa = eng.get_population()
    return fs, fa, eng.take_conjunctions(), eng.take_step_stats()


def configure(ks, eng):
    eng.set_precision(ks.PRECISION_FP64)
    eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
    eng.set_screening(True, 5.0, 1.0, 0.01)


@pytest.mark.parametrize("fused", [0, 1])
def test_lookback_wait_that_runs_out_is_reported_and_recoverable(ks, fused):
    # 400 000 objects: 196 sort tiles per pass, most of them running at once;
    # or one block per SM of the fused launch.
    st, sz, al = ks.generate_population(5, 20000, 400000, 40, 86400.0)
    with ks.Engine(0) as want_eng:
        configure(ks, want_eng)
        want_eng.set_tuning("sort_fused", 0)
        want = run_steps(ks, want_eng, st, sz, al, 3)
    with ks.Engine(0) as eng:
        configure(ks, eng)
        eng.set_tuning("sort_fused", fused)
        eng.set_tuning("lookback_polls", 0)
        err = None
        for _ in range(10):  # whether a tile finds its predecessor unpublished is a race: retry
            eng.set_population(st, sz, al)
            try:
                eng.run(1)
            except ks.KsError as e:
                err = e
                break
            eng.take_conjunctions()
            eng.take_step_stats()
        assert err is not None, "no look-back wait ran out in 10 runs"
        assert err.code == KS_ERR_TIMEOUT and "look-back" in str(err)
        # Nothing of the failed chunk is reported, and the clock did not move.
        assert len(eng.take_conjunctions()) == 0 and len(eng.take_step_stats()) == 0
        assert eng.clock()[1] == 0
        # With the default limit the same context runs on from where the failed
        # chunk began and gives the results of a clean run.
        eng.set_tuning("lookback_polls", 1 << 22)
        eng.run(3)
        fs, fa = eng.get_population()
        got = (fs, fa, eng.take_conjunctions(), eng.take_step_stats())
        assert eng.timing()["sort_cells_fused"] == fused
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    assert len(got[2]) == len(want[2])
    for f in ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision"):
        assert np.array_equal(got[2][f], want[2][f]), f
    for f in ("step", "candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km",
              "max_cell_objects", "alive"):
        assert np.array_equal(got[3][f], want[3][f]), f


def test_lookback_limit_is_validated(ks):
    with ks.Engine(0) as eng:
        with pytest.raises(ks.KsError):
            eng.set_tuning("lookback_polls", -1)
        with pytest.raises(ks.KsError):
            eng.set_tuning("lookback_polls", (1 << 30) + 1)
