"""Split precision: FP32 J2 / lunar terms and FP32 recentred pair gate.

Screening in split precision must make exactly the decisions of the FP64
filter on the same states (the FP32 gate only removes pairs the exact filter
rejects; survivors go through filter_pair in FP64). Propagation in split
precision is compared with the FP64 path, which is bit-identical to the
reference: the position error must stay below 1 m after 24 h (8 640 steps of
10 s), the target of the split form.
"""
import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

STAT_FIELDS = ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects",
               "alive")


def same_conj(got, want):
    assert len(got) == len(want)
    for f in ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision"):
        assert np.array_equal(got[f], want[f]), f


@pytest.mark.parametrize("age,thr", [(0.0, 5.0), (3600.0, 5.0), (86400.0, 25.0)])
def test_split_screening_decides_like_fp64(engine, ks, age, thr):
    st, sz, al = ks.generate_population(51, 5000, 30000, 12, age)
    after, alive_after = engine.propagate(st, al, ks.DEFAULT_EPOCH_JD, 0.0, 10.0, 1)
    out = {}
    for prec in (ks.PRECISION_FP64, ks.PRECISION_SPLIT):
        engine.set_precision(prec)
        engine.set_screening(True, thr, 1.0, 0.01)
        out[prec] = engine.screen(st, after, alive_after, sz, 0.0, 10.0)
    engine.set_precision(ks.PRECISION_FP64)
    engine.set_screening(True, 5.0, 1.0, 0.01)
    (c64, s64), (c32, s32) = out[ks.PRECISION_FP64], out[ks.PRECISION_SPLIT]
    same_conj(c32, c64)
    for f in STAT_FIELDS:
        assert s32[f] == s64[f], f


@pytest.mark.parametrize("dt,fast", [(120.0, False), (120.0, True), (600.0, False)])
def test_split_screening_decides_like_fp64_on_large_cells(engine, ks, dt, fast):
    # Long steps (cell edges of 2 500 to 13 000 km) and objects at 33 km/s: the
    # FP32 record error bounds grow with the cell edge and the largest speed.
    st, sz, al = ks.generate_population(52, 4000, 24000, 10, 3600.0)
    if fast:
        st = st.copy()
        st[:40, 3:] *= 4.3
    after, alive_after = engine.propagate(st, al, ks.DEFAULT_EPOCH_JD, 0.0, dt, 1)
    out = {}
    for prec in (ks.PRECISION_FP64, ks.PRECISION_SPLIT):
        engine.set_precision(prec)
        engine.set_screening(True, 5.0, 1.0, 0.01)
        out[prec] = engine.screen(st, after, alive_after, sz, 0.0, dt)
    engine.set_precision(ks.PRECISION_FP64)
    (c64, s64), (c32, s32) = out[ks.PRECISION_FP64], out[ks.PRECISION_SPLIT]
    assert s64["cell_km"] > 2000.0 and len(c64) > 0
    same_conj(c32, c64)
    for f in STAT_FIELDS:
        assert s32[f] == s64[f], f


def test_split_run_screening_matches_fp64_screening_of_its_own_states(engine, ks):
    """Over a multi-step split run, each step's conjunctions equal a one-shot
    FP64 screen of that step's split-precision before/after states."""
    fx = dict(np.load(golden_path("run_mixed.npz")))
    engine.set_precision(ks.PRECISION_SPLIT)
    engine.set_clock(float(fx["epoch_jd"]), 0.0, 10.0)
    engine.set_screening(True, 5.0, 1.0, 0.01)
    engine.set_population(fx["states"], fx["size_m"], fx["alive"])
    states = [engine.get_population()]
    conj, stats = [], []
    for _ in range(6):
        engine.run(1)
        states.append(engine.get_population())
        conj.append(engine.take_conjunctions())
        stats.append(engine.take_step_stats()[0])
    engine.set_precision(ks.PRECISION_FP64)
    for k in range(6):
        (b, _), (a, alive_after) = states[k], states[k + 1]
        want, ws = engine.screen(b, a, alive_after, fx["size_m"], 10.0 * k, 10.0)
        got = conj[k].copy()
        got["step"] = 0
        same_conj(got, want)
        for f in STAT_FIELDS[:-1]:
            assert stats[k][f] == ws[f], f


def test_split_propagation_error_budget(engine, ks):
    st, sz, al = ks.generate_population(61, 8000, 20000, 20, 86400.0)
    err = {}
    s64, s32 = st.copy(), st.copy()
    a64, a32 = al.copy(), al.copy()
    t = 0.0
    for hours in (1, 6, 24):
        steps = int(round((hours * 3600.0 - t) / 10.0))
        engine.set_precision(ks.PRECISION_FP64)
        s64, a64 = engine.propagate(s64, a64, ks.DEFAULT_EPOCH_JD, t, 10.0, steps)
        engine.set_precision(ks.PRECISION_SPLIT)
        s32, a32 = engine.propagate(s32, a32, ks.DEFAULT_EPOCH_JD, t, 10.0, steps)
        t = hours * 3600.0
        live = (a64 == 1) & (a32 == 1)
        dr = np.linalg.norm(s32[live, :3] - s64[live, :3], axis=1) * 1000.0  # m
        dv = np.linalg.norm(s32[live, 3:] - s64[live, 3:], axis=1) * 1e6     # mm/s
        err[hours] = (dr.max(), np.median(dr), dv.max())
    engine.set_precision(ks.PRECISION_FP64)
    print("split vs FP64 position error [m] max/median, velocity error max [mm/s]:", err)
    assert err[1][0] < 0.05
    assert err[24][0] < 1.0


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("sub,box", [(0, 8), (2, 0), (3, 1), (1, 33)])
def test_grid_order_and_pruning_knobs_do_not_change_results(engine, ks, prec, sub, box):
    """Morton order inside cells and tile pruning only change the amount of
    work: conjunctions and counters stay those of the default settings."""
    st, sz, al = ks.generate_population(71, 3000, 20000, 10, 1800.0)

    def run():
        engine.set_precision(prec)
        engine.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
        engine.set_screening(True, 5.0, 1.0, 0.01)
        engine.set_population(st, sz, al)
        engine.run(8)
        return engine.get_population(), engine.take_conjunctions(), engine.take_step_stats()

    base = run()
    engine.set_tuning("subcell_bits", sub)
    engine.set_tuning("box_min_rows", box)
    try:
        got = run()
    finally:
        engine.set_tuning("subcell_bits", 1)
        engine.set_tuning("box_min_rows", 4)
        engine.set_precision(ks.PRECISION_FP64)
    assert np.array_equal(got[0][0], base[0][0])
    same_conj(got[1], base[1])
    for f in STAT_FIELDS:
        assert np.array_equal(got[2][f], base[2][f]), f
