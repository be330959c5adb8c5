"""Host-side NASA SBM fragmentation against the reference's own Fragmentation.

ks_sbm_impact (the engine's SBM, host code, no device) must reproduce
Fragmentation::impact of the reference compiled from its sources
(oracle/_ref/libksref.so) bit for bit: the event record, every fragment's birth
state, size, mass and area-to-mass ratio, and what happens to the target.
Cases cover both Poisson branches (mean below / above 10), catastrophic and
cratering impacts, a projectile heavier than the target (roles swap), a
target smaller than L_c, mass budgets that run out, and hyperbolic escapes.
"""
import importlib

import numpy as np
import pytest

ks = importlib.import_module("kessler-syndrom-simulation_b200")

LEO = [6878.137, 0.0, 0.0, 0.0, 7.61268, 0.0]
LEO_INCL = [-1200.0, 6200.0, 2900.0, -7.1, -1.9, 2.4]
GTO_PERIGEE = [6628.137, 0.0, 0.0, 0.0, 10.2, 0.9]  # ~10.3 km/s: some fragments escape

# (state, target mass, target size, projectile mass, v_rel, lc, seed)
CASES = [
    (LEO, 500.0, 4.0, 800.0, 10.0, 0.05, 1),        # catastrophic, many fragments (PTRS)
    (LEO, 1000.0, 4.0, 0.05, 2.0, 0.10, 2),         # cratering, few fragments (Knuth)
    (LEO_INCL, 0.0, 0.8, 300.0, 10.0, 0.10, 3),     # unknown target mass -> 100 kg; projectile heavier: roles swap
    (LEO_INCL, 50.0, 0.08, 5.0, 7.0, 0.10, 4),      # target smaller than L_c: only projectile fragments
    (GTO_PERIGEE, 2000.0, 4.0, 1500.0, 14.0, 0.02, 5),  # large event, escapes
    (LEO, 100.0, 0.8, 1.0, 0.5, 0.10, 6),           # very low energy
    (LEO, 20.0, 1.5, 10.0, 20.0, 0.10, 7),          # v_rel above twice the horizontal speed: theta = pi
]


@pytest.mark.parametrize("case", CASES)
def test_sbm_impact_equals_reference(reference, case):
    state, mt, size, mp, vrel, lc, seed = case
    got = ks.sbm_impact(state, mt, size, mp, vrel, t=1234.5, seed=seed, lc_m=lc)
    want = reference.impact(state, mt, size, mp, vrel, t=1234.5, seed=seed, lc_m=lc)
    gev, wev = got[0], want[0]
    for f in ("t", "target", "projectile", "catastrophic", "fragments", "escaped", "v_rel_km_s", "energy_j_per_g",
              "target_mass_kg", "projectile_mass_kg", "sbm_mass_kg", "expected_fragments", "fragments_mass_kg",
              "position"):
        assert np.array_equal(gev[f], wev[f]), f
    for k, name in enumerate(("states", "size_m", "mass_kg", "area_to_mass", "target_after"), start=1):
        assert got[k].shape == want[k].shape, name
        assert np.array_equal(got[k], want[k]), name


def test_sbm_cases_reach_every_branch(reference):
    outs = [ks.sbm_impact(c[0], c[1], c[2], c[3], c[4], seed=c[6], lc_m=c[5]) for c in CASES]
    ev = [o[0] for o in outs]
    assert any(e["expected_fragments"] >= 10 for e in ev) and any(0 < e["expected_fragments"] < 10 for e in ev)
    assert any(e["catastrophic"] for e in ev) and any(not e["catastrophic"] for e in ev)
    assert any(e["target"] == -1 for e in ev)          # fictitious projectile was the heavier body
    assert any(e["escaped"] > 0 for e in ev)
    assert any(e["fragments_mass_kg"] < e["sbm_mass_kg"] for e in ev)


def test_sbm_statistics_follow_the_model():
    # Size law N(>2L)/N(>L) = 2^-1.71 and the delta-v scale of the SBM, over a large event.
    # A small projectile: > 99% of the fragments come from the target, whose velocity is LEO's.
    ev, st, size, mass, a2m, _ = ks.sbm_impact(LEO, 2000.0, 4.0, 10.0, 10.0, seed=11, lc_m=0.01)
    assert ev["catastrophic"] and ev["fragments"] > 20000
    ratio = (size > 0.02).sum() / (size > 0.01).sum()
    assert abs(ratio - 2 ** -1.71) < 0.02
    dv = np.linalg.norm(st[:, 3:] - np.array(LEO[3:]), axis=1) * 1000.0
    # log10(dv / m/s) ~ N(0.9 log10(A/m) + 2.9, 0.4)
    resid = np.log10(dv) - (0.9 * np.log10(a2m) + 2.9)
    assert abs(np.median(resid)) < 0.05 and abs(np.std(resid[np.abs(resid) < 2]) - 0.4) < 0.05
    assert np.all(size >= 0.01) and np.all(mass > 0) and np.all(a2m > 0)
