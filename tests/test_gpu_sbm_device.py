"""NASA SBM fragmentation on the device (ks_set_breakup_mode KS_BREAKUP_DEVICE).

The device SBM draws from Philox counters, not from the reference's Mersenne
Twister, so its fragments cannot equal the reference's one by one: parity is
statistical. The reference side of every comparison is the host SBM of this
library (ks_sbm_impact / the host breakup mode), which reproduces the
reference's Fragmentation (src/core/breakup.cpp:192-360) bit for bit
(tests/test_sbm_host.py, tests/test_gpu_breakup.py). Checked here:
  - the laws (README.md:394-402 of the reference): the number of fragments
    above L_c per event, N(> 2 L) / N(> L) = 2^-1.71 for sizes far below the
    parent's, area-to-mass and Delta-v distributions (two-sample
    Kolmogorov-Smirnov tests against the host SBM's fragments), an isotropic
    Delta-v, mass budgets;
  - the loop: collisions found on the device fragment there, in the reference's
    order and with its roles (the same events as the host mode on the same
    step), the population grows inside the chunks' graphs, and the fixed
    population budget is enforced;
  - nothing changes without collisions: a device-mode run that fragments
    nothing equals the host-mode run bit for bit.
"""
import numpy as np
import pytest
from scipy import stats as sps

from conftest import golden_path
from test_gpu_parity import STAT_FIELDS, assert_same_conj

pytestmark = pytest.mark.gpu

LC = 0.10
N_TARGETS = 400


def impact_population(ks, seed=5, n=N_TARGETS):
    """n LEO objects of 2 m and 800 kg, far apart from one another."""
    st, sz, al = ks.generate_population(seed, 4 * n)
    leo = np.flatnonzero(np.linalg.norm(st[:, :3], axis=1) < 6378.137 + 2000.0)[:n]
    assert len(leo) == n
    return st[leo].copy(), np.full(n, 2.0), np.full(n, 800.0)


def device_impacts(ks, st, sz, mass, m_proj, vrel, seed=11):
    with ks.Engine(0) as eng:
        eng.set_breakup_mode(ks.BREAKUP_DEVICE, len(st) + 400_000)
        eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
        eng.set_screening(True, 5.0, 1.0, 0.01)
        eng.set_population(st, sz)
        eng.set_masses(mass)
        eng.set_breakup(True, LC, 40.0, seed)
        for i in range(len(st)):
            eng.impact(i, m_proj, vrel)
        events = eng.take_breakups()
        n = eng.population_size()
        fs, fa = eng.get_population()
        props = eng.objects()
    return events, fs, fa, props, n


def host_impacts(ks, st, sz, mass, m_proj, vrel):
    out = []
    for i in range(len(st)):
        ev, fs, fz, fm, fa, after = ks.sbm_impact(st[i], mass[i], sz[i], m_proj, vrel, 0.0, seed=1000 + i, lc_m=LC)
        out.append((ev, fs, fz, fm, fa))
    return out


@pytest.fixture(scope="module")
def impacts(ks):
    st, sz, mass = impact_population(ks)
    dev = device_impacts(ks, st, sz, mass, 200.0, 10.0)
    host = host_impacts(ks, st, sz, mass, 200.0, 10.0)
    return st, sz, mass, dev, host


def test_device_impacts_follow_the_number_law(ks, impacts):
    st, sz, mass, (events, fs, fa, props, n), host = impacts
    assert len(events) == N_TARGETS
    # 200 kg at 10 km/s on 800 kg: 25 000 J/g, catastrophic; M = 1000 kg.
    assert events["catastrophic"].all()
    expected = 0.1 * 1000.0 ** 0.75 * LC ** -1.71
    assert np.allclose(events["expected_fragments"], expected)
    dev_n = events["fragments"] + events["escaped"]
    host_n = np.array([h[0]["fragments"] + h[0]["escaped"] for h in host])
    # Poisson numbers of candidates, some skipped by the mass budgets: the two
    # implementations' means agree within their standard errors.
    se = np.sqrt(dev_n.var() / len(dev_n) + host_n.var() / len(host_n))
    assert abs(dev_n.mean() - host_n.mean()) < 4 * se + 1.0, (dev_n.mean(), host_n.mean())
    # Every fragment is appended after the population, event by event.
    assert n == N_TARGETS + int(events["fragments"].sum())
    assert (props["event"][N_TARGETS:] >= 0).all() and (props["event"][:N_TARGETS] == -1).all()
    first = events["first_fragment"]
    assert np.array_equal(np.sort(first), first) and first[0] == N_TARGETS
    # Targets destroyed (catastrophic), fragments' mass within the budget.
    assert not fa[:N_TARGETS].any()
    assert (events["fragments_mass_kg"] <= events["sbm_mass_kg"] * (1 + 1e-12)).all()


def test_device_fragment_sizes_area_to_mass_and_delta_v(ks, impacts):
    st, sz, mass, (events, fs, fa, props, n), host = impacts
    d_size = props["size_m"][N_TARGETS:]
    d_a2m = props["area_to_mass"][N_TARGETS:]
    h_size = np.concatenate([h[2] for h in host])
    h_a2m = np.concatenate([h[4] for h in host])
    assert d_size.min() >= LC and h_size.min() >= LC
    # Power law: N(> 2 L) / N(> L) = 2^-1.71 for L far below the parents' 2 m
    # (0.302 with the truncation at 2 m), and the host SBM's ratios.
    for L in (LC, 2 * LC):
        ratio = (d_size > 2 * L).sum() / (d_size > L).sum()
        h_ratio = (h_size > 2 * L).sum() / (h_size > L).sum()
        assert abs(ratio - h_ratio) < 0.01, (L, ratio, h_ratio)
    assert abs((d_size > 2 * LC).sum() / (d_size > LC).sum() - 2 ** -1.71) < 0.01
    for name, d, h in (("log size", np.log10(d_size), np.log10(h_size)),
                       ("log A/m", np.log10(d_a2m), np.log10(h_a2m))):
        p = sps.ks_2samp(d, h).pvalue
        assert p > 1e-3, (name, p, len(d), len(h))
    # Delta-v relative to the target's velocity (fragments of both parents, in
    # both samples alike), and its direction about the target.
    ev_of = props["event"][N_TARGETS:]
    target_v = st[:, 3:][events["target"][np.searchsorted(events["id"], ev_of)]]
    d_dv = np.linalg.norm(fs[N_TARGETS:, 3:] - target_v, axis=1)
    h_dv = np.concatenate([np.linalg.norm(h[1][:, 3:] - st[i, 3:], axis=1) for i, h in enumerate(host)])
    p = sps.ks_2samp(np.log10(d_dv), np.log10(h_dv)).pvalue
    assert p > 1e-3, ("log dv", p)
    # Isotropy of the fragments of the target side (Delta-v below 1 km/s: the
    # projectile's fragments move at ~10 km/s relative to the target).
    slow = d_dv < 1.0
    u = (fs[N_TARGETS:, 3:] - target_v)[slow] / d_dv[slow, None]
    assert slow.sum() > 1000
    assert np.all(np.abs(u.mean(axis=0)) < 5 / np.sqrt(slow.sum()))
    assert np.allclose((u ** 2).mean(axis=0), 1 / 3, atol=0.03)


def test_device_breakup_in_the_loop(ks):
    """The planted collisions of the host-mode golden run: the first collision
    step fragments the same events (roles, times, energies) on the device as
    the host SBM does; the population grows inside the graphs; later steps
    screen the fragments."""
    fx = dict(np.load(golden_path("run_breakup.npz")))
    steps = int(fx["steps"])

    def run(mode, spg):
        with ks.Engine(0) as eng:
            if mode == ks.BREAKUP_DEVICE:
                eng.set_breakup_mode(mode, len(fx["states"]) + 200_000)
            eng.set_steps_per_graph(spg)
            eng.set_clock(float(fx["epoch_jd"]), 0.0, float(fx["dt"]))
            eng.set_screening(True, float(fx["threshold_km"]), float(fx["radius_scale"]), float(fx["min_vrel_km_s"]))
            eng.set_population(fx["states"], fx["size_m"], fx["alive"])
            eng.set_masses(fx["mass_kg"])
            eng.set_breakup(True, float(fx["lc_m"]), 40.0, int(fx["seed"]))
            eng.run(steps)
            fs, fa = eng.get_population()
            return dict(states=fs, alive=fa, conj=eng.take_conjunctions(), events=eng.take_breakups(),
                        stats=eng.take_step_stats(), n=eng.population_size(), **eng.objects())

    host = run(ks.BREAKUP_HOST, 32)
    for spg in (32, 5):
        dev = run(ks.BREAKUP_DEVICE, spg)
        first = int(host["events"]["step"].min())
        he = host["events"][host["events"]["step"] == first]
        de = dev["events"][dev["events"]["step"] == first]
        assert len(de) == len(he) >= 1
        for f in ("t", "target", "projectile", "catastrophic", "v_rel_km_s", "energy_j_per_g", "target_mass_kg",
                  "projectile_mass_kg", "sbm_mass_kg", "expected_fragments", "id"):
            assert np.allclose(de[f], he[f], rtol=1e-12, atol=0), f
        # Up to that step everything is the host mode's, bit for bit.
        for f in STAT_FIELDS:
            assert np.array_equal(dev["stats"][f][:first + 1], host["stats"][f][:first + 1]), f
        keep = lambda c: c[c["step"] <= first]  # noqa: E731
        assert_same_conj(keep(dev["conj"]), keep(host["conj"]))
        # The fragments joined the population and the run went on with them.
        assert dev["n"] == len(fx["states"]) + int(dev["events"]["fragments"].sum())
        assert len(dev["stats"]) == steps
        assert dev["stats"]["alive"][-1] > dev["stats"]["alive"][first - 1] if first > 0 else True
        assert (dev["event"][len(fx["states"]):] >= 0).all()


def test_device_mode_without_fragmentation_equals_host_mode(ks):
    """The device-mode plumbing (live population count, step gate, capacity
    grids) changes nothing when nothing fragments."""
    fx = dict(np.load(golden_path("run_mixed.npz")))

    def run(mode):
        with ks.Engine(0) as eng:
            if mode == ks.BREAKUP_DEVICE:
                eng.set_breakup_mode(mode, 3 * len(fx["states"]))
            eng.set_steps_per_graph(7)
            eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
            eng.set_screening(True, 5.0, 1.0, 0.01)
            eng.set_population(fx["states"], fx["size_m"], fx["alive"])
            eng.run(int(fx["steps"]))
            fs, fa = eng.get_population()
            return fs, fa, eng.take_conjunctions(), eng.take_step_stats()

    h, d = run(ks.BREAKUP_HOST), run(ks.BREAKUP_DEVICE)
    assert np.array_equal(h[0], d[0]) and np.array_equal(h[1], d[1])
    assert np.array_equal(d[0], fx["final_states"])
    assert_same_conj(d[2], h[2])
    for f in STAT_FIELDS:
        assert np.array_equal(d[3][f], h[3][f]), f


def test_device_population_budget_is_enforced(ks):
    st, sz, mass = impact_population(ks, n=4)
    with ks.Engine(0) as eng:
        eng.set_breakup_mode(ks.BREAKUP_DEVICE, len(st) + 50)  # room for 50 fragments
        eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
        eng.set_population(st, sz)
        eng.set_masses(mass)
        eng.set_breakup(True, LC, 40.0, 3)
        with pytest.raises(ks.KsError) as e:
            for i in range(len(st)):
                eng.impact(i, 200.0, 10.0)  # ~170 fragments each
        assert e.value.code == 5 and "budget" in str(e.value)
        with pytest.raises(ks.KsError):
            eng.save_population("/nonexistent/never-written.kspop")


def swarm_population(ks, per_target=300, seed=3):
    """4 LEO targets (10 m, 1 000 kg), each crossed inside one 10 s step by
    per_target small objects (0.1 m) at 10 km/s from random directions, at
    distinct times: thousands of collisions in one step, most of them with a
    parent that collided earlier in the step. Targets 0-1: 1 kg projectiles
    (catastrophic: the first hit destroys the target, later hits are void);
    targets 2-3: 50 g projectiles (cratering: every hit erodes the target
    until its mass is spent)."""
    rng = np.random.default_rng(seed)
    st, sz, al = ks.generate_population(seed, 400)
    leo = np.flatnonzero(np.linalg.norm(st[:, :3], axis=1) < 6378.137 + 1500.0)[:4]
    states, sizes, masses = [st[leo]], [np.full(4, 10.0)], [np.full(4, 1000.0)]
    for k in range(4):
        d = rng.normal(size=(per_target, 3))
        d *= 10.0 / np.linalg.norm(d, axis=1)[:, None]
        tk = np.sort(rng.uniform(0.5, 9.5, per_target))
        s = np.zeros((per_target, 6))
        s[:, :3] = st[leo[k], :3] - d * tk[:, None]
        s[:, 3:] = st[leo[k], 3:] + d
        states.append(s)
        sizes.append(np.full(per_target, 0.1))
        masses.append(np.full(per_target, 1.0 if k < 2 else 0.05))
    return np.vstack(states), np.concatenate(sizes), np.concatenate(masses)


def test_device_conflicting_collisions_follow_the_reference_order(ks):
    st, sz, mass = swarm_population(ks)

    def one_step(mode):
        with ks.Engine(0) as eng:
            if mode == ks.BREAKUP_DEVICE:
                eng.set_breakup_mode(mode, len(st) + 2_000_000)
            eng.set_clock(ks.DEFAULT_EPOCH_JD, 0.0, 10.0)
            eng.set_screening(True, 5.0, 10.0, 0.01)  # radii x10: the hits are certain
            eng.set_population(st, sz)
            eng.set_masses(mass)
            eng.set_breakup(True, 0.10, 40.0, 5)
            eng.run(1)
            conj = eng.take_conjunctions()
            return conj, eng.take_breakups(), eng.get_population()[1]

    hc, he, ha = one_step(ks.BREAKUP_HOST)
    dc, de, da = one_step(ks.BREAKUP_DEVICE)
    assert int(hc["collision"].sum()) == int(dc["collision"].sum()) > 1024
    assert len(de) == len(he)
    for f in ("t", "target", "projectile", "catastrophic"):
        assert np.array_equal(de[f], he[f]), f
    for f in ("target_mass_kg", "projectile_mass_kg", "sbm_mass_kg", "v_rel_km_s", "energy_j_per_g"):
        assert np.allclose(de[f], he[f], rtol=1e-9, atol=0), f
    # One event for each catastrophic swarm; for each cratering one, a long run
    # of events in arrival order, each eroding the target (about 5 kg a hit),
    # until the target's mass is spent and the later hits are void.
    assert int((he["target"] == 0).sum()) == int((he["target"] == 1).sum()) == 1
    for k in (2, 3):
        m = de["target_mass_kg"][de["target"] == k]
        assert len(m) > 100 and np.all(np.diff(m) < 0)
    # The parents' fates (alive flags of the original objects) as on the host.
    n0 = len(st)
    assert np.array_equal(da[:n0], ha[:n0])
