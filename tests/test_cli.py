"""The drop-in CLI (ks_sim) against the reference CLI on the same catalogue file.

tests/golden/cli_ref_*.csv were written by the reference's own CLI
(oracle/_ref/kessler_sim, built from its sources) for
tests/golden/cli_catalog.txt over 15 simulated minutes at dt = 10 s with
--conj-km 5. ks_sim must write the same files, byte for byte.
"""
import importlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path

PKG = os.path.join(ROOT, "kessler-syndrom-simulation_b200")
ARGS = ["0.25", "10", "--conj-km", "5"]


def fmt10(x):
    # std::ostream with setprecision(10), default float format (%.10g).
    return f"{x:.10g}"


def test_oracle_reproduces_reference_cli_conjunctions(oracle):
    cio = importlib.import_module("kessler-syndrom-simulation_b200.catalog_io")
    ids, names, rcs, states = cio.read_catalog(golden_path("cli_catalog.txt"))
    size_m = np.array([cio.RCS_SIZE_M.get(r, 0.8) for r in rcs])
    epoch = 2461253.916666667
    _, _, conj, _ = oracle.run(states, size_m, None, epoch_jd=epoch, dt=10.0, steps=90, threshold_km=5.0)
    lines = [f"{fmt10(c['t'])},{ids[c['i']]},{ids[c['j']]},\"{names[c['i']]}\",\"{names[c['j']]}\","
             f"{fmt10(c['miss_km'])},{fmt10(c['v_rel_km_s'])},{int(c['collision'])}" for c in conj]
    want = open(golden_path("cli_ref_conjunctions.csv")).read().splitlines()[1:]
    assert len(want) == 20
    assert lines == want


@pytest.mark.gpu
def test_cli_matches_reference_cli_files(tmp_path):
    exe = os.path.join(PKG, "ks_sim")
    assert os.path.exists(exe), "build the package first (make -C kessler-syndrom-simulation_b200)"
    out = subprocess.run([exe, golden_path("cli_catalog.txt")] + ARGS + ["--out", str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    for name in ("conjunctions.csv", "final_state.csv"):
        got = open(tmp_path / name).read()
        want = open(golden_path("cli_ref_" + name)).read()
        assert got == want, name


@pytest.mark.gpu
def test_cli_split_precision_finds_the_same_encounters(tmp_path):
    exe = os.path.join(PKG, "ks_sim")
    out = subprocess.run([exe, golden_path("cli_catalog.txt")] + ARGS + ["--split", "--out", str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    got = [ln.split(",") for ln in open(tmp_path / "conjunctions.csv").read().splitlines()[1:]]
    want = [ln.split(",") for ln in open(golden_path("cli_ref_conjunctions.csv")).read().splitlines()[1:]]
    assert [(g[1], g[2]) for g in got] == [(w[1], w[2]) for w in want]
    for g, w in zip(got, want):
        assert abs(float(g[5]) - float(w[5])) < 1e-4  # miss distance within 10 cm after 15 minutes


BREAKUP_ARGS = ["1.2", "10", "--breakup", "--radius-scale", "500", "--lc", "0.1", "--seed", "3",
                "--impact", "100051", "--impact-mass", "500", "--impact-vrel", "10", "--impact-at", "0.05"]


@pytest.mark.gpu
@pytest.mark.parametrize("spg", ["32", "5"])
def test_cli_breakup_matches_reference_cli_files(tmp_path, spg):
    # tests/golden/cli_breakup_ref_*.csv: the reference CLI with --breakup and a
    # forced impact; collisions fragment objects (fragments of fragments too).
    exe = os.path.join(PKG, "ks_sim")
    out = subprocess.run([exe, golden_path("cli_breakup_catalog.txt")] + BREAKUP_ARGS +
                         ["--steps-per-graph", spg, "--out", str(tmp_path)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    for name in ("breakups.csv", "population.csv", "conjunctions.csv", "final_state.csv"):
        got = open(tmp_path / name).read()
        want = open(golden_path("cli_breakup_ref_" + name)).read()
        assert got == want, name


@pytest.mark.gpu
@pytest.mark.parametrize("run", ["snapshots", "tracks"])
def test_cli_snapshots_match_reference_cli(tmp_path, run):
    # tests/golden/cli_snapshot_ref.json: SHA-256 of the reference CLI's periodic
    # snapshot files, or of its trajectories.csv and moon.csv for tracked ids.
    import hashlib
    import json
    ref = json.load(open(golden_path("cli_snapshot_ref.json")))[run]
    exe = os.path.join(PKG, "ks_sim")
    out = subprocess.run([exe, golden_path("cli_catalog.txt")] + ref["args"] + ["--out", str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    got = sorted(f for f in os.listdir(tmp_path) if f.startswith(("snapshot_", "trajectories", "moon")))
    assert got == sorted(ref["sha256"])
    for f in got:
        assert hashlib.sha256(open(tmp_path / f, "rb").read()).hexdigest() == ref["sha256"][f], f
