"""The drop-in behind the reference's own calls: its CLI with --gpu.

kessler-syndrom-simulation_b200/host/wire_reference.py copies the reference's
src/ tree, inserts the engine behind the reference's calls (Screener::set_gpu,
gpu, begin, finish and Simulation::step call the engine through
host/kessler_b200.hpp with the reference's own State / Object / Conjunction
types) and builds the reference's main.cpp against libkessler_b200.so into
kessler-syndrom-simulation_b200/_wired/kessler_sim. That binary, run with
--gpu, must write the files the unmodified reference CLI wrote
(tests/golden/cli_ref_*.csv, cli_breakup_ref_*.csv), byte for byte.
"""
import importlib.util
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import REFERENCE_TREE, ROOT, golden_path

PKG = os.path.join(ROOT, "kessler-syndrom-simulation_b200")
WIRED = os.path.join(PKG, "_wired", "kessler_sim")
WIRING = os.path.join(PKG, "host", "wire_reference.py")


def wiring_module():
    spec = importlib.util.spec_from_file_location("wire_reference", WIRING)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_wiring_applies_to_the_reference_sources():
    """Every anchor of the wiring is found exactly once in the reference's
    sources, and the wired copy keeps building without the engine."""
    src_ref = os.path.join(REFERENCE_TREE, "src")
    if not os.path.isdir(src_ref):
        pytest.skip("reference tree not present")
    mod = wiring_module()
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "src")
        shutil.copytree(src_ref, src)
        mod.apply_edits(src)
        text = open(os.path.join(src, "core", "collision.cpp")).read()
        assert text.count("#ifdef KESSLER_HAS_B200") == 7
        assert "impl_->b200.screen<Conjunction>" in text
        assert "kessler_b200::step_objects" in open(os.path.join(src, "core", "orbital.cpp")).read()
        # Without KESSLER_HAS_B200 the edited sources are the reference's program.
        subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-fopenmp", "-I" + src,
                        os.path.join(src, "core", "collision.cpp"), os.path.join(src, "core", "orbital.cpp")],
                       check=True)


def run_wired(args, cwd):
    if not os.path.exists(WIRED):
        pytest.skip("wired reference CLI not built (needs the reference tree at build time)")
    return subprocess.run([WIRED] + args, cwd=cwd, capture_output=True, text=True, timeout=900)


@pytest.mark.gpu
def test_reference_cli_with_gpu_switch_writes_the_reference_files(tmp_path):
    out = run_wired([golden_path("cli_catalog.txt"), "0.25", "10", "--conj-km", "5", "--gpu"], tmp_path)
    assert out.returncode == 0, out.stderr
    assert "Detection sur GPU" in out.stdout, out.stdout  # set_gpu(true) reached the engine
    for name in ("conjunctions.csv", "final_state.csv"):
        got = open(tmp_path / "output" / name).read()
        want = open(golden_path("cli_ref_" + name)).read()
        assert got == want, name


@pytest.mark.gpu
def test_reference_cli_with_gpu_switch_and_breakup(tmp_path):
    # Fragmentation stays the reference's own (Fragmentation::apply on the host
    # objects); steps and screening run on the engine.
    args = [golden_path("cli_breakup_catalog.txt"), "1.2", "10", "--breakup", "--radius-scale", "500", "--lc", "0.1",
            "--seed", "3", "--impact", "100051", "--impact-mass", "500", "--impact-vrel", "10", "--impact-at", "0.05",
            "--gpu"]
    out = run_wired(args, tmp_path)
    assert out.returncode == 0, out.stderr
    for name in ("breakups.csv", "population.csv", "conjunctions.csv", "final_state.csv"):
        got = open(tmp_path / "output" / name).read()
        want = open(golden_path("cli_breakup_ref_" + name)).read()
        assert got == want, name
