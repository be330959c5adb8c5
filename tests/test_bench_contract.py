"""Host-side bookkeeping of bench.py (no GPU): the roofline fields of the JSON
line and the count of kernels it claims per step and per chunk."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def timing(steps=10, n=1_000_000, passes=4):
    return {"steps": steps, "propagate_ms": 0.05 * steps, "sort_ms": 0.09 * steps, "cells_ms": 0.07 * steps,
            "pairs_ms": 0.28 * steps, "refine_ms": 0.025 * steps, "chunk_ms": 0.007 * steps,
            "object_steps": n * steps, "candidate_pairs": 3.2e8 * steps, "sort_passes": passes}


def test_roofline_names_the_pair_kernel_and_its_fp32_rate(bench):
    r = bench.roofline_of(timing(), None, 17.6e12, 35.9e12, True)
    assert r["kernel"] == "pairs" and r["bound"] == "fp32" and r["unit"] == "TFLOP/s"
    assert r["peak"] == pytest.approx(35.9)
    assert r["achieved"] == pytest.approx(bench.FLOPS_PAIR_CHEAP * 3.2e8 / 0.28e-3 / 1e12)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    # both precisions screen with the FP32-gated kernel
    assert bench.roofline_of(timing(), None, 17.6e12, 35.9e12, False)["bound"] == "fp32"
    # the pipes the committed ncu capture saw beside the algorithmic rate
    pipes = r["pipes_ncu"]
    assert 0.0 < pipes["issue_active"] <= 1.0 and 0.0 < pipes["fma_pipe"] <= 1.0


def test_hbm_phases_use_algorithmic_bytes(bench):
    r = bench.roofline_of(timing(passes=4), None, 17.6e12, 35.9e12, True)["hbm"]
    assert r["peak_gbs"] > 0
    sort, cells, pairs = r["phases"]["sort"], r["phases"]["cells"], r["phases"]["pairs"]
    assert sort["algorithmic_bytes"] == pytest.approx(4 * 16 * 1e6)
    assert cells["algorithmic_bytes"] == pytest.approx(76 * 1e6)
    assert pairs["algorithmic_bytes"] == pytest.approx(32 * 1e6)
    assert sort["gbs"] == pytest.approx(64e6 / 0.09e-3 / 1e9)
    assert sort["frac"] == pytest.approx(sort["gbs"] / r["peak_gbs"])


def test_kernel_counts(bench):
    # propagate, fix_keys, P passes, cell count, scan, cell write, neighbours,
    # item count, scan, item write, pairs, refine
    assert bench.launches_per_step(4) == 15
    assert bench.launches_per_step(5) == 16
    # propagate, fix_keys, the fused sort + cells, pairs, refine
    assert bench.launches_per_step(4, True) == 5
    assert bench.LAUNCHES_PER_CHUNK == 8


def test_fused_sort_and_cells_are_one_memory_phase(bench):
    tm = dict(timing(passes=4), sort_cells_fused=1, cells_ms=0.0)
    r = bench.roofline_of(tm, None, 17.6e12, 35.9e12, True)["hbm"]["phases"]
    assert set(r) == {"sort_cells", "pairs"}
    assert r["sort_cells"]["algorithmic_bytes"] == pytest.approx((4 * 16 + 76) * 1e6)
    assert r["sort_cells"]["ms"] == pytest.approx(0.09)


def test_reference_arm_loads_nothing_of_the_engine():
    """bench.py --impl reference runs the reference's own CPU path on inputs
    from oracle/libks_workload.so: the engine library never enters the
    process, and the line reports exactly the requested steps and warm-up."""
    import json
    import subprocess

    code = r'''
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--objects", "3000", "--base", "2000", "--parents", "2",
            "--steps", "3", "--warmup", "2"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
print(json.dumps({"maps": sorted(set(l.split()[-1] for l in maps.splitlines() if l.endswith(".so")))}))
'''
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    line, maps = json.loads(lines[0]), json.loads(lines[-1])["maps"]
    assert line["impl"] == "reference" and line["steps"] == 3 and line["warmup"] == 2
    ours = [m for m in maps if m.startswith(ROOT)]
    assert ours and all(m.startswith(os.path.join(ROOT, "oracle")) for m in ours), ours
    assert not any("libkessler_b200" in m for m in maps)
