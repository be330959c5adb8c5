"""ks_screen_noalloc: the screening entry point that allocates no GPU memory.

It serves callers that must not allocate at call time (device memory already
handed to their own pool, or a loop that cannot pay for cudaMalloc / cudaFree
synchronising the device). It must give exactly what ks_screen gives on the
same inputs, call after call, although every call reuses one fixed device
array. This file is collected last on purpose: a failure here comes after
every other test has run. It also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

MAX_OBJECTS = 16384


def noalloc(lib, ks, before, after, alive, size_m, t0, dt, thr=5.0, rscale=1.0, vmin=0.01, cap=1 << 15):
    ptr = ks._abi.ptr
    b = np.ascontiguousarray(before, dtype=np.float64)
    a = np.ascontiguousarray(after, dtype=np.float64)
    al = np.ascontiguousarray(alive, dtype=np.uint8)
    sz = np.ascontiguousarray(size_m, dtype=np.float64)
    out = np.zeros(cap, dtype=ks.CONJ_DTYPE)
    stats = np.zeros(1, dtype=ks.STATS_DTYPE)
    cnt = C.c_int64(-1)
    err = C.create_string_buffer(256)
    rc = lib.ks_screen_noalloc(len(b), ptr(b), ptr(a), ptr(al), ptr(sz), float(t0), float(dt), float(thr),
                               float(rscale), float(vmin), ptr(out), cap, C.byref(cnt), ptr(stats), None, err, 256)
    noalloc.count = cnt.value  # conjunctions found, also when the output is too small
    return rc, out[: max(min(cnt.value, cap), 0)], stats[0], err.value.decode()


def same(got, want):
    assert len(got) == len(want)
    for f in ("i", "j", "step", "t", "miss_km", "v_rel_km_s", "collision", "realisation"):
        assert np.array_equal(got[f], want[f]), f


STAT_FIELDS = ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km", "max_cell_objects",
               "alive")


def crossing_groups(per_group):
    """Two flat sheets of objects, per_group each, that fly through one another
    head-on at 15 km/s in the middle of a 10 s step: every pair of objects from
    different sheets passes within about 1 km (a conjunction at 5 km, no
    collision), pairs inside one sheet are co-orbiting."""
    nx = 20
    nz = -(-per_group // nx)
    k = np.arange(per_group)
    x, z = 0.04 * (k % nx), 0.04 * (k // nx)
    a = np.zeros((per_group, 6))
    a[:, 0], a[:, 1], a[:, 2], a[:, 4] = 7000.0 + x, -37.5, z, 7.5
    b = np.zeros((per_group, 6))
    b[:, 0], b[:, 1], b[:, 2], b[:, 4] = 7000.02 + x, 37.5, 0.02 + z, -7.5
    before = np.vstack([a, b])
    after = before.copy()
    after[:, :3] += 10.0 * before[:, 3:]
    n = len(before)
    assert nz * nx >= per_group
    return before, after, np.ones(n, np.uint8), np.ones(n)


def check_against_screen(lib, ks, eng, before, after, alive, size_m, t0, dt, thr=5.0):
    eng.set_screening(True, thr, 1.0, 0.01)
    want, wstats = eng.screen(before, after, alive, size_m, t0, dt)
    for _ in range(2):  # two calls in a row on the shared array
        rc, got, gstats, err = noalloc(lib, ks, before, after, alive, size_m, t0, dt, thr=thr)
        assert rc == 0, err
        same(got, want)
        for f in STAT_FIELDS:
            assert gstats[f] == wstats[f], f
    return want


def test_noalloc_matches_screen(ks):
    lib = ks.load_library()
    with ks.Engine(0) as eng:
        eng.set_screening(True, 5.0, 1.0, 0.01)
        fx = dict(np.load(golden_path("screen_cases.npz")))
        want = check_against_screen(lib, ks, eng, fx["before"], fx["after"], fx["alive_after"], fx["size_m"],
                                    float(fx["t0"]), float(fx["dt"]))
        assert len(want) == 5
        # ... and what the reference's own Screener returned on those inputs.
        rc, got, gstats, err = noalloc(lib, ks, fx["before"], fx["after"], fx["alive_after"], fx["size_m"],
                                       float(fx["t0"]), float(fx["dt"]))
        assert rc == 0, err
        same(got, fx["conj"])
        for f in STAT_FIELDS[:-1]:
            assert gstats[f] == fx["stats"][0][f], f
        # A population at the size limit with day-old fragment clouds, screened at
        # 20 km: about 10 000 pairs refined and 140 conjunctions.
        st, sz, al = ks.generate_population(41, 4000, MAX_OBJECTS, 6, 86400.0)
        after, alive_after = eng.propagate(st, al, ks.DEFAULT_EPOCH_JD, 0.0, 10.0, 1)
        want = check_against_screen(lib, ks, eng, st, after, alive_after, sz, 0.0, 10.0, thr=20.0)
        assert len(want) > 100


def test_noalloc_rejects_sizes_beyond_its_limit(ks):
    lib = ks.load_library()
    n = MAX_OBJECTS + 1
    z = np.zeros((n, 6))
    z[:, 0] = 7000.0
    rc, got, _, err = noalloc(lib, ks, z, z, np.ones(n, np.uint8), np.ones(n), 0.0, 10.0)
    assert rc == 6  # KS_ERR_RANGE
    assert "16384" in err and len(got) == 0


def test_noalloc_leaves_device_memory_untouched(ks):
    """Repeated calls must not change the device's free memory: nothing is
    allocated per call (kernels and the fixed array are loaded by the first)."""
    import torch

    lib = ks.load_library()
    fx = dict(np.load(golden_path("screen_cases.npz")))
    args = (fx["before"], fx["after"], fx["alive_after"], fx["size_m"], float(fx["t0"]), float(fx["dt"]))
    rc, _, _, err = noalloc(lib, ks, *args)
    assert rc == 0, err
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        rc, got, _, err = noalloc(lib, ks, *args)
        assert rc == 0 and len(got) == 5, err
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_reports_overflows_with_counts(ks):
    lib = ks.load_library()
    fx = dict(np.load(golden_path("screen_cases.npz")))
    args = (fx["before"], fx["after"], fx["alive_after"], fx["size_m"], float(fx["t0"]), float(fx["dt"]))
    # Output array too small: an error, no records written, and the count found.
    rc, got, _, err = noalloc(lib, ks, *args, cap=2)
    assert rc == 5 and noalloc.count == 5 and not got["t"].any(), err  # KS_ERR_OVERFLOW, out left zeroed
    # 200 x 200 = 40 000 conjunctions: beyond the fixed 32 768-record capacity.
    rc, got, st, err = noalloc(lib, ks, *crossing_groups(200), 0.0, 10.0, cap=1 << 16)
    assert rc == 5 and "conjunctions" in err, err
    assert noalloc.count == 40000 and not got["t"].any()
    # 400 x 400 = 160 000 pairs to refine: beyond the fixed 131 072-pair capacity.
    rc, got, _, err = noalloc(lib, ks, *crossing_groups(400), 0.0, 10.0, cap=1 << 16)
    assert rc == 5 and "refine" in err and noalloc.count == 0, err
    # Below the limits the same sheets screen normally, twice in a row, and
    # agree with the context-based entry point.
    with ks.Engine(0) as eng:
        want = check_against_screen(lib, ks, eng, *crossing_groups(100), 0.0, 10.0)
    assert len(want) == 100 * 100 and not want["collision"].any()
