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
    return rc, out[: max(cnt.value, 0)], stats[0], err.value.decode()


def same(got, want):
    assert len(got) == len(want)
    for f in ("i", "j", "t", "miss_km", "v_rel_km_s", "collision"):
        assert np.array_equal(got[f], want[f]), f


def check_against_screen(lib, ks, eng, before, after, alive, size_m, t0, dt, thr=5.0):
    eng.set_screening(True, thr, 1.0, 0.01)
    want, wstats = eng.screen(before, after, alive, size_m, t0, dt)
    for _ in range(2):  # two calls in a row on the shared array
        rc, got, gstats, err = noalloc(lib, ks, before, after, alive, size_m, t0, dt, thr=thr)
        assert rc == 0, err
        same(got, want)
        for f in ("candidate_pairs", "refined_pairs", "co_orbiting", "conjunctions", "cell_km",
                  "max_cell_objects", "alive"):
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
