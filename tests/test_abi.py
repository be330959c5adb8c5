"""C-ABI library: loads, exports every declared symbol, host-side helpers.

No device work here; these run on a machine without a GPU.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("kessler_b200.h", "ks_records.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[\w\*]+\s+)+\**(ks_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("ks_create", "ks_run", "ks_screen", "ks_propagate", "ks_take_conjunctions",
                 "ks_set_population", "ks_moon_position"):
        assert must in names


def test_library_exports_every_declared_symbol(ks):
    lib = C.CDLL(ks._abi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # and the Python layer declares a prototype for each of them
    assert set(declared_functions()) <= set(ks._abi.SIGNATURES)


def test_record_layouts_match_header(ks):
    assert ks.CONJ_DTYPE.itemsize == 48
    assert ks.STATS_DTYPE.itemsize == 56
    assert ks.CONJ_DTYPE.fields["t"][1] == 16 and ks.CONJ_DTYPE.fields["collision"][1] == 40


def test_every_exported_entry_point_is_declared(ks):
    out = os.popen(f"nm -D --defined-only {ks._abi.LIB_PATH}").read()
    exported = {m.group(1) for m in re.finditer(r"\sT\s(ks_\w+)$", out, flags=re.M)}
    assert exported, "no ks_ symbols exported"
    undeclared = sorted(exported - set(declared_functions()))
    assert not undeclared, f"exported but not declared in include/: {undeclared}"


def test_library_is_built_for_sm100a_only():
    # The build compiles device code for one target only: sm_100a.
    mk = open(os.path.join(ROOT, "kessler-syndrom-simulation_b200", "Makefile")).read()
    arch = re.findall(r"arch=compute_\w+,code=\w+", mk)
    assert arch == ["arch=compute_100a,code=sm_100a"]


def test_no_device_means_an_error_not_a_fallback(ks):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(ks.KsError) as e:
        ks.Engine(0)
    assert e.value.code == 3  # KS_ERR_NO_DEVICE


def test_product_ephemeris_matches_reference(ks, reference):
    rng = np.random.default_rng(9)
    for jd in 2461253.916666667 + np.concatenate([[0.0, 10.0 / 86400.0], rng.random(200) * 3650.0]):
        assert np.array_equal(ks.moon_position(jd), reference.moon_position(jd))


def test_generator_is_deterministic_and_shaped(ks):
    a = ks.generate_population(20260801, 28340)
    b = ks.generate_population(20260801, 28340)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    st, sz, al = a
    r = np.linalg.norm(st[:, :3], axis=1)
    v = np.linalg.norm(st[:, 3:], axis=1)
    mu = 398600.4418
    energy = v ** 2 / 2 - mu / r
    sma = -mu / (2 * energy)
    leo = (sma < 9000).mean()
    geo = (np.abs(sma - 42164) < 50).mean()
    meo = (np.abs(sma - 26560) < 50).mean()
    assert abs(leo - 0.75) < 0.02 and abs(geo - 0.06) < 0.01 and abs(meo - 0.06) < 0.01
    assert (r > 6378.137 + 200).all()
    radius = sz / 2
    assert radius.min() >= 0.05 and radius.max() <= 15.0
    assert abs(np.median(radius) - 0.5) < 0.03
    assert al.all()


def test_generator_fragment_clouds(ks):
    st, sz, al = ks.generate_population(5, 2000, 12000, 10, 0.0)
    frag = st[2000:]
    assert len(frag) == 10000
    # Released at the epoch: each cloud sits at its parent's position.
    centres = {tuple(np.round(x[:3], 6)) for x in frag}
    assert len(centres) <= 10
    dv = []
    for c in range(10):
        f = frag[1000 * c:1000 * (c + 1)]
        parent = np.where((st[:2000, :3] == f[0, :3]).all(axis=1))[0]
        assert len(parent) == 1
        dv.append(np.linalg.norm(f[:, 3:] - st[parent[0], 3:], axis=1))
    dv = np.concatenate(dv)
    assert abs(np.median(dv) - 0.05) < 0.005
    r = sz[2000:] / 2
    assert r.min() >= 0.05 - 1e-12 and r.max() <= 0.5 + 1e-12
    # exponent -1.6: half of the fragments below ~0.0767 m (median of the truncated law)
    a1 = -0.6
    med = (0.05 ** a1 + 0.5 * (0.5 ** a1 - 0.05 ** a1)) ** (1 / a1)
    assert abs(np.median(r) - med) < 0.003
    aged = ks.generate_population(5, 2000, 12000, 10, 86400.0)[0][2000:]
    assert len({tuple(np.round(x[:3], 6)) for x in aged}) > 9000


def test_checker_generator_equals_engine_generator(ks):
    """The CPU-baseline harness's copy of the generator (oracle/libks_workload.so)
    gives the engine's populations bit for bit."""
    import checkers

    for args in ((7, 500, 500, 1, 0.0), (20260801, 2000, 9000, 12, 86400.0), (3, 300, 4000, 3, 0.0)):
        got = checkers.generate_population(*args)
        want = ks.generate_population(*args)
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
