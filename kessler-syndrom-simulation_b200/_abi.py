"""ctypes declarations of the C ABI in include/kessler_b200.h.

The shared library is built in-tree (``make -C kessler-syndrom-simulation_b200``).
Loading fails loudly when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkessler_b200.so")

CONJ_DTYPE = np.dtype(
    [("i", "<i4"), ("j", "<i4"), ("step", "<i8"), ("t", "<f8"), ("miss_km", "<f8"),
     ("v_rel_km_s", "<f8"), ("collision", "<i4"), ("realisation", "<i4")], align=True)
STATS_DTYPE = np.dtype(
    [("step", "<i8"), ("candidate_pairs", "<i8"), ("refined_pairs", "<i8"), ("co_orbiting", "<i8"),
     ("conjunctions", "<i8"), ("cell_km", "<f8"), ("max_cell_objects", "<i4"), ("alive", "<i4")],
    align=True)
BREAKUP_DTYPE = np.dtype(
    [("step", "<i8"), ("t", "<f8"), ("id", "<i4"), ("realisation", "<i4"), ("target", "<i8"), ("projectile", "<i8"),
     ("catastrophic", "<i4"), ("fragments", "<i4"), ("escaped", "<i4"), ("pad", "<i4"), ("first_fragment", "<i8"),
     ("v_rel_km_s", "<f8"), ("energy_j_per_g", "<f8"), ("target_mass_kg", "<f8"), ("projectile_mass_kg", "<f8"),
     ("sbm_mass_kg", "<f8"), ("expected_fragments", "<f8"), ("fragments_mass_kg", "<f8"), ("position", "<f8", (3,))],
    align=True)
assert CONJ_DTYPE.itemsize == 48 and STATS_DTYPE.itemsize == 56 and BREAKUP_DTYPE.itemsize == 144


class Timing(C.Structure):
    _fields_ = [("propagate_ms", C.c_double), ("sort_ms", C.c_double), ("cells_ms", C.c_double),
                ("pairs_ms", C.c_double), ("refine_ms", C.c_double), ("total_ms", C.c_double),
                ("steps", C.c_int64), ("object_steps", C.c_int64), ("sort_passes", C.c_int64),
                ("candidate_pairs", C.c_int64), ("exact_filter_pairs", C.c_int64), ("refined_pairs", C.c_int64),
                ("chunk_ms", C.c_double), ("sort_cells_fused", C.c_int64),
                ("host_chunk_ms", C.c_double), ("host_prep_ms", C.c_double), ("host_launch_ms", C.c_double),
                ("host_sync_ms", C.c_double)]


class TuningChoice(C.Structure):
    _fields_ = [("steps_per_graph", C.c_int32), ("pair_variant", C.c_int32), ("pair_blocks_per_sm", C.c_int32),
                ("subcell_bits", C.c_int32), ("box_min_rows", C.c_int32), ("cell_scale_permille", C.c_int32),
                ("prop_block", C.c_int32), ("item_col_blocks", C.c_int32), ("trials", C.c_int32),
                ("ms_per_step_start", C.c_double),
                ("ms_per_step_best", C.c_double)]


KS_OK = 0
STATUS_NAMES = {0: "KS_OK", 1: "KS_ERR_ARG", 2: "KS_ERR_CUDA", 3: "KS_ERR_NO_DEVICE", 4: "KS_ERR_STATE",
                5: "KS_ERR_OVERFLOW", 6: "KS_ERR_RANGE", 7: "KS_ERR_TIMEOUT"}
PRECISION_FP64 = 0
PRECISION_SPLIT = 1

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "ks_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "ks_destroy": (None, [_P]),
    "ks_last_error": (C.c_char_p, [_P]),
    "ks_device_name": (C.c_char_p, [_P]),
    "ks_stream": (_P, [_P]),
    "ks_set_population": (C.c_int, [_P, _I64, _P, _P, _P]),
    "ks_set_population_batch": (C.c_int, [_P, C.c_int32, _P, _P, _P, _P]),
    "ks_get_population": (C.c_int, [_P, _I64, _P, _P]),
    "ks_population_size": (_I64, [_P]),
    "ks_set_clock": (C.c_int, [_P, _D, _D, _D]),
    "ks_get_clock": (C.c_int, [_P, C.POINTER(_D), C.POINTER(_I64)]),
    "ks_set_screening": (C.c_int, [_P, C.c_int, _D, _D, _D]),
    "ks_set_precision": (C.c_int, [_P, C.c_int]),
    "ks_set_steps_per_graph": (C.c_int, [_P, C.c_int]),
    "ks_set_profiling": (C.c_int, [_P, C.c_int]),
    "ks_set_buffer_limits": (C.c_int, [_P, _I64, _I64]),
    "ks_set_l2_flush": (C.c_int, [_P, _I64]),
    "ks_set_tuning": (C.c_int, [_P, C.c_char_p, _I64]),
    "ks_run": (C.c_int, [_P, _I64]),
    "ks_prepare_run": (C.c_int, [_P]),
    "ks_autotune": (C.c_int, [_P, C.c_int32, C.POINTER(TuningChoice)]),
    "ks_take_conjunctions": (C.c_int, [_P, _P, _I64, C.POINTER(_I64)]),
    "ks_take_conjunctions_view": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_I64)]),
    "ks_take_step_stats": (C.c_int, [_P, _P, _I64, C.POINTER(_I64)]),
    "ks_set_breakup": (C.c_int, [_P, C.c_int, _D, _D, C.c_uint64]),
    "ks_set_masses": (C.c_int, [_P, _I64, _P]),
    "ks_set_breakup_mode": (C.c_int, [_P, C.c_int, _I64]),
    "ks_impact": (C.c_int, [_P, _I64, _D, _D]),
    "ks_take_breakups": (C.c_int, [_P, _P, _I64, C.POINTER(_I64)]),
    "ks_save_population": (C.c_int, [_P, C.c_char_p]),
    "ks_load_population": (C.c_int, [_P, C.c_char_p]),
    "ks_sbm_impact": (_I64, [C.c_uint64, _D, _D, _P, _D, _D, _D, _D, _D, _P, _P, _P, _P, _P, _I64, _P]),
    "ks_get_objects": (C.c_int, [_P, _I64, _P, _P, _P, _P, _P]),
    "ks_screen": (C.c_int, [_P, _I64, _P, _P, _P, _P, _D, _D, _P, _I64, C.POINTER(_I64), _P]),
    "ks_propagate": (C.c_int, [_P, _I64, _P, _P, _D, _D, _D, _I64]),
    "ks_screen_noalloc": (C.c_int, [_I64, _P, _P, _P, _P, _D, _D, _D, _D, _D, _P, _I64, C.POINTER(_I64), _P, _P,
                                    C.c_char_p, _I64]),
    "ks_get_timing": (C.c_int, [_P, C.POINTER(Timing)]),
    "ks_moon_position": (None, [_D, _P]),
    "ks_generate_population": (C.c_int, [C.c_uint64, _I64, _I64, C.c_int, _D, _P, _P, _P]),
    "ks_measure_fp64": (C.c_int, [_P, C.POINTER(_D), C.POINTER(_D)]),
    "ks_measure_fp32": (C.c_int, [_P, C.POINTER(_D), C.POINTER(_D)]),
    "ks_measure_fp32x2": (C.c_int, [_P, C.POINTER(_D)]),
}

_lib = None


def load_library(path=LIB_PATH):
    """Loads libkessler_b200.so and declares every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `make -C {HERE}` (or __graft_entry__.build()). "
            "The engine has no CPU fallback.")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """Raw data pointer of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)
