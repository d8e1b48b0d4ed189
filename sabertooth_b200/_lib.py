"""ctypes binding of libsabertooth_b200.so (the C ABI in include/sabertooth_b200.h).

The library is required: importing this module without it raises, and no
operation of this package has a CPU substitute.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsabertooth_b200.so")

ST_OK = 0
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ETIMEOUT", -5: "ESTATE"}


class StError(RuntimeError):
    """A failed C-ABI call: .code is the ST_E* status."""

    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class st_pair(C.Structure):
    _fields_ = [("profile", C.c_uint32), ("target", C.c_uint32), ("band_center", C.c_int32),
                ("band_radius", C.c_int32)]


class st_lane(C.Structure):
    _fields_ = [("target", C.c_uint32), ("lo", C.c_uint32), ("hi", C.c_uint32), ("diag", C.c_int32)]


class st_lane_slice(C.Structure):
    _fields_ = [("target", C.c_void_p), ("len", C.c_uint64), ("diag", C.c_int64), ("lo", C.c_uint64),
                ("hi", C.c_uint64)]


class st_hit(C.Structure):
    _fields_ = [("query", C.c_uint32), ("target", C.c_uint32), ("diag", C.c_int32)]


from .dtypes import CANDIDATE_DTYPE, HIT_DTYPE, LANE_DTYPE, PAIR_DTYPE, SEED_HIT_DTYPE  # noqa: E402,F401
PREFILTER_STATS_FIELDS = ("targets_hit", "targets_evaluated", "diagonals_scored", "chains_used", "candidates",
                          "candidates_capped", "hits_rejected")


class PrefilterParamsC(C.Structure):
    _fields_ = [("min_hits", C.c_uint32), ("diag_hits", C.c_uint32), ("max_diagonals", C.c_uint32),
                ("diag_window", C.c_uint32), ("span", C.c_uint32), ("min_diag_score", C.c_int32),
                ("gap_open", C.c_int32), ("gap_ext", C.c_int32), ("max_candidates", C.c_uint32),
                ("regions", C.c_uint32)]


class CalibrationC(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("k", C.c_double), ("mu", C.c_double), ("n", C.c_uint32),
                ("ok", C.c_int32)]


class SeedParamsC(C.Structure):
    _fields_ = [("kmer_score", C.c_int32), ("max_kmers_per_pos", C.c_uint32), ("exact_seeds", C.c_uint32),
                ("max_seed_occ", C.c_uint32)]


SEED_STATS_FIELDS = ("windows", "windows_skipped", "kmers_generated", "windows_at_cap", "exact_seeds_added", "seeds",
                     "postings_visited", "seeds_over_occ_cap", "postings_skipped_occ")


class SeedStatsC(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in SEED_STATS_FIELDS]


class PrefilterStatsC(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in PREFILTER_STATS_FIELDS]

_P = C.c_void_p
_u32, _i32, _u64, _i64, _sz = C.c_uint32, C.c_int32, C.c_uint64, C.c_int64, C.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "st_init": (_P, [C.c_int, _sz]),
    "st_shutdown": (None, [_P]),
    "st_last_error": (C.c_char_p, []),
    "st_set_stream": (C.c_int, [_P, _P]),
    "st_synchronize": (C.c_int, [_P]),
    "st_mem_used": (C.c_int, [_P, _P]),
    "st_db_upload": (C.c_int, [_P, _P, _P, _u32]),
    "st_db_info": (C.c_int, [_P, _P, _P]),
    "st_profile_create": (C.c_int, [_P, _P, _u32, _P]),
    "st_profile_free": (C.c_int, [_P, _u32]),
    "st_profiles_free": (C.c_int, [_P, _P, _u32]),
    "st_sw_score_pairs_async": (C.c_int, [_P, _P, _u64, _i32, _i32, _P, _P, _P]),
    "st_batch_wait": (C.c_int, [_P]),
    "st_sw_score_end": (C.c_int, [_P, _u32, _P, _u32, _i32, _i32, _P, _P, _P]),
    "st_sw_score_end_pairs": (C.c_int, [_P, _P, _u64, _i32, _i32, _P, _P]),
    "st_sw_align_span_pairs": (C.c_int, [_P, _P, _u64, _i32, _i32, _P, _P, _P]),
    "st_batch_query": (C.c_int, [_P]),
    "st_server_create": (_P, [_P, _i32, _i32, _u64, _u64]),
    "st_server_submit": (C.c_int, [_P, _P, _u32, _P, _P, _P, _u32, _P]),
    "st_server_submit_many": (C.c_int, [_P, _u32, _P, _P, _P, _P, _P, _P, _P]),
    "st_server_wait": (C.c_int, [_P, _u64, _P, _u32, _P]),
    "st_server_stats": (C.c_int, [_P, _P, _P]),
    "st_server_destroy": (None, [_P]),
    "st_profiles_create": (C.c_int, [_P, _P, _P, _u32, _P]),
    "st_sw_score": (C.c_int, [_P, _u32, _P, _u32, _i32, _i32, _P, _P]),
    "st_sw_score_pairs": (C.c_int, [_P, _P, _u64, _i32, _i32, _P, _P]),
    "st_plan_create": (C.c_int, [_P, _P, _u64, _i32, _i32, _P, _P, _P]),
    "st_plan_run": (C.c_int, [_P]),
    "st_plan_stats": (C.c_int, [_P, _P, _P, _P]),
    "st_plan_profile": (C.c_int, [_P, _u32, _P, _P, _P, _P]),
    "st_plan_destroy": (None, [_P]),
    "st_ungapped_score": (C.c_int, [_P, _u32, _P, _u32, _P]),
    "st_ungapped_score_slices": (C.c_int, [_P, _u32, _P, _u32, _P]),
    "st_ungapped_hits": (C.c_int, [_P, _P, _u64, _P, _P, _P, _P, _P]),
    "st_ungapped_hits_device": (C.c_int, [_P, _P, _u64, _P, _P, _P, _P, _P]),
    "st_prefilter_gate": (C.c_int, [_P, _P, _u64, _P, _P, _u64, _P, _P]),
    "st_prefilter_gate_device": (C.c_int, [_P, _P, _u64, _P, _P, _P, _P]),
    "st_calibrate_profiles": (C.c_int, [_P, _P, _u32, _P, _u32, _u32, _u64, _P, _i32, _i32, _P, _P]),
    "st_seed_index_build": (C.c_int, [_P, C.c_char_p]),
    "st_search_server_create": (_P, [_P, _P, _P, C.c_int, _u32]),
    "st_search_server_submit": (C.c_int, [_P, _P, _u32, _P, _P]),
    "st_search_server_wait": (C.c_int, [_P, _u64, _P, _P, _u64, _P, _P]),
    "st_search_server_stats": (C.c_int, [_P, _P, _P]),
    "st_search_server_destroy": (None, [_P]),
    "st_seed_hits": (C.c_int, [_P, _P, _u32, _P, _P, _P, _P, _u64, _P, _P]),
    "st_prefilter_queries": (C.c_int, [_P, _P, _u32, _P, _P, _P, _P, _P, _u64, _P, _P, _P]),
    "st_tune_num_classes": (C.c_int, []),
    "st_tune_class_shape": (C.c_int, [C.c_int, _P, _P, _P]),
    "st_tune_get": (C.c_int, [_P, _P]),
    "st_tune_set": (C.c_int, [_P, _P]),
    "st_tune_get_rates": (C.c_int, [_P, _P, _u32]),
    "st_tune_set_rates": (C.c_int, [_P, _P, _u32]),
    "st_autotune": (C.c_int, [_P, _P, _u64, _i32, _i32, _u32, _P]),
    "st_sw_score_noalloc": (C.c_int, [_P, _u32, _P, _u32, _i32, _i32, _P, _P]),
    "st_probe_dpx": (C.c_int, [_P, _P]),
    "st_launch_count": (C.c_int, [_P, _P]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python sabertooth_b200/_build.py` "
            "(the package has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status):
    if status != ST_OK:
        msg = lib.st_last_error()
        raise StError(status, msg.decode() if msg else "")
    return status


def ptr(a):
    """Address of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data
