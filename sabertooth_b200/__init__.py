"""sabertooth_b200: the B200 (sm_100a) alignment hot path of Sabertooth.

Smith-Waterman-Gotoh scoring (packed 16-bit DPX kernel with an exact 32-bit
rescore), batched ungapped diagonal scoring and the prefilter's segment
evidence, chaining and gate, behind a C ABI
(include/sabertooth_b200.h) that mirrors the reference crate's call
signatures.

The residue alphabet, BLOSUM62 (`matrix`) and the ABI record types (`dtypes`)
are plain Python.  Every other name (Context, QueryProfile, score_batch, ...)
comes from `api`, which loads libsabertooth_b200.so on first use and raises
ImportError if it is missing; build it with `python sabertooth_b200/_build.py`.
There is no CPU substitute for any operation.
"""
from .dtypes import CANDIDATE_DTYPE, SEED_HIT_DTYPE
from .matrix import SubstitutionMatrix, blosum62, decode, encode

_API = ("Batch", "Context", "DiagProfile", "GapCosts", "Kernel", "Lane", "Plan", "PrefilterParams", "QueryProfile",
        "SearchServer", "Server", "default_context", "diag_range", "kadane_score", "score_batch", "tile_classes")

__all__ = ["CANDIDATE_DTYPE", "SEED_HIT_DTYPE", "SubstitutionMatrix", "blosum62", "decode", "encode", *_API]


def __getattr__(name):
    if name in _API:
        from . import api
        return getattr(api, name)
    raise AttributeError(f"module 'sabertooth_b200' has no attribute {name!r}")
