"""sabertooth_b200: the B200 (sm_100a) alignment hot path of Sabertooth.

Smith-Waterman-Gotoh scoring (packed 16-bit DPX kernel with an exact 32-bit
rescore), batched ungapped diagonal scoring and the prefilter's segment
evidence, chaining and gate, behind a C ABI
(include/sabertooth_b200.h) that mirrors the reference crate's call
signatures.  Importing the package loads libsabertooth_b200.so and fails if it
is missing; build it with `python sabertooth_b200/_build.py`.
"""
from ._lib import CANDIDATE_DTYPE, SEED_HIT_DTYPE
from .api import (Batch, Context, DiagProfile, GapCosts, Kernel, Lane, Plan, PrefilterParams, QueryProfile, SearchServer, Server,
                  default_context, diag_range, kadane_score, score_batch, tile_classes)
from .matrix import SubstitutionMatrix, blosum62, decode, encode

__all__ = ["Batch", "CANDIDATE_DTYPE", "PrefilterParams", "SEED_HIT_DTYPE", "SearchServer", "Server", "Context", "DiagProfile", "GapCosts", "Kernel", "Lane", "Plan", "QueryProfile", "default_context",
           "diag_range", "kadane_score", "score_batch", "tile_classes", "SubstitutionMatrix", "blosum62",
           "decode", "encode"]
