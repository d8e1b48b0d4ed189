"""sabertooth_b200: the B200 (sm_100a) alignment hot path of Sabertooth.

Smith-Waterman-Gotoh scoring (packed 16-bit DPX kernel with an exact 32-bit
rescore) and batched ungapped diagonal scoring, behind a C ABI
(include/sabertooth_b200.h) that mirrors the reference crate's call
signatures.  Importing the package loads libsabertooth_b200.so and fails if it
is missing; build it with `python sabertooth_b200/_build.py`.
"""
from .api import (Batch, Context, DiagProfile, GapCosts, Kernel, Lane, Plan, QueryProfile, Server, default_context,
                  diag_range, kadane_score, score_batch, tile_classes)
from .matrix import SubstitutionMatrix, blosum62, decode, encode

__all__ = ["Context", "DiagProfile", "GapCosts", "Kernel", "Lane", "Plan", "QueryProfile", "default_context",
           "diag_range", "kadane_score", "score_batch", "tile_classes", "SubstitutionMatrix", "blosum62",
           "decode", "encode"]
