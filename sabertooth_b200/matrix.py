"""Residue alphabet and the BLOSUM62 integer matrix (reference src/alphabet.rs, src/matrix.rs).

The matrix data (data/blosum62.json) is regenerated from the reference's
blosum62.out by data/make_blosum62.py, which restates
SubstitutionMatrix::from_out_str (src/matrix.rs:56-175).
"""
import json
import os

import numpy as np

LETTERS = "ACDEFGHIKLMNPQRSTVWYX"  # src/alphabet.rs:8-10
PROFILE_AA_SIZE = 20               # src/alphabet.rs:17
ALPHABET_SIZE = 21                 # src/alphabet.rs:20
ANY = 20                           # X
GAP = 0xFF                         # src/alphabet.rs:36


def build_aa2num():
    """ASCII -> residue code; ambiguity codes and unknown bytes -> X (src/alphabet.rs:41-50)."""
    t = np.full(256, ANY, dtype=np.uint8)
    for i, ch in enumerate(LETTERS):
        t[ord(ch)] = i
        t[ord(ch.lower())] = i
    return t


AA2NUM = build_aa2num()


def encode(seq: str) -> np.ndarray:
    return AA2NUM[np.frombuffer(seq.encode("ascii"), dtype=np.uint8)]


def decode(codes) -> str:
    return "".join(LETTERS[c] if c < ALPHABET_SIZE else "-" for c in np.asarray(codes))


class SubstitutionMatrix:
    """The reconstructed integer matrix with its probabilities (src/matrix.rs:24-45)."""

    def __init__(self, d):
        self.name = d["name"]
        self.score = np.array(d["score"], dtype=np.int8)          # [21][21]
        self.p_back = np.array(d["p_back"], dtype=np.float64)     # [21]
        self.prob = np.array(d["prob"], dtype=np.float64)         # [21][21] joint P(a,b)
        self.r = np.array(d["r"], dtype=np.float32)               # [20][20] P(a|b)
        self.lam = float(d["lambda"])
        self.bit_factor = float(d["bit_factor"])
        self.bias = float(d["bias"])

    @staticmethod
    def blosum62():
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "blosum62.json")) as f:
            return SubstitutionMatrix(json.load(f))

    def sequence_rows(self, query_codes) -> np.ndarray:
        """ScoreTable rows of a sequence query: rows[i][r] = score[q_i][r] (SeqScorer, src/align.rs:61-79)."""
        q = np.asarray(query_codes, dtype=np.int64)
        if q.size and q.max() >= ALPHABET_SIZE:
            raise ValueError("query codes must be < 21")
        return np.ascontiguousarray(self.score[q].astype(np.int32))


_BLOSUM62 = None


def blosum62() -> SubstitutionMatrix:
    global _BLOSUM62
    if _BLOSUM62 is None:
        _BLOSUM62 = SubstitutionMatrix.blosum62()
    return _BLOSUM62
