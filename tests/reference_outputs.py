"""The reference's own recorded search output as score pins (fixtures in tests/golden/).

tests/data/v1_fixture_k2.v03.m8 is a search of the reference's test database
against itself that its test cli_db_equivalence.rs requires the current code
to reproduce: BLOSUM62, gaps 11/1, composition-bias correction on, the scoring
mask on (src/search.rs:432-455, SearchParams::sequence_default).  Each line
prints the bit score (lambda 0.3649, K 0.1076 for 11/1 with the correction,
src/evalue.rs:289-301) to 0.1 bit, which fixes the raw score
S = (bits * ln 2 + ln K) / lambda to within 0.1 of an integer.  The reported
alignment is optimal inside the target window it was computed in, so the
Smith-Waterman score of its span (query rows qstart..qend, target
tstart..tend) equals S exactly.
"""
import json
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def read_fasta(path):
    seqs, name = {}, None
    for ln in open(path):
        ln = ln.strip()
        if ln.startswith(">"):
            name = ln[1:].split()[0]
            seqs[name] = ""
        elif name is not None:
            seqs[name] += ln
    return seqs


def v1_fixture_cases(comp_bias_corr=True, mask_scoring=(15, 2.3, 2.3)):
    """[(rows, target, span, raw score, raw score before rounding)] of every recorded hit; rows are built
    as the reference's search builds them (oracle.search_rows)."""
    from oracle import oracle as O
    from sabertooth_b200 import blosum62, encode
    fx = json.load(open(os.path.join(GOLDEN, "v1_fixture_k2_v03.json")))
    seqs = read_fasta(os.path.join(GOLDEN, "v1_fixture.fa"))
    m = blosum62()
    lam, k = fx["lambda"], fx["k"]
    out = []
    for h in fx["hits"]:
        q = encode(seqs[h["query"]])
        t = np.ascontiguousarray(encode(seqs[h["target"]]), dtype=np.uint8)
        rows = O.search_rows(q, m.score, m.p_back, comp_bias_corr=comp_bias_corr, mask_scoring=mask_scoring)
        s_real = (float(h["bits"]) * math.log(2) + math.log(k)) / lam
        span = (h["qstart"] - 1, h["qend"], h["tstart"] - 1, h["tend"])
        out.append((rows, t, span, int(round(s_real)), s_real))
    return out
