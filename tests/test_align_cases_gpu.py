"""The reference's alignment test cases, through the GPU score passes.

Traceback itself is out of scope; what the GPU computes for these cases is the
score (batched and per call), the end cell (sw_score_end_with) and the start of
the alignment (the reverse pass of align_canonical). All must equal the oracle:

  * long_gaps_repeats_ties_and_boundaries: a 30-residue insertion, a
    25-residue deletion, tandem repeats, single residues, boundary-touching
    matches, ambiguous residues, empty inputs           src/align.rs:1250-1283
  * v02_traceback_regression_case: WFMMHGWW vs WFMWW at 11/1 src/align.rs:1285-1300
  * large_problem_uses_banded_path_and_matches_reference: 4,500 random
    residues (xorshift seed 42), the target a 2,000-residue random prefix and
    the query's [1000, 3500) mutated with indels up to 8 src/align.rs:1364-1382,
    mutate :1183-1201
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, QueryProfile, blosum62, encode
from sabertooth_b200._lib import PAIR_DTYPE
from tests.refrng import XorShift

pytestmark = pytest.mark.gpu

GAPS = GapCosts(11, 1)  # GapCosts::sequence_default


def _mutate(rng, s, indel_len):
    """mutate (src/align.rs:1183-1201) with the same draws."""
    out, i = [], 0
    while i < len(s):
        r = rng.below(100)
        if r < 4:
            i += 1 + rng.below(indel_len)
            continue
        if r < 8:
            for _ in range(1 + rng.below(indel_len)):
                out.append(rng.below(20))
        out.append(rng.below(20) if r < 30 else s[i])
        i += 1
    return out


def _cases():
    cases = [
        ("MKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIKMKV", "MKVLLACDEFGHIKLMNPQR" + "G" * 30 + "STVWYACDEFGHIKMKV"),
        ("MKVLLACDEFGHIKLMNPQR" + "W" * 25 + "STVWYACDEFGHIK", "MKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIK"),
        ("ACDEFACDEFACDEF", "ACDEFACDEFACDEFACDEFACDEF"),
        ("WWWW", "WWWWWWWWWW"),
        ("W", "W"),
        ("W", "AAAAW"),
        ("A", "W"),
        ("MKVL", "MKVLXXXXMKVL"),
        ("MKXXLLAXCDE", "MKVVLLAXCDE"),
        ("XXXXXX", "XXXXXX"),
        ("WFMMHGWW", "WFMWW"),
    ]
    out = [(encode(q), encode(t)) for q, t in cases]
    rng = XorShift(42)
    q = [rng.below(20) for _ in range(4500)]
    t = _mutate(rng, q[1000:3500], 8)
    pre = [rng.below(20) for _ in range(2000)]
    out.append((np.array(q, dtype=np.uint8), np.array(pre + t, dtype=np.uint8)))
    return out


def _start(rows, t, end):
    """The reverse pass: the end cell of the reversed prefixes, mapped back to a start."""
    s, ie, je = end
    r = O.gotoh_score_end(np.ascontiguousarray(rows[: ie + 1][::-1]), np.ascontiguousarray(t[: je + 1][::-1]),
                          GAPS.open, GAPS.extend)
    assert r[0] == s
    return ie - r[1], je - r[2]


def test_reference_align_cases(ctx):
    m = blosum62()
    cases = _cases()
    assert (4500 + 1) * (len(cases[-1][1]) + 1) > 1 << 22  # FULL_TRACEBACK_MAX_CELLS: the banded path
    rows = [m.sequence_rows(q) for q, _ in cases]
    targets = [t for _, t in cases]
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    pairs = np.zeros(len(cases), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(cases))
    pairs["band_radius"] = -1
    try:
        scores = ctx.sw_score_pairs(pairs, GAPS)
        s_end, ends = ctx.sw_score_end_pairs(pairs, GAPS)
        s_span, starts, ends2 = ctx.align_span_pairs(pairs, GAPS)
        for i, (r, t) in enumerate(zip(rows, targets)):
            want = O.gotoh_score_end(r, t, GAPS.open, GAPS.extend)
            ref = O.gotoh_score(r, t, GAPS.open, GAPS.extend)
            assert int(scores[i]) == ref == int(s_end[i]) == int(s_span[i]), i
            if want is None:
                assert ref == 0 and tuple(ends[i]) == (-1, -1) and tuple(starts[i]) == (-1, -1)
                continue
            assert (int(s_end[i]), int(ends[i][0]), int(ends[i][1])) == want, i
            assert tuple(ends2[i]) == tuple(ends[i])
            assert tuple(int(x) for x in starts[i]) == _start(r, t, want), i
        # the plain per-call path, and empty inputs (local_align returns None: score 0)
        qp = QueryProfile.from_rows(rows[-2], ctx)  # WFMMHGWW
        assert qp.sw_score(targets[-2], GAPS) == int(scores[-2])
        assert qp.sw_score(np.zeros(0, np.uint8), GAPS) == 0
        qp.free()
        empty = QueryProfile.from_rows(np.zeros((0, 21), np.int32), ctx)
        assert empty.sw_score(encode("MKV"), GAPS) == 0
        empty.free()
    finally:
        ctx.free_profiles(ids)
