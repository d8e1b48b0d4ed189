"""Score + end cell (sw_score_end_with, column-major-first tie rule) and the alignment
span of align_canonical's two score passes, on the GPU, against the oracle.

Known answers restated from the reference's tests:
  * W x 3000 against itself at 11/1: end cell (3000 * s(W,W), 2999, 2999)   src/simd.rs:1229-1233
  * ties: the first optimum in column-major order                         src/simd.rs:1167-1195
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, QueryProfile, blosum62, encode
from sabertooth_b200._lib import PAIR_DTYPE
from tests.refrng import XorShift, rand_seq

pytestmark = pytest.mark.gpu


def _rev_span(rows, t, open_, ext, end):
    """The reference's reverse pass: end cell of the reversed prefixes, mapped back to a start."""
    s, ie, je = end
    r = O.gotoh_score_end(np.ascontiguousarray(rows[: ie + 1][::-1]), np.ascontiguousarray(t[: je + 1][::-1]),
                          open_, ext)
    assert r[0] == s
    return ie - r[1], je - r[2]


def test_end_cell_known_answer_and_plain_per_call(ctx):
    m = blosum62()
    w = int(encode("W")[0])
    q = np.full(3000, w, dtype=np.uint8)
    qp = QueryProfile.from_rows(m.sequence_rows(q), ctx)
    sww = int(m.score[w, w])
    assert qp.sw_score_end(q, GapCosts(11, 1)) == (3000 * sww, 2999, 2999)
    assert qp.sw_score_end(np.zeros(0, np.uint8), GapCosts(11, 1)) is None
    neg = QueryProfile.from_rows(np.full((5, 21), -3, dtype=np.int32), ctx)
    assert neg.sw_score_end(q[:10], GapCosts(11, 1)) is None
    qp.free()
    neg.free()


def test_end_cells_and_spans_match_oracle(ctx):
    m = blosum62()
    rng = XorShift(4242)
    rows_list, targets, pq, pt = [], [], [], []
    for i in range(160):
        alpha = 2 + rng.range(5) if i % 3 == 0 else 20  # small alphabets make ties frequent
        q = rand_seq(rng, 1 + rng.range(400 if i % 10 == 0 else 90), alpha)
        t = rand_seq(rng, 1 + rng.range(700 if i % 10 == 0 else 120), alpha)
        if i % 4 == 0:
            p = rng.range(len(t) + 1)
            t = t[:p] + q + t[p:]
        rows_list.append(m.sequence_rows(q))
        targets.append(np.asarray(t, dtype=np.uint8))
        pq.append(i)
        pt.append(i)
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows_list)
    pairs = np.zeros(len(pq), dtype=PAIR_DTYPE)
    pairs["profile"] = ids[pq]
    pairs["target"] = pt
    pairs["band_radius"] = -1
    try:
        for open_, ext in [(11, 1), (5, 5), (2, 0), (44, 4)]:
            s1, ends1 = ctx.sw_score_end_pairs(pairs, GapCosts(open_, ext))
            s2, starts, ends2 = ctx.align_span_pairs(pairs, GapCosts(open_, ext))
            assert np.array_equal(s1, s2) and np.array_equal(ends1, ends2)
            for i in range(len(pq)):
                want = O.gotoh_score_end(rows_list[i], targets[i], open_, ext)
                if want is None:
                    assert s1[i] == 0 and tuple(ends1[i]) == (-1, -1) and tuple(starts[i]) == (-1, -1)
                    continue
                assert (int(s1[i]), int(ends1[i][0]), int(ends1[i][1])) == want, (i, open_, ext)
                assert tuple(int(x) for x in starts[i]) == _rev_span(rows_list[i], targets[i], open_, ext, want)
        bad = pairs.copy()
        bad["band_radius"][0] = 5
        from sabertooth_b200._lib import StError
        with pytest.raises(StError, match="full local"):
            ctx.sw_score_end_pairs(bad, GapCosts(11, 1))
    finally:
        ctx.free_profiles(ids)
