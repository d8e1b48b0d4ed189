"""The oracle against the reference's own recorded search output (CPU).

88 hits of tests/data/v1_fixture_k2.v03.m8 (see tests/reference_outputs.py):
for every hit the oracle's scalar Gotoh (src/simd.rs:347-390) over the
alignment span, with the rows built by the restated composition-bias
correction (src/compbias.rs:38-70) and scoring mask (src/mask.rs:68-128),
equals the raw score the reference printed; so does the whole pair's score.
Without the correction almost every score differs, so the pin exercises the
row preparation as well as the recurrence.
"""
import numpy as np

from oracle import oracle as O
from sabertooth_b200 import blosum62, encode
from tests.reference_outputs import v1_fixture_cases


def test_recorded_raw_scores_are_recovered_exactly_from_the_bits():
    cases = v1_fixture_cases()
    assert len(cases) == 88
    for _, _, _, s, s_real in cases:
        assert abs(s_real - s) < 0.2


def test_span_and_whole_pair_scores_equal_the_recorded_raw_scores():
    for rows, t, (q0, q1, t0, t1), s, _ in v1_fixture_cases():
        assert O.gotoh_score(rows[q0:q1], t[t0:t1], 11, 1) == s
        assert O.gotoh_score(rows, t, 11, 1) == s
        assert O.reference_score(rows, t, 11, 1) == s


def test_the_pin_depends_on_the_composition_bias_rows():
    wrong = sum(O.gotoh_score(rows[q0:q1], t[t0:t1], 11, 1) != s
                for rows, t, (q0, q1, t0, t1), s, _ in v1_fixture_cases(comp_bias_corr=False))
    assert wrong >= 80


def test_comp_bias_known_answers():
    # src/compbias.rs:91-106
    m = blosum62()
    c = O.comp_bias(encode("Q" * 60), m.score, m.p_back)
    assert np.all(c <= -5)
    c2 = O.comp_bias(encode("MKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIKLMNPQRSTVWYMKVLLAC"), m.score, m.p_back)
    assert abs(c2.mean()) < 1.5
    assert O.comp_bias(encode(""), m.score, m.p_back).size == 0
    assert O.comp_bias(encode("W"), m.score, m.p_back).size == 1


def test_low_complexity_mask_known_answers():
    # src/mask.rs:141-171 with MaskParams::default() (12, 2.2, 2.5)
    s = encode("MKVLLACDEFGHIK" + "Q" * 30 + "MKVLLACDEFGHIK")
    mk = O.low_complexity_mask(s, 12, 2.2, 2.5)
    assert mk[14:44].all() and not mk[:8].any()
    r = encode("MKVLLACDEFGHIKLMNPQRSTVWY" + "GPP" * 10 + "ACDEFGHIKLMNPQRSTVWY")
    assert O.low_complexity_mask(r, 12, 2.2, 2.5).sum() >= 30
    k = encode("MADENKLKLGSGSFGEVFLVKHKESGNIYAMKKIRLEVEEEGVPSTAIREISLLKELKHENIVRLYDVVHSDKKLTLVFEYLDKDLKKYMDS"
               "CPEFAKDPRLIKMFLYQILRGLAYCHRRKVLHRDLKPQNLLIDRRTNSLKLADFGLARAFGVPLRTYTHEVVTLWYRAPEILLG")
    assert O.low_complexity_mask(k, 12, 2.2, 2.5).mean() < 0.1
    assert not O.low_complexity_mask(encode("QQQQQ"), 12, 2.2, 2.5).any()
