"""Host-side inputs pinned against the reference's fixtures and matrix tests (CPU).

* The PSSM built from demo/family.a3m equals the reference's demo/family.pssm
  cell for cell (tests/golden/, made by tests/golden/make_golden.py).
* The BLOSUM62 reconstruction passes the reference's matrix tests
  (src/matrix.rs:213-240).
* MSA parsing errors as the reference's profile tests require (src/profile.rs:460-531).
"""
import json
import os

import numpy as np
import pytest

from sabertooth_b200 import blosum62, encode
from synth.profile import Profile, parse_msa

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_family_pssm_matches_reference_output():
    g = json.load(open(os.path.join(GOLD, "family_pssm.json")))
    p = Profile.from_msa_str(open(os.path.join(GOLD, "family.a3m")).read())
    assert p.pssm.shape == (len(g["pssm"]), 20)
    assert np.array_equal(p.pssm, np.array(g["pssm"], dtype=np.int8))
    assert np.allclose(np.round(p.neff.astype(np.float64), 2), g["neff_2dp"], atol=1e-6)
    assert "".join("ACDEFGHIKLMNPQRSTVWYX"[c] for c in p.query_num) == g["query"]


def test_blosum62_reference_properties():
    m = blosum62()
    w, a = int(encode("W")[0]), int(encode("A")[0])
    assert m.score[w, w] > m.score[a, a]
    assert all(m.score[i, i] > 0 for i in range(20))
    assert np.all(np.abs(m.r.sum(axis=0) - 1.0) < 0.02)
    assert abs(m.p_back[:20].sum() - 1.0) < 0.01
    assert np.array_equal(m.score, m.score.T)
    assert m.score[20].tolist() == [-1] * 21


def test_profile_rows_score_x_as_zero():
    p = Profile.from_msa_str(">q\nMKVLA\n")
    rows = p.rows()
    assert rows.shape == (5, 21) and np.all(rows[:, 20] == 0)
    assert p.pssm[0, int(encode("M")[0])] > p.pssm[0, int(encode("P")[0])]


def test_msa_errors():
    with pytest.raises(ValueError):
        parse_msa("")
    with pytest.raises(ValueError):
        parse_msa(">q\nMKVLA\n>bad\nMKVLAaG\n")
    msa, L = parse_msa(">q\nMKVLA\n>h\nMKaVLA\n")
    assert L == 5 and msa.shape == (2, 5)
