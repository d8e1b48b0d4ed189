"""Oracle of the prefilter evidence / chain / gate stage, pinned on the CPU.

* The reference's own prefilter tests restated on brute-force seed hits
  (src/prefilter.rs:1926-1959 diagonal_mode_is_selected and
  second_diagonal_and_chain_rescue_indel_split_homolog; the cap semantics of
  target_blocks_give_identical_candidates :1961-2005).
* The C oracle (scalar and AVX2-batched scoring) against the literal Python
  restatement in tests/seedhits.py on random cases with planted split homologs.
"""
import numpy as np
import pytest

import oracle.oracle as O
from sabertooth_b200 import blosum62, encode
from synth import workloads as W
from tests.seedhits import brute_seed_hits, default_params, py_prefilter, similar_kmer_count


def _run_oracle(rows, targets, hits, p, simd=True):
    a = O.Arena([rows], targets)
    h = np.array(hits, dtype=np.int64).reshape(-1, 4)
    return O.prefilter_queries(a, h[:, 0], h[:, 1], h[:, 2], h[:, 3], p, simd=simd)


def _tuples(c):
    return [tuple(int(x) for x in r) for r in c]


def test_diagonal_mode_is_selected():
    # src/prefilter.rs:1926-1935: k = 6, kmer_score 22, default parameters
    m = blosum62()
    q = encode("MKVLLACDEFGHIK")
    t = encode("MKVLLACDEFGHIKMKVLLAC")
    hits = brute_seed_hits(m.score, q, [t], 6, 22)
    c, st = _run_oracle(m.sequence_rows(q), [t], hits, default_params(span=6))
    assert len(c) > 0
    assert c[0]["diag_score"] > 0
    assert c[0]["best_diag"] == 0


def test_chain_rescues_indel_split_homolog():
    # src/prefilter.rs:1937-1959: a repeat on the most frequent (wrong) diagonal
    # plus the real homology split by a 4-residue insertion; four diagonals with
    # the chain score above the single most-frequent diagonal
    m = blosum62()
    q = encode("MKVLLACDEFGHIKLMNPQRSTVWYHHHHWWCCMM")
    t = encode("QRSTQRSTQRSTQRSTQRSTQRSTQRST" + "MKVLLACDEFGHIKLMNP" + "GGGGQRSTVWYHHHHWWCCMM")
    assert similar_kmer_count(m.score, q, 4, 18) <= 512  # brute force == the reference's generator here
    hits = brute_seed_hits(m.score, q, [t], 4, 18)
    rows = m.sequence_rows(q)
    one, _ = _run_oracle(rows, [t], hits, default_params(span=4, max_diagonals=1))
    four, st4 = _run_oracle(rows, [t], hits, default_params(span=4))
    assert len(four) == 1
    assert four[0]["diag_score"] > (int(one[0]["diag_score"]) if len(one) else 0)
    assert st4["chains_used"] == 1
    # the literal restatement agrees field by field
    ref, st = py_prefilter(rows, [t], [(h[1], h[2], h[3]) for h in hits], default_params(span=4))
    assert _tuples(four) == ref


def test_candidate_cap_keeps_the_ranked_prefix():
    # src/prefilter.rs:1990-1996: max_candidates = 10 returns the first 10 of the full ranking
    w = W.seed_hits(seed=4, n_queries=3, n_targets=400, n_hits=6000, homolog_frac=0.5)
    a = O.Arena(w.rows, [w.db_residues[int(w.db_offsets[i]):int(w.db_offsets[i + 1])]
                         for i in range(len(w.db_offsets) - 1)])
    h = w.hits
    p = default_params(min_diag_score=20)
    full, sf = O.prefilter_queries(a, h["query"], h["target"], h["diag"], h["qpos"], p)
    capped, sc = O.prefilter_queries(a, h["query"], h["target"], h["diag"], h["qpos"], dict(p, max_candidates=10))
    for q in np.unique(full["query"]):
        f = full[full["query"] == q]
        c = capped[capped["query"] == q]
        assert len(c) == min(10, len(f))
        assert (c == f[:len(c)]).all()
    assert sc["candidates_capped"] == sf["candidates"] - sc["candidates"]


@pytest.mark.parametrize("kw", [dict(), dict(diag_window=0), dict(max_diagonals=1), dict(max_diagonals=20),
                                dict(diag_hits=2, min_hits=2), dict(regions=1), dict(min_diag_score=0, regions=1),
                                dict(max_candidates=3, regions=1)])
def test_oracle_matches_literal_restatement(kw):
    w = W.seed_hits(seed=7, n_queries=4, n_targets=120, n_hits=3000, homolog_frac=0.4, keep=0.7)
    targets = [w.db_residues[int(w.db_offsets[i]):int(w.db_offsets[i + 1])] for i in range(len(w.db_offsets) - 1)]
    a = O.Arena(w.rows, targets)
    h = w.hits
    p = default_params(**dict(dict(min_diag_score=25), **kw))
    got, st = O.prefilter_queries(a, h["query"], h["target"], h["diag"], h["qpos"], p, simd=True)
    got0, st0 = O.prefilter_queries(a, h["query"], h["target"], h["diag"], h["qpos"], p, simd=False)
    assert (got == got0).all() and st == st0
    ref, tot = [], {}
    for q in range(len(w.rows)):
        sel = h["query"] == q
        r, s = py_prefilter(w.rows[q], targets, list(zip(h["target"][sel], h["diag"][sel], h["qpos"][sel])), p,
                            query_id=q)
        ref += r
        for k, v in s.items():
            tot[k] = tot.get(k, 0) + v
    assert _tuples(got) == ref
    assert st == tot


def test_oracle_chains_on_split_homologs():
    # the generator's two-piece homologs must exercise the chain rule
    w = W.seed_hits(seed=11, n_queries=6, n_targets=300, n_hits=20000, homolog_frac=0.5, keep=0.8)
    targets = [w.db_residues[int(w.db_offsets[i]):int(w.db_offsets[i + 1])] for i in range(len(w.db_offsets) - 1)]
    a = O.Arena(w.rows, targets)
    h = w.hits
    _, st = O.prefilter_queries(a, h["query"], h["target"], h["diag"], h["qpos"], default_params(regions=1))
    assert st["chains_used"] > 0
    assert st["candidates"] > 0


def test_oracle_rows_above_u8_limit():
    # PSSM-like rows outside the u8 profile: the AVX2 batch falls back to scalar Kadane
    rng = np.random.default_rng(3)
    rows = rng.integers(-300, 400, size=(60, 21)).astype(np.int32)
    targets = [rng.integers(0, 21, size=int(rng.integers(30, 200))).astype(np.uint8) for _ in range(30)]
    hits = []
    for _ in range(500):
        t = int(rng.integers(0, 30))
        qp = int(rng.integers(0, 60))
        tp = int(rng.integers(0, len(targets[t])))
        hits.append((0, t, tp - qp, qp))
    p = default_params(min_diag_score=500, regions=1)
    c1, s1 = _run_oracle(rows, targets, hits, p, simd=True)
    c0, s0 = _run_oracle(rows, targets, hits, p, simd=False)
    ref, st = py_prefilter(rows, targets, [(x[1], x[2], x[3]) for x in hits], p)
    assert _tuples(c1) == _tuples(c0) == ref
    assert s1 == s0 == st
