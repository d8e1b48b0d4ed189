"""Oracle of the seed stage (similar k-mers, seed index, hits), pinned on the CPU
by the reference's own prefilter tests (src/prefilter.rs):

* top_kmers_is_exact_global_order (:1754-1812): brute force over all 20^w
  k-mers (w = 2..4, SplitMix64 seed 11, caps 1..100,000) in canonical order,
  for the best-first restatement (that order) and the reference's default
  depth-first generator with cap_boundary (the same set, in walk order);
* old_dfs_generator_was_not_globally_ordered (:1839-1857): the global top-2;
* exact_kmer_is_found, exact_seed_below_threshold_is_kept,
  similar_kmer_reaches_diverged_target, profile_prefilter_finds_target,
  diagonal_mode_is_selected, second_diagonal_and_chain_rescue_indel_split_homolog,
  spaced_seed_finds_what_contiguous_misses (:1859-1959, 2042-2059): the whole
  prefilter (seeds -> hits -> evidence -> gate) on their sequences;
* the oracle's hits against a literal brute force of the same definition.
"""
import numpy as np

import oracle.oracle as O
from sabertooth_b200 import blosum62, encode
from synth.profile import Profile
from tests.refrng import SplitMix64
from tests.seedhits import default_params


def test_top_kmers_is_exact_global_order():
    rng = SplitMix64(11)
    capped_cases = 0
    for w in range(2, 5):
        for case in range(40):
            spread = 15 if case % 2 == 0 else 4
            rows = np.array([[rng.below(spread) - spread // 2 for _ in range(21)] for _ in range(w)], dtype=np.int32)
            thr = rng.below(10) - 3
            codes = np.arange(20 ** w, dtype=np.int64)
            sc = np.zeros(20 ** w, dtype=np.int64)
            x = codes.copy()
            for i in range(w - 1, -1, -1):
                sc += rows[i][x % 20]
                x //= 20
            keep = np.nonzero(sc >= thr)[0]
            # canonical order: score descending, then the rank vector (each position's residues ranked by
            # score descending, residue ascending) ascending
            rank = np.zeros((w, 20), dtype=np.int64)
            for i in range(w):
                order = sorted(range(20), key=lambda r: (-int(rows[i][r]), r))
                rank[i][order] = np.arange(20)
            digits = [(keep // 20 ** (w - 1 - i)) % 20 for i in range(w)]
            cols = [rank[i][digits[i]] for i in range(w)]
            order = np.lexsort(cols[::-1] + [-sc[keep]])
            allk = [(-int(sc[c]), None, int(c)) for c in keep[order]]
            for cap in (1, 2, 5, 50, 333, 100000):
                want = [(c, -s) for s, _, c in allk[:cap]]
                got_c, got_s, capped = O.top_kmers(rows, thr, cap)
                assert list(zip(got_c.tolist(), got_s.tolist())) == want, (w, case, cap)
                assert capped == (len(allk) > cap)
                capped_cases += capped
                # the reference's default depth-first generator: the same set, in walk order
                d_c, d_s, d_capped = O.top_kmers_dfs(rows, thr, cap)
                assert sorted(zip(d_c.tolist(), d_s.tolist())) == sorted(want), (w, case, cap)
                assert d_capped == capped
                if not capped:
                    walk = sorted(range(len(keep)), key=lambda k: [int(cc[k]) for cc in cols])
                    assert d_c.tolist() == [int(keep[k]) for k in walk]
    assert capped_cases > 100


def test_old_dfs_generator_was_not_globally_ordered():
    r0 = np.full(21, -10, np.int32)
    r0[0], r0[1] = 10, 9
    r1 = np.full(21, -10, np.int32)
    r1[0], r1[1] = 10, 0
    c, s, _ = O.top_kmers(np.stack([r0, r1]), 0, 2)
    assert sorted(zip(c.tolist(), s.tolist())) == [(0, 20), (20, 19)]


def prefilter(rows, residues, targets, mask, kmer_score, p, exact_seeds=True, max_kmers=512, max_occ=0):
    """The whole restated prefilter of one query: seed hits -> evidence -> gate -> ranking."""
    arena = O.Arena([rows], targets)
    idx = O.SeedIndex(arena, mask)
    ht, hd, hq, sst = O.seed_hits(rows, residues, idx, kmer_score, max_kmers, exact_seeds, max_occ)
    p = dict(p, span=idx.span)
    cands, st = O.prefilter_queries(arena, np.zeros(len(ht), np.uint32), ht, hd, hq, p)
    return cands, st, sst


def test_exact_kmer_is_found():
    m = blosum62()
    q = encode("MKVLLACDEFGHIK")
    c, _, _ = prefilter(m.sequence_rows(q), q, [encode("GGGGGMKVLLACDEFGHIKGGGG"), encode("PPPPPPPPPPPPPP")],
                        "111111", 22, default_params())
    assert len(c) > 0 and c[0]["target"] == 0


def test_exact_seed_below_threshold_is_kept():
    m = blosum62()
    q = encode("AAAAAA")
    t = [encode("WWWWAAAAAAWWWW")]
    p = default_params(min_diag_score=1)
    c, _, _ = prefilter(m.sequence_rows(q), q, t, "111111", 25, p, exact_seeds=False)
    assert len(c) == 0
    c, _, sst = prefilter(m.sequence_rows(q), q, t, "111111", 25, p, exact_seeds=True)
    assert len(c) == 1 and sst["exact_seeds_added"] == 1


def test_similar_kmer_reaches_diverged_target():
    m = blosum62()
    q = encode("MKVLLACDEFGHIK")
    c, _, _ = prefilter(m.sequence_rows(q), q, [encode("GGGGMKILLSCDEFGHLKGGGG")], "111111", 15, default_params())
    assert len(c) > 0


def test_profile_prefilter_finds_target():
    m = blosum62()
    prof = Profile.from_msa_str(">q\nMKVLLACDEFGHIK\n>h\nMKILLSCDEFGHLK\n", m)
    # profile_default: kmer_score 40, min_diag_score 30, no exact seeds (no residues); k = 6
    c, _, _ = prefilter(prof.rows(), None, [encode("GGGGMKVLLACDEFGHIKGGGG")], "111111", 40,
                        default_params(min_diag_score=30), exact_seeds=False)
    assert len(c) > 0


def test_diagonal_mode_and_chain_rescue_with_real_seeds():
    m = blosum62()
    q = encode("MKVLLACDEFGHIK")
    c, _, _ = prefilter(m.sequence_rows(q), q, [encode("MKVLLACDEFGHIKMKVLLAC")], "111111", 22, default_params())
    assert len(c) > 0 and c[0]["diag_score"] > 0 and c[0]["best_diag"] == 0
    q = encode("MKVLLACDEFGHIKLMNPQRSTVWYHHHHWWCCMM")
    t = [encode("QRSTQRSTQRSTQRSTQRSTQRSTQRST" + "MKVLLACDEFGHIKLMNP" + "GGGGQRSTVWYHHHHWWCCMM")]
    one, _, _ = prefilter(m.sequence_rows(q), q, t, "1111", 18, default_params(max_diagonals=1))
    four, st, _ = prefilter(m.sequence_rows(q), q, t, "1111", 18, default_params())
    assert len(four) == 1
    assert four[0]["diag_score"] > (int(one[0]["diag_score"]) if len(one) else 0)


def test_spaced_seed_finds_what_contiguous_misses():
    m = blosum62()
    q = encode("MKVLLACDEFGHIK")
    t = [encode("LLACDPF")]
    p = default_params(min_diag_score=1)
    c, _, _ = prefilter(m.sequence_rows(q), q, t, "111111", 30, p, exact_seeds=False)
    assert not any(int(x["diag_score"]) > 0 for x in c)
    c, _, _ = prefilter(m.sequence_rows(q), q, t, "1111101", 30, p, exact_seeds=False)
    assert any(int(x["diag_score"]) > 0 for x in c)


def test_seed_hits_match_brute_force_definition():
    # every window, every k-mer >= threshold (no window reaches the cap here), every posting
    m = blosum62()
    rng = np.random.default_rng(5)
    for mask, thr in (("111001101", 22), ("11111", 16), ("1101", 12)):
        offs = [i for i, ch in enumerate(mask) if ch == "1"]
        span = len(mask)
        q = rng.integers(0, 21, 40).astype(np.uint8)
        targets = [rng.integers(0, 21, int(rng.integers(5, 80))).astype(np.uint8) for _ in range(12)]
        rows = m.sequence_rows(q)
        idx = O.SeedIndex(O.Arena([rows], targets), mask)
        ht, hd, hq, st = O.seed_hits(rows, q, idx, thr, 100000, True, 0)
        want = set()
        for s in range(len(q) - span + 1):
            if any(q[s + o] >= 20 for o in offs):
                continue
            for ti, t in enumerate(targets):
                for u in range(len(t) - span + 1):
                    if any(t[u + o] >= 20 for o in offs):
                        continue
                    score = sum(int(rows[s + o][t[u + o]]) for o in offs)
                    exact = all(q[s + o] == t[u + o] for o in offs)
                    if score >= thr or exact:
                        want.add((ti, u - s, s))
        got = set(zip(ht.tolist(), hd.tolist(), hq.tolist()))
        assert len(got) == len(ht) and got == want, mask
