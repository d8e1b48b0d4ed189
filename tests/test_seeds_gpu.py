"""GPU parity of the seed stage (st_seed_index_build, st_seed_hits) and of the
whole device prefilter (st_prefilter_queries) against the oracle.

Seed hits must be the oracle's as a multiset (the device emits them unordered)
with equal seed counters: spaced and contiguous patterns, caps that cut inside
runs of tied scores (narrow score rows), exact seeds, windows with X,
profile (PSSM) queries, max_seed_occ.  The whole prefilter must give the
oracle's candidate lists field for field and in order, on the reference's own
prefilter tests and on a batch of homolog queries.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, PrefilterParams, blosum62, encode
from synth import workloads as W
from sabertooth_b200._lib import StError
from synth.profile import Profile
from tests.seedhits import default_params

pytestmark = pytest.mark.gpu

SEED_STATS = ("windows", "windows_skipped", "kmers_generated", "windows_at_cap", "exact_seeds_added", "seeds",
              "postings_visited", "seeds_over_occ_cap", "postings_skipped_occ")


def _oracle_hits(rows_list, residues, targets, mask, p):
    idx = O.SeedIndex(O.Arena(rows_list, targets), mask)
    hits, tot = [], dict.fromkeys(SEED_STATS, 0)
    for q, rows in enumerate(rows_list):
        ht, hd, hq, st = O.seed_hits(rows, None if residues is None else residues[q], idx, p.kmer_score,
                                     p.max_kmers_per_pos, p.exact_seeds, p.max_seed_occ)
        hits += [(q, int(t), int(d), int(x)) for t, d, x in zip(ht, hd, hq)]
        for k in SEED_STATS:
            tot[k] += st[k]
    return sorted(hits), tot, idx


def _check_hits(ctx, rows_list, residues, targets, mask, p):
    ctx.upload_db_list(targets)
    ctx.seed_index_build(mask)
    ids = ctx.create_profiles(rows_list)
    try:
        got, gst = ctx.seed_hits(ids, residues, p)
        inv = {int(i): k for k, i in enumerate(ids)}
        g = sorted((inv[int(h["query"])], int(h["target"]), int(h["diag"]), int(h["qpos"])) for h in got)
        want, wst, _ = _oracle_hits(rows_list, residues, targets, mask, p)
        assert g == want
        assert gst == wst
        return gst
    finally:
        ctx.free_profiles(ids)


@pytest.mark.parametrize("mask", ["111001101", "111111", "11111", "1101", "1111101"])
def test_seed_hits_blosum_queries(ctx, mask):
    m = blosum62()
    rng = np.random.default_rng(len(mask) * 7 + mask.count("1"))
    qs = [rng.integers(0, 21, int(rng.integers(5, 120))).astype(np.uint8) for _ in range(12)]
    targets = [rng.integers(0, 21, int(rng.integers(3, 300))).astype(np.uint8) for _ in range(400)]
    for thr, cap in ((22, 512), (14, 512), (11, 40), (11, 3)):
        st = _check_hits(ctx, [m.sequence_rows(q) for q in qs], qs, targets, mask,
                         PrefilterParams(kmer_score=thr, max_kmers_per_pos=cap))
        assert st["windows_skipped"] > 0  # X residues in the queries
    assert st["windows_at_cap"] > 0


def test_caps_inside_tied_scores(ctx):
    # narrow score rows: many k-mers tie at the cap boundary, so the kept ties
    # must follow the rank-vector order
    rng = np.random.default_rng(3)
    rows = [rng.integers(-2, 3, size=(int(rng.integers(8, 40)), 21)).astype(np.int32) for _ in range(10)]
    targets = [rng.integers(0, 20, int(rng.integers(10, 200))).astype(np.uint8) for _ in range(300)]
    for cap in (1, 7, 100):
        st = _check_hits(ctx, rows, None, targets, "1101", PrefilterParams(kmer_score=1, max_kmers_per_pos=cap,
                                                                           exact_seeds=False))
        assert st["windows_at_cap"] > 0


def test_profile_queries_and_occurrence_cap(ctx):
    m = blosum62()
    w = W.config3(seed=2, n_queries=6, db_residues=60_000, per_query=5)
    targets = [w.db_residues[int(a):int(b)] for a, b in zip(w.db_offsets[:-1], w.db_offsets[1:])]
    p = PrefilterParams.profile_default()
    _check_hits(ctx, list(w.rows), None, targets, "11111", p)
    st = _check_hits(ctx, list(w.rows), None, targets, "11111",
                     PrefilterParams(kmer_score=30, exact_seeds=False, max_seed_occ=2))
    assert st["seeds_over_occ_cap"] > 0


def test_errors(ctx):
    m = blosum62()
    ctx.upload_db_list([encode("MKVLLACDEFGHIK")])
    ids = ctx.create_profiles([m.sequence_rows(encode("MKVLLACDEFGH"))])
    try:
        with pytest.raises(StError):
            ctx.seed_hits(ids)  # no index for this database
        for bad in ("", "0110", "11x1", "1", "11111111"):
            with pytest.raises(StError):
                ctx.seed_index_build(bad)
        ctx.seed_index_build("111111")
        with pytest.raises(StError):
            ctx.seed_hits(ids, params=PrefilterParams(max_kmers_per_pos=0))
        hits, st = ctx.seed_hits(ids, [encode("MKVLLACDEFGH")])
        assert len(hits) > 0 and st["windows"] == 12 - 6 + 1
        with pytest.raises(StError):  # the same profile twice in one prefilter call
            ctx.prefilter_queries(np.concatenate([ids, ids]), [encode("MKVLLACDEFGH")] * 2)
    finally:
        ctx.free_profiles(ids)


def _oracle_prefilter(rows_list, residues, targets, mask, p, gaps):
    hits, _, idx = _oracle_hits(rows_list, residues, targets, mask, p)
    h = np.array(hits, dtype=np.int64).reshape(-1, 4)
    gp = default_params(min_hits=p.min_hits, diag_hits=p.diag_hits, max_diagonals=p.max_diagonals,
                        diag_window=p.diag_window, span=idx.span, min_diag_score=p.min_diag_score,
                        gap_open=gaps.open, gap_ext=gaps.extend, max_candidates=p.max_candidates,
                        regions=int(p.regions))
    return O.prefilter_queries(O.Arena(rows_list, targets), h[:, 0], h[:, 1], h[:, 2], h[:, 3], gp)


def _check_prefilter(ctx, rows_list, residues, targets, mask, p, gaps):
    ctx.upload_db_list(targets)
    ctx.seed_index_build(mask)
    ids = ctx.create_profiles(rows_list)
    try:
        got, st, sst = ctx.prefilter_queries(ids, residues, p, gaps)
        want, wst = _oracle_prefilter(rows_list, residues, targets, mask, p, gaps)
        for q in range(len(rows_list)):
            g = got[got["query"] == ids[q]].copy()
            g["query"] = q
            assert np.array_equal(g, want[want["query"] == q]), q
        for k in wst:
            assert st[k] == wst[k], k
        return got
    finally:
        ctx.free_profiles(ids)


def test_reference_prefilter_tests_on_the_device(ctx):
    m = blosum62()
    seq = GapCosts.sequence_default()
    q = encode("MKVLLACDEFGHIK")
    c = _check_prefilter(ctx, [m.sequence_rows(q)], [q], [encode("GGGGGMKVLLACDEFGHIKGGGG"),
                                                           encode("PPPPPPPPPPPPPP")], "111111",
                         PrefilterParams(span=6), seq)
    assert len(c) > 0 and c[0]["target"] == 0  # exact_kmer_is_found
    a = encode("AAAAAA")
    p = PrefilterParams(kmer_score=25, min_diag_score=1, exact_seeds=False)
    assert len(_check_prefilter(ctx, [m.sequence_rows(a)], [a], [encode("WWWWAAAAAAWWWW")], "111111", p, seq)) == 0
    p = PrefilterParams(kmer_score=25, min_diag_score=1, exact_seeds=True)
    assert len(_check_prefilter(ctx, [m.sequence_rows(a)], [a], [encode("WWWWAAAAAAWWWW")], "111111", p, seq)) == 1
    c = _check_prefilter(ctx, [m.sequence_rows(q)], [q], [encode("GGGGMKILLSCDEFGHLKGGGG")], "111111",
                         PrefilterParams(kmer_score=15), seq)
    assert len(c) > 0  # similar_kmer_reaches_diverged_target
    prof = Profile.from_msa_str(">q\nMKVLLACDEFGHIK\n>h\nMKILLSCDEFGHLK\n", m)
    c = _check_prefilter(ctx, [prof.rows()], None, [encode("GGGGMKVLLACDEFGHIKGGGG")], "111111",
                         PrefilterParams.profile_default(), GapCosts.profile_default())
    assert len(c) > 0  # profile_prefilter_finds_target
    q2 = encode("MKVLLACDEFGHIKLMNPQRSTVWYHHHHWWCCMM")
    t2 = [encode("QRSTQRSTQRSTQRSTQRSTQRSTQRST" + "MKVLLACDEFGHIKLMNP" + "GGGGQRSTVWYHHHHWWCCMM")]
    one = _check_prefilter(ctx, [m.sequence_rows(q2)], [q2], t2, "1111",
                           PrefilterParams(kmer_score=18, max_diagonals=1), seq)
    four = _check_prefilter(ctx, [m.sequence_rows(q2)], [q2], t2, "1111", PrefilterParams(kmer_score=18), seq)
    assert len(four) == 1 and four[0]["diag_score"] > (int(one[0]["diag_score"]) if len(one) else 0)
    t3 = [encode("LLACDPF")]
    p = PrefilterParams(kmer_score=30, min_diag_score=1, exact_seeds=False)
    c = _check_prefilter(ctx, [m.sequence_rows(q)], [q], t3, "111111", p, seq)
    assert not any(int(x["diag_score"]) > 0 for x in c)
    c = _check_prefilter(ctx, [m.sequence_rows(q)], [q], t3, "1111101", p, seq)
    assert any(int(x["diag_score"]) > 0 for x in c)  # spaced_seed_finds_what_contiguous_misses


def test_batch_of_homolog_queries(ctx):
    model = W.Model()
    rng = W.Rng(9)
    m = blosum62()
    qs = [model.background(rng.child(i), int(n)) for i, n in enumerate(W.lognormal_lengths(rng, 40, 200, 0.5, 30, 600))]
    targets = []
    for k in range(3000):
        if k % 10 == 0:  # a mutated copy of a query, with indels
            targets.append(model.mutate(rng.child(1000 + k), qs[k % 40], 0.55, indel_rate=0.03))
        else:
            targets.append(model.background(rng.child(1000 + k), 60 + k % 400))
    for p in (PrefilterParams(regions=True), PrefilterParams(kmer_score=20, max_diagonals=16, max_candidates=25)):
        got = _check_prefilter(ctx, [m.sequence_rows(q) for q in qs], qs, targets, "111001101", p,
                               GapCosts.sequence_default())
        assert len(got) > 0


def test_many_queries_in_several_chunks(ctx):
    # more than 65,536 windows: the device prefilter takes the queries in length order in several chunks and
    # must still return every query's candidates ranked, in query id order, and cut to a given capacity
    model = W.Model()
    rng = W.Rng(12)
    m = blosum62()
    lens = W.lognormal_lengths(rng, 320, 250, 0.6, 30, 1200)
    qs = [model.background(rng.child(i), int(n)) for i, n in enumerate(lens)]
    targets = []
    for k in range(1500):
        if k % 5 == 0:
            targets.append(model.mutate(rng.child(5000 + k), qs[k % 320], 0.6, indel_rate=0.02))
        else:
            targets.append(model.background(rng.child(5000 + k), 80 + k % 300))
    assert sum(max(int(n) - 8, 0) for n in lens) > 65536
    got = _check_prefilter(ctx, [m.sequence_rows(q) for q in qs], qs, targets, "111001101",
                           PrefilterParams(kmer_score=20), GapCosts.sequence_default())
    assert len(got) > 0
    # a capacity below the count writes the first candidates of the same order
    ctx.upload_db_list(targets)
    ctx.seed_index_build("111001101")
    ids = ctx.create_profiles([m.sequence_rows(q) for q in qs])
    try:
        full, _, _ = ctx.prefilter_queries(ids, qs, PrefilterParams(kmer_score=20))
        from sabertooth_b200._lib import CANDIDATE_DTYPE, check, lib, ptr
        import ctypes as C
        p = PrefilterParams(kmer_score=20)
        sp, gp = p.seed_c(), p.to_c(GapCosts.sequence_default())
        res = np.ascontiguousarray(np.concatenate(qs))
        offs = np.zeros(len(qs) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(q) for q in qs])
        k = len(full) // 3
        out = np.zeros(k, dtype=CANDIDATE_DTYPE)
        n = C.c_uint64()
        check(lib.st_prefilter_queries(ctx.handle, ptr(ids), len(ids), ptr(res), ptr(offs), C.byref(sp), C.byref(gp),
                                       ptr(out), k, C.byref(n), None, None))
        assert n.value == len(full) and np.array_equal(out, full[:k])
    finally:
        ctx.free_profiles(ids)
