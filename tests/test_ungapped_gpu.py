"""GPU parity of ungapped diagonal scoring against the CPU oracle.

Cases follow the reference's tests (src/ungapped.rs:531-616): every diagonal
of random pairs with sub-windows (seed 3), random and homologous lanes with
windows and empty ranges (seed 17), and wide PSSM-like rows, plus the batched
hit form with its per-(query, target) runs.  Bar: bit-exact int32.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import DiagProfile, Lane, blosum62, score_batch
from synth import workloads as W
from sabertooth_b200.api import diag_range
from tests.refrng import SplitMix64

pytestmark = pytest.mark.gpu


def test_every_diagonal_and_subwindows(ctx):
    rng = SplitMix64(3)
    m = blosum62()
    cases = []
    for _ in range(60):
        q = [rng.below(21) for _ in range(1 + rng.below(80))]
        t = [rng.below(21) for _ in range(1 + rng.below(120))]
        cases.append((q, t))
    ctx.upload_db_list([np.array(t, np.uint8) for _, t in cases])
    for k, (q, t) in enumerate(cases):
        rows = m.sequence_rows(q)
        prof = DiagProfile.build(rows, ctx)
        lanes, want = [], []
        for d in range(-len(q) - 2, len(t) + 2):
            lo, hi = diag_range(len(q), len(t), d)
            lanes.append(Lane(k, d, lo, hi))
            want.append(O.kadane_score(rows, t, d, lo, hi))
            if hi > lo + 2:
                lanes.append(Lane(k, d, lo + 1, hi - 1))
                want.append(O.kadane_score(rows, t, d, lo + 1, hi - 1))
        got = score_batch(prof, lanes)
        prof.qp.free()
        assert np.array_equal(got, np.array(want, dtype=np.int32)), k


def test_random_and_homologous_lanes(ctx):
    rng = SplitMix64(17)
    mat = blosum62()
    for case in range(12):
        qlen = 1 + rng.below(400 if case % 3 == 0 else 90)
        q = [rng.below(21) for _ in range(qlen)]
        rows = mat.sequence_rows(q)
        targets = []
        for k in range(70):
            if k % 5 == 0:  # a copy of the query with a few substitutions: long, high-scoring
                t = list(q)
                for _ in range(qlen // 10):
                    t[rng.below(qlen)] = rng.below(20)
            else:
                t = [rng.below(21) for _ in range(1 + rng.below(300))]
            targets.append(t)
        ctx.upload_db_list([np.array(t, np.uint8) for t in targets])
        prof = DiagProfile.build(rows, ctx)
        lanes, want = [], []
        for k, t in enumerate(targets):
            d = 0 if k % 5 == 0 else rng.below(len(t) + qlen + 4) - qlen - 2
            lo, hi = diag_range(qlen, len(t), d)
            if k % 3 == 1 and hi > lo + 4:
                a = lo + rng.below(hi - lo)
                b = a + rng.below(hi - a) + 1
                lo, hi = a, b
            lanes.append(Lane(k, d, lo, hi))
            want.append(O.kadane_score(rows, t, d, lo, hi))
        got = score_batch(prof, lanes)
        prof.qp.free()
        assert np.array_equal(got, np.array(want, dtype=np.int32)), case


def test_wide_score_rows(ctx):
    # rows the reference's u8 kernel rejects (src/ungapped.rs:608-616) are exact here
    rows = np.zeros((50, 21), dtype=np.int32)
    rows[::2, 0] = 200
    rows[1::2, 1] = -100
    t = np.array([0, 1] * 40 + [0] * 30, dtype=np.uint8)
    ctx.upload_db_list([t])
    prof = DiagProfile.build(rows, ctx)
    lanes = [Lane(0, d, *diag_range(50, t.size, d)) for d in range(-49, t.size)]
    want = [O.kadane_score(rows, t, l.diag, l.lo, l.hi) for l in lanes]
    assert np.array_equal(score_batch(prof, lanes), np.array(want, dtype=np.int32))
    prof.qp.free()


def test_window_outside_the_diagonal_is_rejected(ctx):
    from sabertooth_b200._lib import StError
    t = np.zeros(10, dtype=np.uint8)
    ctx.upload_db_list([t])
    prof = DiagProfile.build(np.ones((5, 21), dtype=np.int32), ctx)
    with pytest.raises(StError):
        score_batch(prof, [Lane(0, 8, 0, 5)])  # diag 8 leaves only query positions 0..1
    prof.qp.free()


@pytest.fixture(params=["refill", "split"])
def hit_kernel(request, monkeypatch):
    """Runs a hit test with the default refill kernel and with the split-work kernel (ST_UNGAPPED_SPLIT=1)."""
    monkeypatch.setenv("ST_UNGAPPED_SPLIT", "1" if request.param == "split" else "0")
    return request.param


def test_hits_and_pair_runs_match_oracle(ctx, hit_kernel):
    w = W.config2(seed=2, n_queries=40, n_targets=3000, n_hits=60_000)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    hits = w.hits.copy()
    hits["query"] = ids[hits["query"]]
    per_hit, (pb, pq, pt) = ctx.ungapped_hits(hits)
    ar = O.Arena(w.rows, [w.db_residues[int(a):int(b)] for a, b in zip(w.db_offsets[:-1], w.db_offsets[1:])])
    want = O.ungapped_hits(ar, w.hits["query"], w.hits["target"], w.hits["diag"])
    assert np.array_equal(per_hit, want)
    # runs of equal (query, target) in hit order
    key = w.hits["query"].astype(np.int64) * (1 << 32) + w.hits["target"]
    start = np.ones(len(key), dtype=bool)
    start[1:] = key[1:] != key[:-1]
    idx = np.nonzero(start)[0]
    run_best = np.maximum.reduceat(want, idx)
    assert np.array_equal(pb, run_best)
    assert np.array_equal(pq, ids[w.hits["query"][idx]])
    assert np.array_equal(pt, w.hits["target"][idx])
    for i in ids:
        ctx.free_profile(i)


def test_unsorted_hits_are_still_exact(ctx, hit_kernel):
    w = W.config2(seed=4, n_queries=30, n_targets=2000, n_hits=20_000)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    perm = np.random.default_rng(0).permutation(len(w.hits))
    hits = w.hits[perm].copy()
    want = O.ungapped_hits(O.Arena(w.rows, [w.db_residues[int(a):int(b)] for a, b in
                                             zip(w.db_offsets[:-1], w.db_offsets[1:])]),
                           hits["query"], hits["target"], hits["diag"])
    hits["query"] = ids[hits["query"]]
    got = ctx.ungapped_hits(hits, with_pairs=False)
    assert np.array_equal(got, want)
    for i in ids:
        ctx.free_profile(i)


@pytest.mark.parametrize("wide", [False, True])
def test_hit_edges(ctx, hit_kernel, wide):
    """Every diagonal of short and vector-edge lengths (queries of 1, 15, 16, 17, 33 and 1,024 residues, targets
    of 1, 15, 16, 17, 32 and 48 residues, so windows start and end on and off the 16-byte target vectors and
    targets end on and off the arena's 16-byte boundaries), hits in query runs and shuffled, with int8 rows and
    with rows outside int8 (the int32 path)."""
    rng = np.random.default_rng(31)
    qlens, tlens = [1, 15, 16, 17, 33, 1024], [1, 15, 16, 17, 32, 48]
    span = 300 if wide else 11
    rows = [rng.integers(-span, span + 1, size=(m, 21)).astype(np.int32) for m in qlens]
    seqs = [rng.integers(0, 21, size=n).astype(np.uint8) for n in tlens]
    offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum([len(x) for x in seqs])
    ctx.upload_db(np.concatenate(seqs), offs)
    ids = ctx.create_profiles(rows)
    q, t, d = [], [], []
    for qi, m in enumerate(qlens):
        for ti, n in enumerate(tlens):
            for dd in range(-(m - 1) - 2, n + 2):
                if abs(dd) > 80 and rng.random() < 0.9:
                    continue
                q.append(qi)
                t.append(ti)
                d.append(dd)
    from sabertooth_b200.dtypes import HIT_DTYPE
    hits = np.zeros(len(q), dtype=HIT_DTYPE)
    hits["query"], hits["target"], hits["diag"] = q, t, d
    want = O.ungapped_hits(O.Arena(rows, seqs), hits["query"], hits["target"], hits["diag"])
    for order in (np.arange(len(hits)), np.random.default_rng(1).permutation(len(hits))):
        h = hits[order].copy()
        h["query"] = ids[h["query"]]
        got = ctx.ungapped_hits(h, with_pairs=False)
        assert np.array_equal(got, want[order])
    for i in ids:
        ctx.free_profile(i)


def test_lanes_carry_arena_slices_as_the_reference_builds_them(ctx):
    """Lanes whose target is a slice of the uploaded arena (src/ungapped.rs:265-270, built from
    index.seq(tid) in src/prefilter.rs:1563-1568), through st_ungapped_score_slices: whole sequences
    and sub-slices, every diagonal, sub-windows, empty windows."""
    rng = SplitMix64(29)
    m = blosum62()
    seqs = [np.array([rng.below(21) for _ in range(rng.below(150))], np.uint8) for _ in range(40)]
    seqs[0] = np.array([rng.below(20) for _ in range(60)], np.uint8)
    seqs[1] = np.array([rng.below(20) for _ in range(60)], np.uint8)
    seqs[3] = np.zeros(0, np.uint8)  # an empty sequence inside the arena
    ctx.upload_db_list(seqs)
    for case in range(10):
        q = [rng.below(21) for _ in range(1 + rng.below(90))]
        rows = m.sequence_rows(q)
        prof = DiagProfile.build(rows, ctx)
        lanes, want = [], []
        for tid in range(len(seqs)):
            full = ctx.db_seq(tid)
            assert np.array_equal(full, seqs[tid])
            a = rng.below(len(full) + 1)
            b = a + rng.below(len(full) - a + 1)
            for t in (full, full[a:b]):
                for d in range(-len(q) - 1, len(t) + 1, 1 + case):
                    lo, hi = diag_range(len(q), len(t), d)
                    lanes.append(Lane(t, d, lo, hi))
                    want.append(O.kadane_score(rows, t, d, lo, hi))
                    if hi > lo + 2:
                        lanes.append(Lane(t, d, lo + 1, hi - 1))
                        want.append(O.kadane_score(rows, t, d, lo + 1, hi - 1))
        got = score_batch(prof, lanes)
        assert np.array_equal(got, np.array(want, dtype=np.int32)), case
        # a buffer that is not the uploaded arena, and a window outside the slice's diagonal range, are errors
        from sabertooth_b200._lib import StError
        with pytest.raises(StError, match="not inside the database arena"):
            score_batch(prof, [Lane(seqs[0].copy(), 0, 0, min(len(q), len(seqs[0])))])
        t = ctx.db_seq(1)
        with pytest.raises(StError, match="outside the diagonal's range"):
            score_batch(prof, [Lane(t[:5], 0, 0, min(len(q), 5) + 1)])
        prof.qp.free()
