"""The planned (CUDA-graph) batched form: replay determinism, accounting, autotuning, per-launch profile."""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts
from synth import workloads as W
from sabertooth_b200._lib import PAIR_DTYPE

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("planner")]


def _pairs(ids, w):
    p = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
    p["profile"] = ids[w.pair_q]
    p["target"] = w.pair_t
    p["band_center"] = 0 if w.band_center is None else w.band_center
    p["band_radius"] = -1 if w.band_radius is None else w.band_radius
    return p


def test_plan_replays_identically_and_counts_cells(ctx):
    import torch
    w = W.config4(seed=3, n_pairs=80, kind="blosum62", near_identical=0.2)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = _pairs(ids, w)
    d_s = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    d_k = torch.empty(w.n_pairs, dtype=torch.int32, device="cuda")
    plan = ctx.plan(pairs, GapCosts(11, 1), d_s.data_ptr(), d_k.data_ptr())
    plan.run()
    ctx.synchronize()
    first = d_s.cpu().numpy().copy()
    plan.run()
    plan.run()
    ctx.synchronize()
    assert np.array_equal(first, d_s.cpu().numpy())
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 11, 1, w.band_center.astype(np.int64),
                      w.band_radius.astype(np.int64))
    assert np.array_equal(first, want)
    st = plan.stats()
    assert st["cells"] == w.cells()
    prof = plan.profile()
    assert sum(c for _, c, _ in prof) == st["cells"]
    assert np.array_equal(d_s.cpu().numpy(), want)  # the per-launch profile writes the same scores
    plan.close()
    for i in ids:
        ctx.free_profile(i)


def test_autotune_keeps_scores_exact(ctx):
    w = W.config3(seed=9, n_queries=40, db_residues=80_000, per_query=60)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = _pairs(ids, w)
    saved, saved_rates = ctx.tuning_table(), ctx.tuning_rates()
    try:
        tuned = ctx.autotune(pairs, GapCosts(44, 4), max_pairs=2000)
        assert tuned >= 1
        assert np.array_equal(ctx.tuning_table(), saved)  # the forcing table comes back
        rates = ctx.tuning_rates()
        assert (rates > 0).sum() == tuned
        got = ctx.sw_score_pairs(pairs, GapCosts(44, 4))
        want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4)
        assert np.array_equal(got, want)
        # a model with one class left gives the same scores
        only = np.zeros_like(rates)
        only[1] = 1.0
        ctx.set_tuning_rates(only)
        assert np.array_equal(ctx.sw_score_pairs(pairs, GapCosts(44, 4)), want)
    finally:
        ctx.set_tuning_table(saved)
        ctx.set_tuning_rates(saved_rates)
        for i in ids:
            ctx.free_profile(i)


def test_bad_pairs_are_rejected_with_a_message(ctx):
    from sabertooth_b200._lib import StError
    w = W.config3(seed=1, n_queries=4, db_residues=10_000, per_query=5)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = _pairs(ids, w)
    bad = pairs.copy()
    bad["target"][3] = 10_000_000
    with pytest.raises(StError, match="outside the database"):
        ctx.sw_score_pairs(bad, GapCosts(44, 4))
    bad = pairs.copy()
    bad["profile"][0] = 999_999
    with pytest.raises(StError, match="unknown profile"):
        ctx.sw_score_pairs(bad, GapCosts(44, 4))
    # the context stays usable
    got = ctx.sw_score_pairs(pairs, GapCosts(44, 4))
    assert np.array_equal(got, O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4))
    for i in ids:
        ctx.free_profile(i)


def test_memory_budget_is_enforced():
    from sabertooth_b200 import Context
    from sabertooth_b200._lib import StError
    c = Context(0, hbm_budget_bytes=1 << 20)
    try:
        with pytest.raises(StError, match="budget"):
            c.create_profiles([np.zeros((20000, 21), dtype=np.int32)])
    finally:
        c.close()


def _big_batch(seed, n_pairs, n_q=700, n_t=4000):
    """Many short pairs: enough for the pipelined (chunked, two-stream) form, cheap for the oracle."""
    from sabertooth_b200 import blosum62
    rng = np.random.default_rng(seed)
    m = blosum62()
    queries = [rng.integers(0, 21, int(L)).astype(np.uint8) for L in rng.integers(0, 70, n_q)]
    targets = [rng.integers(0, 22, int(L)).astype(np.uint8) for L in rng.integers(0, 90, n_t)]
    for k in range(0, n_t, 7):  # near-identical targets so that some scores are high
        q = queries[k % n_q]
        targets[k] = np.concatenate([targets[k][:5], q, targets[k][5:]]).astype(np.uint8)
    rows = [m.sequence_rows(q) for q in queries]
    pq = rng.integers(0, n_q, n_pairs).astype(np.uint32)
    pt = rng.integers(0, n_t, n_pairs).astype(np.uint32)
    return rows, targets, pq, pt


def test_pipelined_batch_matches_oracle_and_single_plan(ctx, monkeypatch):
    import torch
    monkeypatch.setenv("ST_PIPELINE_PAIRS", "65536")  # seven chunks
    rows, targets, pq, pt = _big_batch(11, 420_000)
    n = len(pq)
    center = np.zeros(n, dtype=np.int32)
    radius = np.full(n, -1, dtype=np.int32)
    banded = np.arange(0, n, 997)  # banded pairs in every chunk take the 32-bit kernel
    radius[banded] = 3
    center[banded] = (np.arange(len(banded)) % 9) - 4
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    try:
        pairs = np.zeros(n, dtype=PAIR_DTYPE)
        pairs["profile"] = ids[pq]
        pairs["target"] = pt
        pairs["band_center"] = center
        pairs["band_radius"] = radius
        for gaps in [GapCosts(11, 1), GapCosts(300, 1)]:  # the second routes every pair to the 32-bit kernel
            got, kinds = ctx.sw_score_pairs(pairs, gaps, with_kernels=True)
            want = O.sw_pairs(O.Arena(rows, targets), pq, pt, gaps.open, gaps.extend, center.astype(np.int64),
                              radius.astype(np.int64))
            assert np.array_equal(got, want), gaps
            # the single captured plan (no chunking) gives the same scores and kernel tags
            d_s = torch.empty(n, dtype=torch.int32, device="cuda")
            d_k = torch.empty(n, dtype=torch.int32, device="cuda")
            plan = ctx.plan(pairs, gaps, d_s.data_ptr(), d_k.data_ptr())
            plan.run()
            ctx.synchronize()
            assert np.array_equal(d_s.cpu().numpy(), got)
            assert np.array_equal(d_k.cpu().numpy().view(np.uint32), kinds)
            plan.close()
        # twice in a row: pooled arenas and the staging ring give the same result
        assert np.array_equal(ctx.sw_score_pairs(pairs, GapCosts(11, 1)), ctx.sw_score_pairs(pairs, GapCosts(11, 1)))
    finally:
        for i in ids:
            ctx.free_profile(i)


def test_pipelined_batch_error_in_a_late_chunk_leaves_context_usable(ctx, monkeypatch):
    from sabertooth_b200._lib import StError
    monkeypatch.setenv("ST_PIPELINE_PAIRS", "65536")
    rows, targets, pq, pt = _big_batch(12, 400_000)
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    try:
        pairs = np.zeros(len(pq), dtype=PAIR_DTYPE)
        pairs["profile"] = ids[pq]
        pairs["target"] = pt
        pairs["band_radius"] = -1
        bad = pairs.copy()
        bad["target"][len(pq) - 5] = 10_000_000  # in the last chunk, after earlier chunks were launched
        with pytest.raises(StError, match="outside the database"):
            ctx.sw_score_pairs(bad, GapCosts(11, 1))
        got = ctx.sw_score_pairs(pairs, GapCosts(11, 1))
        assert np.array_equal(got, O.sw_pairs(O.Arena(rows, targets), pq, pt, 11, 1))
    finally:
        for i in ids:
            ctx.free_profile(i)


def test_profile_ids_are_reused_and_batch_free_checks_ids(ctx):
    from sabertooth_b200._lib import StError
    w = W.config3(seed=4, n_queries=6, db_residues=20_000, per_query=10)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    first = ctx.sw_score_pairs(_pairs(ids, w), GapCosts(44, 4))
    ctx.free_profiles(ids)
    with pytest.raises(StError, match="unknown profile"):
        ctx.free_profiles(ids[:1])
    again = ctx.create_profiles(w.rows[::-1])  # the same ids come back, now for other rows
    assert sorted(again.tolist()) == sorted(ids.tolist())
    rev = again[::-1]
    assert np.array_equal(ctx.sw_score_pairs(_pairs(rev, w), GapCosts(44, 4)), first)
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4)
    assert np.array_equal(first, want)
    ctx.free_profiles(again)


def test_async_batches_overlap_and_early_profile_free(ctx):
    """Two batches in flight; the first batch's profiles are freed (and their ids reused by
    the second batch's profiles) before it is waited for: queued work keeps its profiles."""
    import torch
    w1 = W.config3(seed=21, n_queries=30, db_residues=60_000, per_query=80)
    w2 = W.config3(seed=22, n_queries=25, db_residues=60_000, per_query=90)
    # one database for both: w2's targets appended after w1's
    t1, t2 = w1.targets(), w2.targets()
    ctx.upload_db_list(t1 + t2)
    ids1 = ctx.create_profiles(w1.rows)
    p1 = _pairs(ids1, w1)
    out1 = torch.empty(w1.n_pairs, dtype=torch.int32, pin_memory=True).numpy()
    b1 = ctx.sw_score_pairs_async(p1, GapCosts(44, 4), scores=out1)
    ctx.free_profiles(ids1)  # before b1 is waited for
    ids2 = ctx.create_profiles(w2.rows)
    assert set(ids2.tolist()) & set(ids1.tolist())  # ids were handed out again
    p2 = _pairs(ids2, w2)
    p2["target"] += len(t1)
    b2 = ctx.sw_score_pairs_async(p2, GapCosts(11, 1))  # pageable output
    got2 = b2.wait()
    got1 = b1.wait()
    want1 = O.sw_pairs(O.Arena(w1.rows, t1), w1.pair_q, w1.pair_t, 44, 4)
    want2 = O.sw_pairs(O.Arena(w2.rows, t2), w2.pair_q, w2.pair_t, 11, 1)
    assert np.array_equal(got1, want1)
    assert np.array_equal(got2, want2)
    with pytest.raises(RuntimeError):
        b1.wait()
    ctx.free_profiles(ids2)


def test_async_batch_of_nothing_and_sync_equals_async(ctx):
    w = W.config3(seed=23, n_queries=12, db_residues=30_000, per_query=40)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    pairs = _pairs(ids, w)
    empty = ctx.sw_score_pairs_async(pairs[:0], GapCosts(44, 4))
    assert len(empty.wait()) == 0
    s, k = ctx.sw_score_pairs_async(pairs, GapCosts(44, 4), with_kernels=True).wait()
    s2, k2 = ctx.sw_score_pairs(pairs, GapCosts(44, 4), with_kernels=True)
    assert np.array_equal(s, s2) and np.array_equal(k, k2)
    ctx.free_profiles(ids)
