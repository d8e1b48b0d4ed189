"""The planned (CUDA-graph) batched form: replay determinism, accounting, autotuning, per-launch profile."""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts
from sabertooth_b200 import workloads as W
from sabertooth_b200._lib import PAIR_DTYPE

pytestmark = pytest.mark.gpu


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
    saved = ctx.tuning_table()
    try:
        tuned = ctx.autotune(pairs, GapCosts(44, 4), max_pairs_per_bin=2000)
        assert tuned >= 1
        table = ctx.tuning_table()
        assert (table >= 0).sum() >= tuned
        got = ctx.sw_score_pairs(pairs, GapCosts(44, 4))
        want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4)
        assert np.array_equal(got, want)
    finally:
        ctx.set_tuning_table(saved)
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
