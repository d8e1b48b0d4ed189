"""Banded pairs in packed 16-bit cells (sw16_band_kernel), against the oracle.

The band rule of local_align_in_band (src/align.rs:439-447) restated in the
oracle (or_band_score).  The packed kernel takes banded pairs with int8 rows
(two per warp, one per 16-bit half) when the gap costs fit 16 bits; banded
pairs with wider rows, and every unbanded pair of the 32-bit list, stay with
the 32-bit kernel.  Cases: an odd number of banded pairs (a warp with one half
empty), queries of one to several 256-row passes against band windows from
one column to thousands (windows narrower than a warp with several passes),
centres before, inside and past the target, radius 0 to wide, pairs with no
band cell at all, and near-identical long pairs whose 16-bit cells pass the
headroom and are rescored in 32 bits by the same warp.  Host- and
device-planned batches, and the captured plan.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, Kernel, blosum62
from sabertooth_b200._lib import PAIR_DTYPE
from synth import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("planner")]


def _cases(seed):
    model = W.Model()
    r = W.Rng(seed)
    rs = np.random.default_rng(seed)
    rows, targets, centers, radii = [], [], [], []
    for i in range(301):  # odd
        m = int(rs.choice([1, 7, 60, 255, 256, 257, 300, 700, 1300]))
        n = int(rs.choice([1, 5, 31, 33, 200, 1000, 3000]))
        q = model.background(r, m)
        t = model.background(r, n)
        c = int(rs.integers(-m - 20, n + 20))
        if i % 5 == 0 and n > 20:  # a homologous stretch on the band's diagonal
            pos = max(0, min(n - 1, c))
            k = min(m, n - pos)
            t[pos:pos + k] = model.mutate(r, q[:k], 0.8)
            c = pos
        rows.append(model.mat.sequence_rows(q))
        targets.append(t)
        centers.append(c)
        radii.append(int(rs.choice([0, 1, 3, 16, 64, 200, 5000])))
    return rows, targets, np.array(centers, np.int32), np.array(radii, np.int32)


def _score(ctx, rows, targets, centers, radii, gaps, with_kernels=True):
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    pairs = np.zeros(len(rows), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(rows))
    pairs["band_center"] = centers
    pairs["band_radius"] = radii
    try:
        return ctx.sw_score_pairs(pairs, gaps, with_kernels=with_kernels)
    finally:
        ctx.free_profiles(ids)


@pytest.mark.parametrize("gaps", [(11, 1), (44, 4), (3, 1)])
def test_banded_pairs_match_oracle(ctx, gaps):
    rows, targets, centers, radii = _cases(7 + gaps[0])
    got, kinds = _score(ctx, rows, targets, centers, radii, GapCosts(*gaps))
    want = O.sw_pairs(O.Arena(rows, targets), np.arange(len(rows)), np.arange(len(rows)), *gaps,
                      centers.astype(np.int64), radii.astype(np.int64))
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, [(len(rows[i]), len(targets[i]), int(centers[i]), int(radii[i]), int(got[i]), int(want[i]))
                           for i in bad[:8]]
    assert (kinds == Kernel.GPU16).sum() > len(rows) // 2  # the packed kernel took them


def test_wide_rows_and_mixed_lists(ctx):
    """Banded pairs with rows outside int8 (the 32-bit kernel) beside int8 ones and unbanded pairs."""
    rows, targets, centers, radii = _cases(21)
    rows = [r * 13 if i % 4 == 0 else r for i, r in enumerate(rows)]  # every fourth: scores up to 143, outside int8
    radii = np.where(np.arange(len(rows)) % 6 == 5, -1, radii).astype(np.int32)  # some unbanded
    got, kinds = _score(ctx, rows, targets, centers, radii, GapCosts(11, 1))
    want = O.sw_pairs(O.Arena(rows, targets), np.arange(len(rows)), np.arange(len(rows)), 11, 1,
                      centers.astype(np.int64), radii.astype(np.int64))
    assert np.array_equal(got, want)
    wide = np.array([np.abs(r).max() > 127 for r in rows])
    assert np.all(kinds[wide & (radii >= 0) & (got > 0)] == Kernel.GPU32)


def test_headroom_overflow_is_rescored_exactly(ctx):
    """Near-identical long banded pairs: scores far above 32767 come from the 32-bit rescore."""
    m = blosum62()
    w = 18  # W, s(W, W) = 11
    rows, targets, centers, radii = [], [], [], []
    for k, n in enumerate((4000, 4100, 3500, 5000, 3700)):
        q = np.full(n - 50, w, dtype=np.uint8)
        t = np.full(n, w, dtype=np.uint8)
        t[::97] = 3  # a few mismatches
        rows.append(m.sequence_rows(q))
        targets.append(t)
        centers.append(k * 7)
        radii.append(64)
    # and a short pair sharing a warp with an overflowing one
    rows.append(m.sequence_rows(np.arange(60, dtype=np.uint8) % 20))
    targets.append((np.arange(80, dtype=np.uint8) * 7) % 20)
    centers.append(3)
    radii.append(10)
    got, kinds = _score(ctx, rows, targets, np.array(centers, np.int32), np.array(radii, np.int32), GapCosts(11, 1))
    want = O.sw_pairs(O.Arena(rows, targets), np.arange(len(rows)), np.arange(len(rows)), 11, 1,
                      np.array(centers, np.int64), np.array(radii, np.int64))
    assert np.array_equal(got, want)
    assert np.all(want[:5] > 32767)
    assert np.all(kinds[:5] == Kernel.GPU32)


def test_captured_plan_repeats_band_scores(ctx):
    import torch
    rows, targets, centers, radii = _cases(33)
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    pairs = np.zeros(len(rows), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(rows))
    pairs["band_center"] = centers
    pairs["band_radius"] = radii
    d_s = torch.empty(len(rows), dtype=torch.int32, device="cuda")
    plan = ctx.plan(pairs, GapCosts(11, 1), d_s.data_ptr())
    try:
        want = O.sw_pairs(O.Arena(rows, targets), np.arange(len(rows)), np.arange(len(rows)), 11, 1,
                          centers.astype(np.int64), radii.astype(np.int64))
        for _ in range(3):
            plan.run()
            ctx.synchronize()
            assert np.array_equal(d_s.cpu().numpy(), want)
        prof = plan.profile()
        assert any(sh == "band16" for sh, _, _ in prof)
        assert np.array_equal(d_s.cpu().numpy(), want)
    finally:
        plan.close()
        ctx.free_profiles(ids)
