"""Multi-pass queries against targets shorter than one warp, on every route
into the exact 32-bit kernel, against the oracle.

The 32-bit kernel scores a query of more than 256 rows in several passes; the
bottom row of a pass goes to scratch and comes back into lane 0 for the next
pass.  Lane 0 reaches column c of the next pass 32 steps before the last lane
has finished column c of this one unless a pass streams at least 32 columns,
so a pass over a short target is padded with idle columns.  Every case here
pairs m in {257, 700, 5000} with n in {1, 2, 5, 16, 31, 32, 33}.  Before each
set of cases, a long, high-scoring pair runs through the same kernel, so that
stale scratch would show up as a wrong score.

Routes, each against the reference's scalar recurrence (src/simd.rs:347-390)
or band rule (src/align.rs:439-447) restated in the oracle:
  (a) score rows outside int8                       batched and per call
  (b) gap costs outside the 16-bit kernel's range   batched and per call
  (c) score + end cell, and the alignment span      st_sw_score_end[_pairs], st_sw_align_span_pairs
  (d) banded pairs with a negative band centre      batched
  (e) the allocation-free entry point               tests/test_zz_no_alloc.py
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, Kernel, QueryProfile, blosum62
from synth import workloads as W
from sabertooth_b200._lib import PAIR_DTYPE

pytestmark = pytest.mark.gpu

MS = (257, 700, 5000)
NS = (1, 2, 5, 16, 31, 32, 33)


def _cases(seed, wide_rows=False):
    """(rows, target) for every (m, n); targets carry a piece of their query so scores are not all tiny."""
    model = W.Model()
    r = W.Rng(seed)
    rs = np.random.default_rng(seed)
    out = []
    for m in MS:
        for n in NS:
            q = model.background(r, m)
            t = model.background(r, n)
            k = min(n, 12)
            p = int(rs.integers(0, m - k + 1))
            t[:k] = q[p:p + k]
            rows = model.mat.sequence_rows(q)
            if wide_rows:
                rows = rows * 23  # BLOSUM62 x 23: values up to 253, outside int8
                rows[:, 20] = 0
            out.append((np.ascontiguousarray(rows, dtype=np.int32), np.ascontiguousarray(t, dtype=np.uint8)))
    return out


def _stale_fill(ctx, gaps, wide_rows=True):
    """Score one long identical pair through the 32-bit kernel so its scratch holds large H values."""
    m = blosum62()
    q = np.full(3000, 18, dtype=np.uint8)  # W
    rows = m.sequence_rows(q)
    if wide_rows:
        rows = rows * 23
        rows[:, 20] = 0
    ctx.upload_db_list([q])
    ids = ctx.create_profiles([rows])
    pairs = np.zeros(1, dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["band_radius"] = -1
    try:
        s = ctx.sw_score_pairs(pairs, gaps)
        assert s[0] > 100000
    finally:
        ctx.free_profiles(ids)


def _batch(ctx, cases, gaps, centers=None, radii=None):
    ctx.upload_db_list([t for _, t in cases])
    ids = ctx.create_profiles([r for r, _ in cases])
    pairs = np.zeros(len(cases), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(cases))
    pairs["band_center"] = 0 if centers is None else centers
    pairs["band_radius"] = -1 if radii is None else radii
    try:
        return ctx.sw_score_pairs(pairs, gaps, with_kernels=True)
    finally:
        ctx.free_profiles(ids)


@pytest.mark.parametrize("gaps", [(11, 1), (44, 4)])
def test_rows_outside_int8_batched_and_per_call(ctx, gaps):
    g = GapCosts(*gaps)
    cases = _cases(101, wide_rows=True)
    _stale_fill(ctx, g)
    got, kinds = _batch(ctx, cases, g)
    want = np.array([O.gotoh_score(r, t, *gaps) for r, t in cases], dtype=np.int32)
    assert np.array_equal(got, want), [(cases[i][0].shape[0], cases[i][1].size) for i in np.nonzero(got != want)[0]]
    assert np.all(kinds == 2)  # every pair ran on the 32-bit kernel
    _stale_fill(ctx, g)
    for (r, t), w in zip(cases, want):
        qp = QueryProfile.from_rows(r, ctx)
        s, k = qp.sw_score_with(t, g)
        qp.free()
        assert (s, k) == (int(w), Kernel.GPU32), (r.shape[0], t.size)


@pytest.mark.parametrize("gaps", [(20000, 3), (7, -1), (-2, 1)])
def test_gap_costs_outside_16bit_range_batched_and_per_call(ctx, gaps):
    g = GapCosts(*gaps)
    cases = _cases(202)
    _stale_fill(ctx, GapCosts(11, 1))
    got, kinds = _batch(ctx, cases, g)
    want = np.array([O.gotoh_score(r, t, *gaps) for r, t in cases], dtype=np.int32)
    assert np.array_equal(got, want), [(cases[i][0].shape[0], cases[i][1].size) for i in np.nonzero(got != want)[0]]
    assert np.all(kinds == 2)
    _stale_fill(ctx, GapCosts(11, 1))
    for (r, t), w in zip(cases, want):
        qp = QueryProfile.from_rows(r, ctx)
        s, k = qp.sw_score_with(t, g)
        qp.free()
        assert s == int(w), (r.shape[0], t.size)


def _rev_start(rows, t, open_, ext, end):
    s, ie, je = end
    r = O.gotoh_score_end(np.ascontiguousarray(rows[: ie + 1][::-1]), np.ascontiguousarray(t[: je + 1][::-1]),
                          open_, ext)
    assert r[0] == s
    return ie - r[1], je - r[2]


@pytest.mark.parametrize("gaps", [(11, 1), (44, 4)])
def test_end_cells_and_spans(ctx, gaps):
    g = GapCosts(*gaps)
    cases = _cases(303)
    # the reverse pass scores prefixes of the query: put the target's piece late in the query so
    # that the reversed prefix is itself longer than 256 rows
    model = W.Model()
    r = W.Rng(304)
    for m in MS:
        for n in NS:
            q = model.background(r, m)
            t = q[m - n - 3:m - 3].copy() if n + 3 <= m else model.background(r, n)
            cases.append((np.ascontiguousarray(model.mat.sequence_rows(q), dtype=np.int32), t))
    want = [O.gotoh_score_end(rw, t, *gaps) for rw, t in cases]
    _stale_fill(ctx, g)
    ctx.upload_db_list([t for _, t in cases])
    ids = ctx.create_profiles([rw for rw, _ in cases])
    pairs = np.zeros(len(cases), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(cases))
    pairs["band_radius"] = -1
    try:
        s1, ends1 = ctx.sw_score_end_pairs(pairs, g)
        s2, starts, ends2 = ctx.align_span_pairs(pairs, g)
    finally:
        ctx.free_profiles(ids)
    for i, (rw, t) in enumerate(cases):
        w = want[i]
        if w is None:
            assert s1[i] == 0 and tuple(ends1[i]) == (-1, -1) and s2[i] == 0 and tuple(starts[i]) == (-1, -1)
            continue
        assert (int(s1[i]), int(ends1[i][0]), int(ends1[i][1])) == w, (rw.shape[0], t.size)
        assert (int(s2[i]), int(ends2[i][0]), int(ends2[i][1])) == w, (rw.shape[0], t.size)
        assert tuple(int(x) for x in starts[i]) == _rev_start(rw, t, *gaps, w), (rw.shape[0], t.size)
    # the per-call form
    _stale_fill(ctx, g)
    for (rw, t), w in zip(cases, want):
        qp = QueryProfile.from_rows(rw, ctx)
        got = qp.sw_score_end(t, g)
        qp.free()
        assert got == w, (rw.shape[0], t.size)


@pytest.mark.parametrize("gaps", [(11, 1), (44, 4)])
def test_banded_negative_centre(ctx, gaps):
    g = GapCosts(*gaps)
    base = _cases(404)
    cases, centers, radii = [], [], []
    for rw, t in base:
        m = rw.shape[0]
        for center, radius in ((-3, 2), (-40, 64), (-(m - 20), 10), (-1, 0), (-300, 64)):
            cases.append((rw, t))
            centers.append(center)
            radii.append(radius)
    _stale_fill(ctx, g)
    got, kinds = _batch(ctx, cases, g, np.array(centers, np.int32), np.array(radii, np.int32))
    want = np.array([O.band_score(rw, t, *gaps, c, rd) for (rw, t), c, rd in zip(cases, centers, radii)],
                    dtype=np.int32)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, [(cases[i][0].shape[0], cases[i][1].size, centers[i], radii[i]) for i in bad[:8]]
