"""GPU parity of the Smith-Waterman-Gotoh score path against the CPU oracle.

Cases follow the reference's own tests (src/simd.rs:1064-1355,
src/align.rs:1223-1396): gap-cost sweeps with the same xorshift seeds,
saturation and huge-row known answers, adjacent gap runs across stripes, X and
out-of-alphabet codes, the in-band heuristic, plus GPU-specific coverage
(every tile class, multi-pass queries, long targets, mixed batches).
Bar: bit-exact integer scores.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, Kernel, QueryProfile, blosum62, encode, tile_classes
from synth import workloads as W
from tests.refrng import XorShift, rand_seq

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("planner")]

GAP_SWEEP = [(1, 1), (2, 1), (3, 1), (2, 0), (4, 1), (11, 1), (6, 2), (5, 5)]


def batch_scores(ctx, rows_list, targets, pairs, gaps, centers=None, radii=None, with_kernels=False):
    """Upload the targets as the database, create the profiles, score pairs (q, t) in one batched call."""
    ctx.upload_db_list([np.asarray(t, dtype=np.uint8) for t in targets])
    ids = ctx.create_profiles(rows_list)
    arr = np.zeros(len(pairs), dtype=[("profile", "<u4"), ("target", "<u4"), ("band_center", "<i4"),
                                      ("band_radius", "<i4")])
    arr["profile"] = ids[[p[0] for p in pairs]]
    arr["target"] = [p[1] for p in pairs]
    arr["band_center"] = 0 if centers is None else centers
    arr["band_radius"] = -1 if radii is None else radii
    try:
        return ctx.sw_score_pairs(arr, gaps, with_kernels=with_kernels)
    finally:
        for i in ids:
            ctx.free_profile(i)


def test_gap_cost_sweep_batched_matches_oracle(ctx):
    m = blosum62()
    rng = XorShift(12345)
    for open_, ext in GAP_SWEEP:
        rows_list, targets, want = [], [], []
        for _ in range(800):
            ql, tl = 1 + rng.range(90), 1 + rng.range(90)
            alpha = 2 + rng.range(19)
            q = rand_seq(rng, ql, alpha)
            t = rand_seq(rng, tl, alpha)
            rows = m.sequence_rows(q)
            rows_list.append(rows)
            targets.append(t)
            want.append(O.reference_score(rows, t, open_, ext))
        got = batch_scores(ctx, rows_list, targets, [(i, i) for i in range(len(targets))], GapCosts(open_, ext))
        assert np.array_equal(got, np.array(want, dtype=np.int32)), (open_, ext, np.nonzero(got != want)[0][:5])


def test_gap_cost_sweep_plain_per_call(ctx):
    m = blosum62()
    rng = XorShift(12345)
    for open_, ext in GAP_SWEEP:
        for _ in range(40):
            ql, tl = 1 + rng.range(90), 1 + rng.range(90)
            alpha = 2 + rng.range(19)
            q = rand_seq(rng, ql, alpha)
            t = np.array(rand_seq(rng, tl, alpha), dtype=np.uint8)
            rows = m.sequence_rows(q)
            qp = QueryProfile.from_rows(rows, ctx)
            s, k = qp.sw_score_with(t, GapCosts(open_, ext))
            qp.free()
            assert s == O.gotoh_score(rows, t, open_, ext), (open_, ext, q, list(t))
            assert k in (Kernel.GPU16, Kernel.GPU32)


def test_saturation_falls_back_to_exact_32bit(ctx):
    # src/simd.rs:1328-1348: identical 4000-residue W runs exceed i16::MAX
    m = blosum62()
    w = int(encode("W")[0])
    sww = int(m.score[w, w])
    q = np.full(4000, w, dtype=np.uint8)
    qp = QueryProfile.from_rows(m.sequence_rows(q), ctx)
    s, k = qp.sw_score_with(q, GapCosts.sequence_default())
    assert k == Kernel.GPU32
    assert s == 4000 * sww and s > 32767
    n = 32767 // sww - 2
    s2, k2 = qp.sw_score_with(q[:n], GapCosts.sequence_default())
    assert k2 == Kernel.GPU16
    assert s2 == n * sww
    qp.free()


def test_huge_table_scores_use_32bit(ctx):
    # src/simd.rs:1351-1355
    qp = QueryProfile.from_rows(np.full((3, 21), 40000, dtype=np.int32), ctx)
    s, k = qp.sw_score_with(np.array([0, 1, 2], dtype=np.uint8), GapCosts.sequence_default())
    assert (s, k) == (120000, Kernel.GPU32)
    qp.free()


def test_adjacent_gap_runs_across_stripes(ctx):
    # src/simd.rs:1237-1261
    rows = np.full((40, 21), -40, dtype=np.int32)
    for c in range(40):
        rows[c, c % 20] = 30
    tbl_t = [x % 20 for x in list(range(20)) + [5, 5, 5] + list(range(26, 40))]
    rng = XorShift(77)
    for open_, ext in [(44, 4), (20, 1), (12, 2)]:
        targets = [tbl_t] + [rand_seq(rng, 10 + rng.range(60), 20) for _ in range(400)]
        want = [O.reference_score(rows, t, open_, ext) for t in targets]
        got = batch_scores(ctx, [rows], targets, [(0, i) for i in range(len(targets))], GapCosts(open_, ext))
        assert np.array_equal(got, np.array(want, dtype=np.int32)), (open_, ext)


def test_x_and_out_of_alphabet_residues(ctx):
    # src/simd.rs:1306-1325
    m = blosum62()
    q = rand_seq(XorShift(7), 30, 20)
    t = np.array(rand_seq(XorShift(9), 40, 20), dtype=np.uint8)
    t[[5, 15, 20]] = 20
    rows = m.sequence_rows(q)
    qp = QueryProfile.from_rows(rows, ctx)
    g = GapCosts.sequence_default()
    assert qp.sw_score(t, g) == O.gotoh_score(rows, t, 11, 1)
    odd = t.copy()
    odd[7] = 200
    assert qp.sw_score(odd, g) == O.gotoh_score(rows, odd, 11, 1)
    qp.free()


def test_empty_inputs_score_zero(ctx):
    # src/simd.rs:253-255
    m = blosum62()
    qp = QueryProfile.from_rows(m.sequence_rows(encode("MKV")), ctx)
    assert qp.sw_score_with(np.zeros(0, np.uint8), GapCosts.sequence_default()) == (0, Kernel.NONE)
    qp.free()
    e = QueryProfile.from_rows(np.zeros((0, 21), np.int32), ctx)
    assert e.sw_score_with(encode("MKV"), GapCosts.sequence_default()) == (0, Kernel.NONE)
    e.free()


def test_gap_costs_outside_16bit_range(ctx):
    m = blosum62()
    rng = XorShift(4242)
    for open_, ext in [(0, 0), (3, -1), (-2, 1), (20000, 5), (40, 30000), (1, 5)]:
        rows_list, targets, want = [], [], []
        for _ in range(60):
            q = rand_seq(rng, 1 + rng.range(70), 20)
            t = rand_seq(rng, 1 + rng.range(70), 20)
            rows = m.sequence_rows(q)
            rows_list.append(rows)
            targets.append(t)
            want.append(O.gotoh_score(rows, t, open_, ext))
        got = batch_scores(ctx, rows_list, targets, [(i, i) for i in range(60)], GapCosts(open_, ext))
        assert np.array_equal(got, np.array(want, dtype=np.int32)), (open_, ext)


def test_in_band_heuristic_reports_its_own_score(ctx):
    # src/align.rs:1385-1396: the band can only lower the score
    m = blosum62()
    q = encode("MKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIK")
    t = encode("MKVLLACDEFGHIKGGGGGGGGGGLMNPQRSTVWYACDEFGHIK")
    rows = m.sequence_rows(q)
    full = O.gotoh_score(rows, t, 11, 1)
    narrow_want = O.band_score(rows, t, 11, 1, 0, 2)
    assert narrow_want < full
    got = batch_scores(ctx, [rows], [t], [(0, 0), (0, 0)], GapCosts(11, 1), centers=[0, 0], radii=[2, -1])
    assert list(got) == [narrow_want, full]


def test_banded_random(ctx):
    m = blosum62()
    rng = XorShift(31337)
    rows_list, targets, centers, radii, want = [], [], [], [], []
    for i in range(300):
        q = rand_seq(rng, 1 + rng.range(300), 20)
        t = rand_seq(rng, 1 + rng.range(1500), 20)
        if i % 3 == 0 and len(t) > len(q):  # plant the query on a diagonal
            p = rng.range(len(t) - len(q) + 1)
            t[p:p + len(q)] = q
        c = int(rng.range(len(t) + 40)) - 20
        r = [0, 1, 3, 16, 64, 200][i % 6]
        rows = m.sequence_rows(q)
        rows_list.append(rows)
        targets.append(t)
        centers.append(c)
        radii.append(r)
        want.append(O.band_score(rows, t, 11, 1, c, r))
    got, kern = batch_scores(ctx, rows_list, targets, [(i, i) for i in range(300)], GapCosts(11, 1), centers, radii,
                             with_kernels=True)
    assert np.array_equal(got, np.array(want, dtype=np.int32)), np.nonzero(got != np.array(want))[0][:8]
    # banded pairs with int8 rows take the packed band kernel (16-bit cells, 32-bit past the headroom)
    assert set(kern.tolist()) <= {int(Kernel.GPU16), int(Kernel.GPU32), int(Kernel.NONE)}
    assert (kern == int(Kernel.GPU16)).sum() > 0


def test_multipass_queries_and_long_targets(ctx):
    model = W.Model()
    r = W.Rng(5)
    rows_list, targets, pairs = [], [], []
    for i, (m_, n_) in enumerate([(600, 800), (1500, 300), (3000, 1200), (257, 35000), (2048, 2048), (5000, 400)]):
        q = model.background(r, m_)
        t = model.background(r, n_)
        if i % 2 == 0:
            k = min(m_, n_) // 2
            t[:k] = model.mutate(r, q[:k], 0.9)
        rows_list.append(model.mat.sequence_rows(q))
        targets.append(t)
        pairs.append((i, i))
    for g in [GapCosts(11, 1), GapCosts(44, 4)]:
        want = [O.gotoh_score(rows_list[q], targets[t], g.open, g.extend) for q, t in pairs]
        got = batch_scores(ctx, rows_list, targets, pairs, g)
        assert np.array_equal(got, np.array(want, dtype=np.int32))


def test_every_tile_class(ctx):
    model = W.Model()
    r = W.Rng(11)
    rows_list, targets, pairs, want = [], [], [], []
    for i in range(64):
        m_ = int(W.lognormal_lengths(r, 1, 200, 0.9, 1, 1200)[0])
        q = model.background(r, m_)
        for j in range(3):
            n_ = int(W.lognormal_lengths(r, 1, 200, 0.9, 1, 1500)[0])
            t = model.background(r, n_) if j else model.mutate(r, q, 0.5, 0.02)
            targets.append(t)
            pairs.append((i, len(targets) - 1))
        rows_list.append(model.mat.sequence_rows(q))
    want = np.array([O.gotoh_score(rows_list[q], targets[t], 11, 1) for q, t in pairs], dtype=np.int32)
    saved = ctx.tuning_table()
    try:
        for c in range(len(tile_classes())):
            ctx.set_tuning_table(np.full((10, 8), c, dtype=np.int32))
            got, kern = batch_scores(ctx, rows_list, targets, pairs, GapCosts(11, 1), with_kernels=True)
            assert np.array_equal(got, want), (c, tile_classes()[c], np.nonzero(got != want)[0][:5])
            assert (kern == int(Kernel.GPU16)).mean() > 0.9
    finally:
        ctx.set_tuning_table(saved)


def test_pssm_workload_small(ctx):
    w = W.config3(seed=3, n_queries=24, db_residues=60_000, per_query=40)
    ar = O.Arena(w.rows, w.targets())
    want = O.sw_pairs(ar, w.pair_q, w.pair_t, 44, 4)
    got = batch_scores(ctx, w.rows, w.targets(), list(zip(w.pair_q.tolist(), w.pair_t.tolist())), GapCosts(44, 4))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kind", ["blosum62", "pssm"])
def test_long_overflow_band_mix_small(ctx, kind):
    w = W.config4(seed=1, n_pairs=60, kind=kind, near_identical=0.2)
    ar = O.Arena(w.rows, w.targets())
    want = O.sw_pairs(ar, w.pair_q, w.pair_t, w.gap_open, w.gap_extend, w.band_center.astype(np.int64),
                      w.band_radius.astype(np.int64))
    got = batch_scores(ctx, w.rows, w.targets(), list(zip(w.pair_q.tolist(), w.pair_t.tolist())),
                       GapCosts(w.gap_open, w.gap_extend), w.band_center, w.band_radius)
    assert np.array_equal(got, want)


def test_mixed_batch_alone_equals_in_the_mix(ctx):
    """A pair's score does not depend on what else is in the batch."""
    model = W.Model()
    r = W.Rng(21)
    rows_list = [model.mat.sequence_rows(model.background(r, int(l))) for l in [0, 40, 300, 900, 2500]]
    rows_list.append(np.full((5, 21), 300, dtype=np.int32))  # wide rows: 32-bit path
    targets = [model.background(r, int(l)) for l in [0, 50, 400, 1000, 3000]]
    targets.append(np.asarray(model.mutate(r, np.zeros(0, np.uint8), 1.0)))
    pairs = [(q, t) for q in range(len(rows_list)) for t in range(len(targets))]
    mix = batch_scores(ctx, rows_list, targets, pairs, GapCosts(11, 1))
    for k in [0, 7, 13, 20, len(pairs) - 1]:
        alone = batch_scores(ctx, rows_list, targets, [pairs[k]], GapCosts(11, 1))
        assert alone[0] == mix[k]
    want = [O.gotoh_score(rows_list[q], targets[t], 11, 1) for q, t in pairs]
    assert np.array_equal(mix, np.array(want, dtype=np.int32))
