"""The CPU oracle pinned against the reference's known answers and its own
differential strategy (an independent three-matrix Gotoh), on the CPU.

Known answers restated from the reference's tests:
  * W x 4000 against itself at 11/1 scores 4000 * s(W,W) (> i16::MAX)  src/simd.rs:1328-1341
  * W x (32767 / s(W,W) - 2) scores n * s(W,W)                        src/simd.rs:1343-1346
  * W x 3000 end cell is (3000 * s(W,W), 2999, 2999)                  src/simd.rs:1229-1233
  * rows [[40000; 21]; 3] against [0, 1, 2] score 120,000            src/simd.rs:1351-1355
  * the in-band score with radius 2 is below the full score         src/align.rs:1385-1396
  * kadane_segment's score equals kadane_score on every diagonal     src/ungapped.rs:531-548
"""
import numpy as np

from oracle import oracle as O
from sabertooth_b200 import blosum62, encode
from tests.refrng import SplitMix64, XorShift, rand_seq


def test_saturation_known_answers():
    m = blosum62()
    w = int(encode("W")[0])
    sww = int(m.score[w, w])
    q = np.full(4000, w, dtype=np.uint8)
    rows = m.sequence_rows(q)
    assert O.gotoh_score(rows, q, 11, 1) == 4000 * sww > 32767
    n = 32767 // sww - 2
    assert O.gotoh_score(rows[:n], q[:n], 11, 1) == n * sww
    q3 = q[:3000]
    assert O.gotoh_score_end(rows[:3000], q3, 11, 1) == (3000 * sww, 2999, 2999)


def test_huge_rows_known_answer():
    rows = np.full((3, 21), 40000, dtype=np.int32)
    assert O.gotoh_score(rows, [0, 1, 2], 11, 1) == 120000


def test_gotoh_matches_three_matrix_reference_across_gap_costs():
    m = blosum62()
    rng = XorShift(12345)
    for open_, ext in [(1, 1), (2, 1), (3, 1), (2, 0), (4, 1), (11, 1), (6, 2), (5, 5)]:
        for _ in range(150):
            ql, tl = 1 + rng.range(90), 1 + rng.range(90)
            alpha = 2 + rng.range(19)
            q = rand_seq(rng, ql, alpha)
            t = rand_seq(rng, tl, alpha)
            rows = m.sequence_rows(q)
            assert O.gotoh_score(rows, t, open_, ext) == O.reference_score(rows, t, open_, ext)


def test_end_cell_is_first_column_major_optimum():
    # src/simd.rs:1167-1195 reference_end: scan columns, then rows, strict improvement
    m = blosum62()
    rng = XorShift(424242)
    for _ in range(200):
        q = rand_seq(rng, 1 + rng.range(40), 2 + rng.range(3))
        t = rand_seq(rng, 1 + rng.range(40), 2 + rng.range(3))
        rows = m.sequence_rows(q)
        h = full_h(rows, t, 11, 1)
        best = (0, 0, 0)
        for j in range(1, len(t) + 1):
            for i in range(1, len(q) + 1):
                if h[i][j] > best[0]:
                    best = (h[i][j], i - 1, j - 1)
        want = best if best[0] > 0 else None
        assert O.gotoh_score_end(rows, t, 11, 1) == want


def full_h(rows, t, open_, ext):
    mq, n = len(rows), len(t)
    neg = -(2 ** 31) // 4
    h = [[0] * (n + 1) for _ in range(mq + 1)]
    e = [[neg] * (n + 1) for _ in range(mq + 1)]
    f = [[neg] * (n + 1) for _ in range(mq + 1)]
    for i in range(1, mq + 1):
        for j in range(1, n + 1):
            e[i][j] = max(h[i][j - 1] - open_, e[i][j - 1] - ext)
            f[i][j] = max(h[i - 1][j] - open_, f[i - 1][j] - ext)
            r = t[j - 1]
            sc = int(rows[i - 1][r]) if r < 21 else 0
            h[i][j] = max(h[i - 1][j - 1] + sc, e[i][j], f[i][j], 0)
    return h


def test_band_rule():
    m = blosum62()
    q = encode("MKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIK")
    t = encode("MKVLLACDEFGHIKGGGGGGGGGGLMNPQRSTVWYACDEFGHIK")
    rows = m.sequence_rows(q)
    full = O.gotoh_score(rows, t, 11, 1)
    assert O.band_score(rows, t, 11, 1, 0, 2) < full
    assert O.band_score(rows, t, 11, 1, 0, 10_000) == full
    assert O.band_score(rows, t, 11, 1, 0, -1) == full
    # brute-force band semantics on small random cases
    rng = XorShift(99)
    for _ in range(100):
        q = rand_seq(rng, 1 + rng.range(25), 20)
        tt = rand_seq(rng, 1 + rng.range(40), 20)
        c, r = rng.range(20) - 10, rng.range(6)
        rows = m.sequence_rows(q)
        assert O.band_score(rows, tt, 11, 1, c, r) == brute_band(rows, tt, 11, 1, c, r)


def brute_band(rows, t, open_, ext, c, r):
    mq, n = len(rows), len(t)
    neg = -(2 ** 31) // 4
    h = [[0] * (n + 1) for _ in range(mq + 1)]
    e = [[neg] * (n + 1) for _ in range(mq + 1)]
    f = [[neg] * (n + 1) for _ in range(mq + 1)]
    best = 0
    for i in range(1, mq + 1):
        for j in range(1, n + 1):
            if abs(j - i - c) > r:
                continue  # H = 0, E = F = -inf
            e[i][j] = max(h[i][j - 1] - open_, e[i][j - 1] - ext)
            f[i][j] = max(h[i - 1][j] - open_, f[i - 1][j] - ext)
            sc = int(rows[i - 1][t[j - 1]])
            h[i][j] = max(h[i - 1][j - 1] + sc, e[i][j], f[i][j], 0)
            best = max(best, h[i][j])
    return best


def test_kadane_segment_and_score_agree():
    rng = SplitMix64(3)
    m = blosum62()
    for _ in range(100):
        q = [rng.below(21) for _ in range(1 + rng.below(80))]
        t = [rng.below(21) for _ in range(1 + rng.below(120))]
        rows = m.sequence_rows(q)
        for d in range(-len(q) - 2, len(t) + 2):
            lo, hi = O.diag_range(len(q), len(t), d)
            s = O.kadane_score(rows, t, d, lo, hi)
            assert s == O.kadane_segment(rows, t, d, lo, hi)[0]
            assert s == brute_kadane(rows, t, d, lo, hi)
            if hi > lo + 2:
                assert O.kadane_score(rows, t, d, lo + 1, hi - 1) == O.kadane_segment(rows, t, d, lo + 1, hi - 1)[0]


def brute_kadane(rows, t, d, lo, hi):
    best = 0
    for a in range(lo, hi):
        s = 0
        for b in range(a, hi):
            s += int(rows[b][t[b + d]]) if t[b + d] < 21 else 0
            best = max(best, s)
    return best


def test_diag_range():
    assert O.diag_range(10, 20, 0) == (0, 10)
    assert O.diag_range(10, 20, -3) == (3, 10)
    assert O.diag_range(10, 5, 2) == (0, 3)
    assert O.diag_range(10, 5, 5) == (0, 0)
    assert O.diag_range(10, 5, -10) == (0, 0)


def test_striped_cpu_baseline_equals_scalar_oracle():
    """The AVX2 restatement of the reference's CPU path (the timed CPU baseline) gives the oracle's scores,
    including u8 headroom fallbacks, i16 saturation and gap costs that force the scalar path."""
    from synth import workloads as W
    m = blosum62()
    rng = XorShift(777)
    rows_list, targets, pq, pt = [], [], [], []
    for i in range(120):
        q = rand_seq(rng, 1 + rng.range(140), 2 + rng.range(19))
        t = rand_seq(rng, 1 + rng.range(200), 2 + rng.range(19))
        if i % 5 == 0:
            p = rng.range(len(t) + 1)
            t = t[:p] + q + t[p:]
        rows_list.append(m.sequence_rows(q))
        targets.append(t)
        pq.append(i)
        pt.append(i)
    w = np.full(4000, int(encode("W")[0]), dtype=np.uint8)
    rows_list.append(m.sequence_rows(w))
    targets.append(w)
    pq.append(len(rows_list) - 1)
    pt.append(len(targets) - 1)
    ar = O.Arena(rows_list, targets)
    for open_, ext in [(11, 1), (6, 2), (5, 5), (1, 1), (44, 4), (300, 1)]:
        want = O.sw_pairs(ar, pq, pt, open_, ext)
        got, kinds = O.striped_pairs(ar, pq, pt, open_, ext, with_kinds=True)
        assert np.array_equal(got, want), (open_, ext)
    assert kinds[-1] == 3  # the saturating W x 4000 pair falls back to the scalar path
    pw = W.config3(seed=5, n_queries=10, db_residues=30_000, per_query=30)
    ar = O.Arena(pw.rows, pw.targets())
    assert np.array_equal(O.striped_pairs(ar, pw.pair_q, pw.pair_t, 44, 4), O.sw_pairs(ar, pw.pair_q, pw.pair_t, 44, 4))


def test_avx2_ungapped_baseline_equals_scalar_kadane():
    """The AVX2 restatement of the reference's batched Kadane (the CPU baseline of ungapped scoring)
    gives the scalar oracle's score on every hit: BLOSUM62 rows on the u8 path, rows with scores
    high enough to saturate u8 (rescored), and PSSM-like rows outside the u8 range (scalar)."""
    from synth import workloads as W
    w = W.config2(seed=7, n_queries=40, n_targets=3000, n_hits=60_000)
    targets = [w.db_residues[int(a):int(b)] for a, b in zip(w.db_offsets[:-1], w.db_offsets[1:])]
    rows = list(w.rows)
    rows[3] = rows[3] * 9           # max 99 -> u8 headroom exceeded on long windows, lanes rescored
    rows[5] = rows[5] * 40          # outside u8 -> every lane scalar
    ar = O.Arena(rows, targets)
    h = w.hits
    want = O.ungapped_hits(ar, h["query"], h["target"], h["diag"])
    got = O.ungapped_hits_avx2(ar, h["query"], h["target"], h["diag"])
    assert np.array_equal(got, want)
    assert (want[h["query"] == 3] > 160).any()
