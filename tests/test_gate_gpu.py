"""GPU parity of the prefilter evidence / chain / gate path against the oracle.

The CUDA path (st_prefilter_gate) must give the oracle's candidate list
(src/prefilter.rs:1412-1660 and the ranking :1074-1083) field for field and in
the same order, and the same evidence counters: on the reference's own prefilter
tests (brute-force seed hits), on two-piece homolog workloads across the
parameter space, on rows outside int8, on edge cases (no hits, one hit,
duplicates, rejected hits) and on a million-hit batch.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, PrefilterParams, blosum62, encode
from synth import workloads as W
from sabertooth_b200._lib import SEED_HIT_DTYPE, StError
from tests.seedhits import brute_seed_hits, default_params

pytestmark = pytest.mark.gpu

STATS = ("targets_hit", "targets_evaluated", "diagonals_scored", "chains_used", "candidates", "candidates_capped")


def _params(p):
    return PrefilterParams(min_hits=p["min_hits"], min_diag_score=p["min_diag_score"], diag_hits=p["diag_hits"],
                           max_diagonals=p["max_diagonals"], max_candidates=p["max_candidates"],
                           regions=bool(p["regions"]), diag_window=p["diag_window"], span=p["span"])


def _targets(w):
    return [w.db_residues[int(a):int(b)] for a, b in zip(w.db_offsets[:-1], w.db_offsets[1:])]


def _check(ctx, rows, targets, hits, p, upload=True):
    """hits: SEED_HIT_DTYPE with query = index into rows."""
    if upload:
        ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    try:
        want, wst = O.prefilter_queries(O.Arena(rows, targets), hits["query"], hits["target"], hits["diag"],
                                        hits["qpos"], p)
        h = hits.copy()
        h["query"] = ids[hits["query"]]
        got, gst = ctx.prefilter_gate(h, _params(p), GapCosts(p["gap_open"], p["gap_ext"]))
        assert len(got) == len(want)
        for q in range(len(rows)):
            g = got[got["query"] == ids[q]].copy()
            g["query"] = q
            wq = want[want["query"] == q]
            assert np.array_equal(g, wq), q
        # queries come out in ascending profile id order
        assert np.all(np.diff(got["query"].astype(np.int64)) >= 0)
        for k in STATS:
            assert gst[k] == wst[k], k
        assert gst["hits_rejected"] == 0
        return got, gst
    finally:
        ctx.free_profiles(ids)


def _as_hits(tuples):
    a = np.zeros(len(tuples), dtype=SEED_HIT_DTYPE)
    for i, t in enumerate(tuples):
        a[i] = t
    return a


def test_reference_prefilter_cases(ctx):
    # src/prefilter.rs:1926-1959 on brute-force seed hits (k = 6 / 22 and k = 4 / 18)
    m = blosum62()
    q1, t1 = encode("MKVLLACDEFGHIK"), encode("MKVLLACDEFGHIKMKVLLAC")
    got, _ = _check(ctx, [m.sequence_rows(q1)], [t1], _as_hits(brute_seed_hits(m.score, q1, [t1], 6, 22)),
                    default_params(span=6))
    assert got[0]["best_diag"] == 0 and got[0]["diag_score"] > 0
    q = encode("MKVLLACDEFGHIKLMNPQRSTVWYHHHHWWCCMM")
    t = encode("QRSTQRSTQRSTQRSTQRSTQRSTQRST" + "MKVLLACDEFGHIKLMNP" + "GGGGQRSTVWYHHHHWWCCMM")
    hits = _as_hits(brute_seed_hits(m.score, q, [t], 4, 18))
    one, _ = _check(ctx, [m.sequence_rows(q)], [t], hits, default_params(span=4, max_diagonals=1))
    four, st = _check(ctx, [m.sequence_rows(q)], [t], hits, default_params(span=4))
    assert len(four) == 1 and st["chains_used"] == 1
    assert four[0]["diag_score"] > (int(one[0]["diag_score"]) if len(one) else 0)


@pytest.mark.parametrize("kw", [dict(), dict(diag_window=0), dict(max_diagonals=1), dict(max_diagonals=2),
                                dict(max_diagonals=16), dict(max_diagonals=20), dict(diag_hits=2),
                                dict(min_hits=3), dict(regions=1), dict(min_diag_score=0, regions=1),
                                dict(max_candidates=5), dict(max_candidates=1, regions=1, diag_window=0),
                                dict(span=9, diag_window=10, gap_open=44, gap_ext=4)])
def test_split_homologs_across_parameters(ctx, kw):
    w = W.seed_hits(seed=21, n_queries=40, n_targets=2500, n_hits=120_000, homolog_frac=0.3, keep=0.6)
    p = default_params(**dict(dict(min_diag_score=25), **kw))
    _, st = _check(ctx, w.rows, _targets(w), w.hits, p)
    assert st["candidates"] > 0


def test_chains_are_exercised(ctx):
    w = W.seed_hits(seed=5, n_queries=20, n_targets=1500, n_hits=80_000, homolog_frac=0.5, keep=0.8)
    _, st = _check(ctx, w.rows, _targets(w), w.hits, default_params(regions=1))
    assert st["chains_used"] > 0


def test_rows_outside_int8(ctx):
    rng = np.random.default_rng(8)
    rows = [rng.integers(-300, 400, size=(int(rng.integers(20, 120)), 21)).astype(np.int32) for _ in range(5)]
    targets = [rng.integers(0, 21, size=int(rng.integers(30, 300))).astype(np.uint8) for _ in range(200)]
    tl = np.array([len(t) for t in targets])
    n = 20000
    q = rng.integers(0, 5, n)
    t = rng.integers(0, 200, n)
    m = np.array([len(r) for r in rows])[q]
    qp = (rng.random(n) * m).astype(np.int64)
    tp = (rng.random(n) * tl[t]).astype(np.int64)
    hits = np.zeros(n, dtype=SEED_HIT_DTYPE)
    hits["query"], hits["target"], hits["diag"], hits["qpos"] = q, t, tp - qp, qp
    _check(ctx, rows, targets, hits, default_params(min_diag_score=800, regions=1))


def test_edge_cases(ctx):
    m = blosum62()
    rng = np.random.default_rng(2)
    rows = [m.sequence_rows(rng.integers(0, 20, 50).astype(np.uint8))]
    targets = [rng.integers(0, 20, int(k)).astype(np.uint8) for k in (5, 60, 200)]
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    try:
        got, st = ctx.prefilter_gate(np.zeros(0, dtype=SEED_HIT_DTYPE))
        assert len(got) == 0 and st["targets_hit"] == 0
        # a hit outside its target is rejected with an error
        bad = _as_hits([(ids[0], 0, 10, 1)])  # target 0 has 5 residues: position 11
        with pytest.raises(StError):
            ctx.prefilter_gate(bad)
        unknown = _as_hits([(0xFFFFFFF0, 1, 0, 0)])
        with pytest.raises(StError):
            ctx.prefilter_gate(unknown)
        with pytest.raises(StError):
            ctx.prefilter_gate(_as_hits([(ids[0], 1, 0, 0)]), PrefilterParams(max_diagonals=0))
    finally:
        ctx.free_profiles(ids)
    # one hit; the same hit many times; all hits on one diagonal
    for hits in ([(0, 2, 3, 10)], [(0, 2, 3, 10)] * 50, [(0, 1, -5, k) for k in range(5, 50)]):
        _check(ctx, rows, targets, _as_hits(hits), default_params(min_diag_score=0, regions=1), upload=False)


def test_million_hits(ctx):
    w = W.seed_hits(seed=33, n_queries=300, n_targets=60_000, n_hits=1_000_000)
    _, st = _check(ctx, w.rows, _targets(w), w.hits, default_params(regions=1, max_candidates=50))
    assert st["candidates"] > 0 and st["chains_used"] > 0


def test_device_buffers_match_host(ctx):
    import torch
    w = W.seed_hits(seed=9, n_queries=30, n_targets=3000, n_hits=100_000)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(w.rows)
    try:
        h = w.hits.copy()
        h["query"] = ids[h["query"]]
        host, hst = ctx.prefilter_gate(h)
        d_h = torch.from_numpy(h.view(np.uint8).copy()).cuda()
        d_o = torch.zeros(len(h) * 32, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        n, dst = ctx.prefilter_gate_device(d_h.data_ptr(), len(h), d_o.data_ptr())
        torch.cuda.synchronize()
        dev = d_o.cpu().numpy()[:n * 32].view(host.dtype)
        assert np.array_equal(dev, host) and dst == hst
    finally:
        ctx.free_profiles(ids)
