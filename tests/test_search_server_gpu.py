"""The search server (st_search_server_*): requests submitted one by one and
from several threads complete with the candidates and SW scores of the same
query searched alone (st_prefilter_queries + st_sw_score_pairs), for sequence
and profile queries; waiting with too little room reports the count and keeps
the request."""
import threading

import numpy as np
import pytest

from sabertooth_b200 import GapCosts, PrefilterParams, SearchServer, blosum62
from synth import workloads as W
from sabertooth_b200._lib import PAIR_DTYPE, check, lib, ptr

pytestmark = pytest.mark.gpu


def _alone(ctx, rows, residues, params, gaps):
    ids = ctx.create_profiles([rows])
    try:
        c, _, _ = ctx.prefilter_queries(ids, None if residues is None else [residues], params, gaps)
        pairs = np.zeros(len(c), dtype=PAIR_DTYPE)
        pairs["profile"], pairs["target"], pairs["band_radius"] = c["query"], c["target"], -1
        sc = ctx.sw_score_pairs(pairs, gaps) if len(c) else np.zeros(0, np.int32)
        c = c.copy()
        c["query"] = 0
        return c, sc
    finally:
        ctx.free_profiles(ids)


def test_requests_equal_queries_searched_alone(ctx):
    w = W.config5(seed=4, n_queries=24, n_targets=20_000)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ctx.seed_index_build("111001101")
    params = PrefilterParams(min_diag_score=30, regions=True)
    gaps = GapCosts.sequence_default()
    want = [_alone(ctx, w.rows[q], w.queries[q], params, gaps) for q in range(len(w.rows))]
    srv = SearchServer(ctx, params, gaps)
    try:
        ids = [None] * len(w.rows)

        def submit(qs):
            for q in qs:
                ids[q] = srv.submit(w.rows[q], w.queries[q])

        th = [threading.Thread(target=submit, args=(range(k, len(w.rows), 3),)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        found = 0
        for q in range(len(w.rows)):
            c, sc, lat = srv.wait(ids[q])
            assert np.array_equal(c, want[q][0]), q
            assert np.array_equal(sc, want[q][1]), q
            assert lat > 0
            found += len(c)
        assert found > 0
        st = srv.stats()
        assert st["queries"] == len(w.rows) and st["batches"] >= 1
        # too little room: the count comes back and the request stays
        rid = srv.submit(w.rows[0], w.queries[0])
        n = np.zeros(1, dtype=np.uint64)
        check(lib.st_search_server_wait(srv._h, rid, None, None, 0, ptr(n), None))
        assert int(n[0]) == len(want[0][0])
        c, sc, _ = srv.wait(rid)
        assert np.array_equal(c, want[0][0])
    finally:
        srv.close()


def test_profile_queries(ctx):
    w = W.config3(seed=5, n_queries=8, db_residues=200_000, per_query=5)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ctx.seed_index_build("11111")
    params = PrefilterParams.profile_default()
    gaps = GapCosts.profile_default()
    want = [_alone(ctx, r, None, params, gaps) for r in w.rows]
    srv = SearchServer(ctx, params, gaps, sequence_queries=False, max_batch_queries=3)
    try:
        ids = [srv.submit(r) for r in w.rows]
        for q, rid in enumerate(ids):
            c, sc, _ = srv.wait(rid)
            assert np.array_equal(c, want[q][0]) and np.array_equal(sc, want[q][1]), q
    finally:
        srv.close()
