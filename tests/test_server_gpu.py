"""The serving loop (continuous batching): every request's scores equal the oracle's and
the same request scored alone, whatever else is in flight; budget admission."""
import threading

import numpy as np
import pytest

from oracle import oracle as O
from sabertooth_b200 import GapCosts, Server
from synth import workloads as W

pytestmark = pytest.mark.gpu


def _requests(w):
    """One request per query: its rows and its candidate targets (with bands)."""
    out = []
    for q in range(len(w.rows)):
        sel = np.nonzero(w.pair_q == q)[0]
        if len(sel):
            bc = None if w.band_center is None else w.band_center[sel]
            br = None if w.band_radius is None else w.band_radius[sel]
            out.append((q, sel, w.rows[q], w.pair_t[sel], bc, br))
    return out


def test_alone_equals_mix_equals_oracle(ctx):
    w = W.config3(seed=31, n_queries=40, db_residues=60_000, per_query=50)
    ctx.upload_db(w.db_residues, w.db_offsets)
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4)
    reqs = _requests(w)
    srv = Server(ctx, GapCosts(44, 4))
    try:
        alone = {}
        for q, sel, rows, t, bc, br in reqs:  # one at a time
            alone[q] = srv.wait(srv.submit(rows, t))[0]
        # all at once from four client threads, waited in reverse order
        ids = {}
        lock = threading.Lock()

        def client(part):
            for q, sel, rows, t, bc, br in part:
                rid = srv.submit(rows, t)
                with lock:
                    ids[q] = rid

        th = [threading.Thread(target=client, args=(reqs[k::4],)) for k in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        mix = {q: srv.wait(ids[q])[0] for q in sorted(ids, reverse=True)}
        for q, sel, rows, t, bc, br in reqs:
            assert np.array_equal(alone[q], want[sel]), q
            assert np.array_equal(mix[q], want[sel]), q
        st = srv.stats()
        assert st["pairs"] == 2 * w.n_pairs
        assert st["batches"] < 2 * len(reqs)  # the mix was batched
    finally:
        srv.close()


def test_banded_long_requests_and_budget(ctx):
    w = W.config4(seed=5, n_pairs=60, kind="blosum62", near_identical=0.2)
    ctx.upload_db(w.db_residues, w.db_offsets)
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 11, 1, w.band_center.astype(np.int64),
                      w.band_radius.astype(np.int64))
    reqs = _requests(w)
    # a budget that holds only a few requests at a time: many small batches
    srv = Server(ctx, GapCosts(11, 1), max_batch_pairs=8, hbm_budget_bytes=8 << 20)
    try:
        ids = [(sel, srv.submit(rows, t, bc, br)) for q, sel, rows, t, bc, br in reqs]
        for sel, rid in ids:
            got, lat = srv.wait(rid)
            assert np.array_equal(got, want[sel])
            assert lat >= 0.0
        assert srv.stats()["batches"] >= len(reqs) // 8
        from sabertooth_b200._lib import StError
        big = np.zeros((200_000, 21), dtype=np.int32)
        with pytest.raises(StError, match="budget"):
            srv.submit(big, np.array([0], dtype=np.uint32))
    finally:
        srv.close()


def test_bulk_submit_equals_single_submits(ctx):
    w = W.config3(seed=33, n_queries=20, db_residues=40_000, per_query=30)
    ctx.upload_db(w.db_residues, w.db_offsets)
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), w.pair_q, w.pair_t, 44, 4)
    reqs = _requests(w)
    srv = Server(ctx, GapCosts(44, 4))
    try:
        ro = np.zeros(len(reqs) + 1, dtype=np.uint64)
        ro[1:] = np.cumsum([len(r[2]) for r in reqs])
        to = np.zeros(len(reqs) + 1, dtype=np.uint64)
        to[1:] = np.cumsum([len(r[3]) for r in reqs])
        ids = srv.submit_many(np.concatenate([r[2] for r in reqs]), ro, np.concatenate([r[3] for r in reqs]), to)
        for (q, sel, rows, t, bc, br), rid in zip(reqs, ids):
            assert np.array_equal(srv.wait(rid)[0], want[sel])
    finally:
        srv.close()
