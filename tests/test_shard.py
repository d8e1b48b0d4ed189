"""Target sharding (sabertooth_b200.shard) on CPU.

* balance: the reference's own test (src/shard.rs:404-423) on its lengths and part counts.
* routing + placement: for 1-5 shards, every pair is scored by exactly one shard against that shard's
  own database (local ordinals), and the placed scores equal the unsharded scores.
* two ranks over gloo (127.0.0.1): ShardedScorer end to end (each rank uploads only its shard, scores
  its share, one gather to rank 0), with a CPU stand-in for the GPU context whose scores come from the
  oracle; rank 0's merged scores equal the single-rank oracle scores bit for bit.
* merge_hits: per-shard hit lists merged by hit_order (src/search.rs:191-197) equal the unsharded list.
"""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from sabertooth_b200.dtypes import PAIR_DTYPE
from sabertooth_b200.shard import HIT_DTYPE, ShardMap, balance, merge_hits, place_scores

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_balance_matches_the_reference_test():
    lens = [50 + (i * 37) % 400 for i in range(1000)]
    for n in (1, 2, 3, 7, 16, 999, 1000, 5000):
        r = balance(lens, n)
        assert len(r) == min(n, len(lens))
        assert r[0][0] == 0 and r[-1][1] == len(lens)
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert all(b > a for a, b in r)
        if n <= 16:
            ideal = sum(lens) // n
            for a, b in r:
                assert abs(sum(lens[a:b]) - ideal) <= 450


def test_balance_edge_cases():
    assert balance([], 4) == []
    assert balance([5], 3) == [(0, 1)]
    # part 0 stops before a sequence whose first half would pass its residue target (1003 * 1 // 2)
    assert balance([1, 1, 1000, 1], 2) == [(0, 2), (2, 4)]
    assert balance([10, 10, 10, 10], 4) == [(0, 1), (1, 2), (2, 3), (3, 4)]


class OracleContext:
    """A CPU stand-in for Context with the calls ShardedScorer makes; scores come from the oracle."""

    def __init__(self):
        self.rows = []

    def upload_db(self, residues, offsets):
        o = np.asarray(offsets, dtype=np.int64)
        self.targets = [np.asarray(residues[o[i]:o[i + 1]], dtype=np.uint8) for i in range(len(o) - 1)]

    def create_profiles(self, rows_list):
        base = len(self.rows)
        self.rows += list(rows_list)
        return np.arange(base, base + len(rows_list), dtype=np.uint32)

    def free_profiles(self, ids):
        pass

    def sw_score_pairs(self, pairs, gaps):
        from oracle import oracle as O
        ar = O.Arena(self.rows, self.targets)
        br = pairs["band_radius"]
        return O.sw_pairs(ar, pairs["profile"], pairs["target"], gaps.open, gaps.extend,
                          pairs["band_center"] if (br >= 0).any() else None, br if (br >= 0).any() else None)


def _workload(seed=3):
    from synth import workloads as W
    w = W.config1(seed=seed, n_queries=6, n_targets=120)
    rng = np.random.default_rng(seed)
    sel = rng.choice(w.n_pairs, 400, replace=False)
    return w, w.pair_q[sel], w.pair_t[sel]


def test_routing_and_placement_equal_the_unsharded_scores():
    from oracle import oracle as O
    w, pq, pt = _workload()
    ar = O.Arena(w.rows, w.targets())
    want = O.sw_pairs(ar, pq, pt, 11, 1)
    pairs = np.zeros(len(pq), dtype=PAIR_DTYPE)
    pairs["profile"] = pq
    pairs["target"] = pt
    pairs["band_radius"] = -1
    for world in range(1, 6):
        sm = ShardMap.of(w.db_offsets, world)
        parts, covered = [], 0
        for r in range(world):
            res, offs = sm.shard_db(w.db_residues, w.db_offsets, r)
            ts = [res[int(offs[i]):int(offs[i + 1])] for i in range(len(offs) - 1)]
            idx, local = sm.route(pairs, r)
            assert np.all(np.diff(idx) > 0)  # global order kept
            assert local["target"].max(initial=0) < max(len(ts), 1)
            parts.append((idx, O.sw_pairs(O.Arena(w.rows, ts), local["profile"], local["target"], 11, 1)))
            covered += len(idx)
        assert covered == len(pq)
        assert np.array_equal(place_scores(len(pq), parts[::-1]), want), world


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      GLOO_SOCKET_IFNAME="lo")
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    from sabertooth_b200.api import GapCosts
    from sabertooth_b200.shard import ShardedScorer
    from tests.test_shard import OracleContext, _workload
    w, pq, pt = _workload()
    ctx = OracleContext()
    sc = ShardedScorer(ctx, w.db_residues, w.db_offsets, w.rows, rank, world)
    got = sc.score(pq, pt, GapCosts(11, 1))
    out[rank] = (None if got is None else got.tolist(), len(ctx.targets), len(sc.local_pairs(pq, pt)[0]))
    sc.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_sharded_scores_equal_the_single_rank_scores():
    from oracle import oracle as O
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    w, pq, pt = _workload()
    want = O.sw_pairs(O.Arena(w.rows, w.targets()), pq, pt, 11, 1)
    (g0, n0, k0), (g1, n1, k1) = out[0], out[1]
    assert g1 is None and g0 is not None
    assert np.array_equal(np.array(g0, dtype=np.int32), want)
    assert n0 + n1 == len(w.db_offsets) - 1 and n0 > 0 and n1 > 0  # each rank holds only its shard
    assert k0 + k1 == len(pq) and k0 > 0 and k1 > 0


def test_merged_shard_hits_equal_the_unsharded_hits():
    rng = np.random.default_rng(9)
    n = 3000
    hits = np.zeros(n, dtype=HIT_DTYPE)
    hits["query"] = rng.integers(0, 40, n)
    hits["target"] = rng.permutation(100_000)[:n]
    hits["score"] = rng.integers(0, 60, n)  # many ties: the target ordinal breaks them
    for max_hits in (0, 1, 7):
        want = merge_hits([hits], max_hits)
        sm = ShardMap([(0, 30_000), (30_000, 71_000), (71_000, 100_000)])
        own = sm.owner(hits["target"])
        parts = [hits[own == r] for r in (2, 0, 1)]
        assert np.array_equal(merge_hits(parts, max_hits), want)
        q = want["query"].astype(np.int64)
        assert np.all(np.diff(q) >= 0)
        same = np.diff(q) == 0
        s = want["score"].astype(np.int64)
        assert np.all((np.diff(s) < 0) | ((np.diff(s) == 0) & (np.diff(want["target"].astype(np.int64)) > 0))
                      | ~same)
        if max_hits:
            assert np.bincount(q).max() <= max_hits
