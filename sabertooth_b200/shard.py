"""Target-sharded scoring over several GPUs (one process per GPU).

The database is split into contiguous, residue-balanced target shards, one
per rank (the rule of the reference's `shard::balance`, src/shard.rs:69-97);
queries and their profiles are replicated.  A batch of (profile, global
target) pairs is routed by target: each rank scores the pairs whose target lies
in its shard, against its shard uploaded as its own device database (local
ordinals), and the per-pair scores come back in global pair order through one
exchange step: a gather of (pair index, score) records, placed
deterministically by pair index.  Search hits merge as the reference merges
shard results (`merge_shard_hits`, src/shard.rs:248-259): per query, sorted by
`hit_order` (src/search.rs:191-197) and cut at max_hits.

No peer memory is read: each GPU scores only its own shard, and the exchange
is a torch.distributed collective (NCCL on GPUs, gloo on CPU).
"""
from dataclasses import dataclass

import numpy as np

from .dtypes import PAIR_DTYPE


def balance(lens, n):
    """Residue-balanced contiguous split of `lens` into at most `n` non-empty parts (src/shard.rs:69-97):
    part s ends once the running residue count passes total*(s+1)/n by half a sequence, taking at least
    one sequence and leaving at least one for every remaining part; the last part takes the rest."""
    lens = [int(x) for x in lens]
    total = sum(lens)
    n = max(1, min(int(n), max(len(lens), 1)))
    out, start, acc = [], 0, 0
    for s in range(n):
        if start >= len(lens):
            break
        remaining = n - s
        if remaining == 1:
            out.append((start, len(lens)))
            break
        target = total * (s + 1) // n
        end = start
        max_end = len(lens) - (remaining - 1)
        while end < max_end and (end == start or acc + lens[end] // 2 < target):
            acc += lens[end]
            end += 1
        out.append((start, end))
        start = end
    return out


@dataclass
class ShardMap:
    """Which rank holds which targets: shard r = global ordinals [ranges[r][0], ranges[r][1])."""

    ranges: list

    @staticmethod
    def of(db_offsets, world):
        lens = np.diff(np.asarray(db_offsets, dtype=np.int64))
        return ShardMap(balance(lens, world))

    @property
    def starts(self):
        return np.array([a for a, _ in self.ranges], dtype=np.int64)

    def owner(self, targets):
        """Rank that holds each global target ordinal."""
        t = np.asarray(targets, dtype=np.int64)
        return np.searchsorted(self.starts, t, side="right") - 1

    def shard_db(self, db_residues, db_offsets, rank):
        """(residues, offsets) of shard `rank` as a database of its own (local ordinals from 0)."""
        a, b = self.ranges[rank]
        offs = np.asarray(db_offsets, dtype=np.uint64)
        lo, hi = int(offs[a]), int(offs[b])
        return db_residues[lo:hi], (offs[a:b + 1] - offs[a]).astype(np.uint64)

    def route(self, pairs, rank):
        """(global indices, local pairs) of the pairs whose target is in shard `rank`; the local pairs
        carry shard-local target ordinals and keep their global order."""
        pairs = np.asarray(pairs)
        idx = np.nonzero(self.owner(pairs["target"]) == rank)[0]
        local = pairs[idx].copy()
        local["target"] = (local["target"].astype(np.int64) - self.ranges[rank][0]).astype(np.uint32)
        return idx.astype(np.int64), local


def place_scores(n, parts):
    """Global score array from per-shard (global indices, scores) parts.  The pairs of a batch are
    partitioned by target, so every pair appears in exactly one part; placement is by index and the
    result does not depend on the order of the parts."""
    out = np.zeros(n, dtype=np.int32)
    seen = np.zeros(n, dtype=np.int64)
    for idx, sc in parts:
        idx = np.asarray(idx, dtype=np.int64)
        out[idx] = sc
        seen[idx] += 1
    if n and not np.all(seen == 1):
        raise ValueError("shard results do not cover every pair exactly once")
    return out


def gather_scores(idx, scores, n, group=None, device=None, dst=0):
    """The exchange step: every rank's (global pair index, score) records to rank `dst`, placed in global
    pair order there (None on the other ranks).  Counts are gathered first so every rank sends a padded
    buffer of the largest count (one all_gather of a fixed size, as NCCL requires)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = device if device is not None else torch.device("cpu")
    cnt = torch.tensor([len(idx)], dtype=torch.int64, device=dev)
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, cnt, group=group)
    counts = [int(c.item()) for c in counts]
    width = max(max(counts), 1)
    rec = torch.zeros((width, 2), dtype=torch.int64, device=dev)
    if len(idx):
        rec[:len(idx), 0] = torch.as_tensor(np.asarray(idx, dtype=np.int64), device=dev)
        rec[:len(idx), 1] = torch.as_tensor(np.asarray(scores, dtype=np.int64), device=dev)
    bufs = [torch.zeros((width, 2), dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(bufs, rec, group=group)
    if rank != dst:
        return None
    parts = []
    for r, b in enumerate(bufs):
        b = b[:counts[r]].cpu().numpy()
        parts.append((b[:, 0], b[:, 1].astype(np.int32)))
    return place_scores(n, parts)


HIT_DTYPE = np.dtype([("query", "<u4"), ("target", "<u4"), ("score", "<i4")])


def merge_hits(parts, max_hits=0):
    """merge_shard_hits (src/shard.rs:248-259) for hits with global target ordinals: per query, the
    engine's hit_order (src/search.rs:191-197) — E-value ascending, bit score descending, target ordinal
    ascending — then the first max_hits (0 = all).  With one statistics model for the whole database the
    E-value and the bit score are monotone in the raw score for a given query, so the order is raw score
    descending, then target ascending.  Returns hits grouped by query in query order."""
    allh = np.concatenate([np.asarray(p, dtype=HIT_DTYPE) for p in parts]) if parts else np.zeros(0, HIT_DTYPE)
    order = np.lexsort((allh["target"], -allh["score"].astype(np.int64), allh["query"]))
    allh = allh[order]
    if max_hits > 0 and allh.size:
        q = allh["query"].astype(np.int64)
        first = np.r_[0, np.nonzero(np.diff(q))[0] + 1]
        rank_in_q = np.arange(allh.size) - np.repeat(first, np.diff(np.r_[first, allh.size]))
        allh = allh[rank_in_q < max_hits]
    return allh


class ShardedScorer:
    """One rank's part of target-sharded batched scoring.

    `ctx` is this rank's Context (its GPU); the rank uploads only its shard of the database and all the
    profiles.  `score` routes a batch of global pairs, scores the rank's share with one batched call, and
    gathers the scores to rank 0 in global pair order."""

    def __init__(self, ctx, db_residues, db_offsets, rows_list, rank, world, group=None, device=None):
        self.ctx, self.rank, self.world, self.group, self.device = ctx, rank, world, group, device
        self.map = ShardMap.of(db_offsets, world)
        res, offs = self.map.shard_db(db_residues, db_offsets, rank)
        ctx.upload_db(res, offs)
        self.ids = ctx.create_profiles(rows_list)

    def local_pairs(self, pair_q, pair_t, band_center=None, band_radius=None):
        """(global indices, device-ready local pairs) of this rank's share of a batch of global pairs."""
        pairs = np.zeros(len(pair_q), dtype=PAIR_DTYPE)
        pairs["profile"] = self.ids[np.asarray(pair_q, dtype=np.int64)]
        pairs["target"] = pair_t
        pairs["band_center"] = 0 if band_center is None else band_center
        pairs["band_radius"] = -1 if band_radius is None else band_radius
        return self.map.route(pairs, self.rank)

    def score(self, pair_q, pair_t, gaps, band_center=None, band_radius=None):
        idx, local = self.local_pairs(pair_q, pair_t, band_center, band_radius)
        sc = self.ctx.sw_score_pairs(local, gaps) if len(local) else np.zeros(0, np.int32)
        return gather_scores(idx, sc, len(pair_q), self.group, self.device)

    def close(self):
        self.ctx.free_profiles(self.ids)
