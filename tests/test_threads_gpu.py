"""Calls from several host threads at once on one context.

The reference calls its scoring functions from rayon workers concurrently
(src/search.rs:553-556, src/prefilter.rs:1570), so the C ABI must give every
thread the result it would get alone. Here six threads each build their own
profiles and run, interleaved with the others: a batch large enough for the
device planner, a small host-planned batch, an asynchronous batch, plain
per-call scores and ungapped hits, then free their profiles. Every result must
equal the same call made from one thread (whose parity with the oracle the
other tests establish), and the context must stay usable afterwards.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from sabertooth_b200 import GapCosts
from synth import workloads as W
from sabertooth_b200._lib import HIT_DTYPE, PAIR_DTYPE, check, lib

pytestmark = pytest.mark.gpu

GAPS = GapCosts(44, 4)
N_THREADS = 6


def _pairs(ids, q, t):
    p = np.zeros(len(q), dtype=PAIR_DTYPE)
    p["profile"] = ids[q]
    p["target"] = t
    p["band_radius"] = -1
    return p


def _hits(ids, q, t, lens, rng):
    h = np.zeros(len(q), dtype=HIT_DTYPE)
    h["query"] = ids[q]
    h["target"] = t
    h["diag"] = rng.integers(-60, np.maximum(lens[t], 1)).astype(np.int32)
    return h


def _plain(ctx, pid, target):
    """One st_sw_score call (the per-call drop-in) on a host target."""
    t = np.ascontiguousarray(target, dtype=np.uint8)
    s, k = C.c_int32(), C.c_uint32()
    check(lib.st_sw_score(ctx.handle, pid, t.ctypes.data, t.size, GAPS.open, GAPS.extend, C.byref(s), C.byref(k)))
    return s.value


def _work(ctx, w, lens, seed):
    """Everything one thread does; returns its results in a fixed order."""
    rng = np.random.default_rng(seed)
    ids = ctx.create_profiles(w.rows)
    try:
        big = _pairs(ids, w.pair_q, w.pair_t)  # >= 16 K pairs: the device planner
        small = big[: 300].copy()              # the host planner
        r_big = ctx.sw_score_pairs(big, GAPS)
        batch = ctx.sw_score_pairs_async(small, GAPS)
        targets = w.targets()
        r_plain = [_plain(ctx, int(ids[w.pair_q[i]]), targets[int(w.pair_t[i])]) for i in range(8)]
        hits = _hits(ids, w.pair_q[:2000], w.pair_t[:2000], lens, rng)
        r_ung = ctx.ungapped_hits(hits, with_pairs=False)
        r_small = batch.wait()
        return r_big, r_small, np.array(r_plain), r_ung
    finally:
        ctx.free_profiles(ids)


def test_concurrent_calls_equal_single_thread_results(ctx):
    w = W.config3(seed=41, n_queries=40, db_residues=80_000, per_query=420)
    assert w.n_pairs >= 16_384
    ctx.upload_db(w.db_residues, w.db_offsets)
    lens = np.diff(w.db_offsets.astype(np.int64))
    want = [_work(ctx, w, lens, seed=100 + k) for k in range(N_THREADS)]

    got = [None] * N_THREADS
    errors = []
    start = threading.Barrier(N_THREADS)

    def run(k):
        try:
            start.wait()
            got[k] = _work(ctx, w, lens, seed=100 + k)
        except Exception as e:  # reported below
            errors.append(repr(e))

    th = [threading.Thread(target=run, args=(k,)) for k in range(N_THREADS)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errors, errors
    for k in range(N_THREADS):
        for a, b in zip(got[k], want[k]):
            assert np.array_equal(a, b), k
    # the context still works, and every profile was freed
    again = _work(ctx, w, lens, seed=100)
    for a, b in zip(again, want[0]):
        assert np.array_equal(a, b)


def test_per_call_scores_from_many_threads_at_once(ctx):
    """st_sw_score (the per-call drop-in of sw_score_with) from 24 threads at once, more threads than the
    context has call slots would need to be busy: every call returns the oracle's score, with profiles
    created by one thread while the others score (the profile tables grow under running calls)."""
    from oracle import oracle as O
    w = W.config3(seed=43, n_queries=24, db_residues=60_000, per_query=40)
    targets = w.targets()
    ids = ctx.create_profiles(w.rows)
    want = O.sw_pairs(O.Arena(w.rows, targets), w.pair_q, w.pair_t, GAPS.open, GAPS.extend)
    got = np.full(w.n_pairs, -1, dtype=np.int64)
    errors = []
    n_thr = 24
    start = threading.Barrier(n_thr + 1)

    def run(k):
        try:
            start.wait()
            for i in range(k, w.n_pairs, n_thr):
                got[i] = _plain(ctx, int(ids[w.pair_q[i]]), targets[int(w.pair_t[i])])
        except Exception as e:  # reported below
            errors.append(repr(e))

    def churn():
        # profile creation and frees while calls run: the device profile tables are rebuilt and grown
        start.wait()
        for _ in range(20):
            extra = ctx.create_profiles(w.rows[:8] * 8)
            ctx.free_profiles(extra)

    th = [threading.Thread(target=run, args=(k,)) for k in range(n_thr)] + [threading.Thread(target=churn)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    ctx.free_profiles(ids)
    assert not errors, errors
    assert np.array_equal(got, want.astype(np.int64))


def test_per_call_score_of_a_profile_created_just_before(ctx):
    """A per-call score right after the profile it uses is created, round after round on one thread: the
    call's stream must start after that profile's layouts are built (a call skips that wait only when no
    profile changed since its call slot's last call).  Each round creates fresh profiles, at once scores one
    pair of them through st_sw_score, and frees them; every score equals the oracle's.  Rows outside int8
    and gap costs outside the 16-bit range (both on the 32-bit kernel) alternate with the packed path."""
    from oracle import oracle as O
    rng = np.random.default_rng(77)
    w = W.config3(seed=44, n_queries=6, db_residues=30_000, per_query=10)
    targets = w.targets()
    gap_sets = [(44, 4), (11, 1), (20000, 1)]
    for rnd in range(24):
        rows = [r if rnd % 2 == 0 else (r * 3).astype(np.int32) for r in w.rows]
        op, ex = gap_sets[rnd % 3]
        ids = ctx.create_profiles(rows)
        k = int(rng.integers(0, w.n_pairs))
        q, t = int(w.pair_q[k]), int(w.pair_t[k])
        tt = np.ascontiguousarray(targets[t], dtype=np.uint8)
        s_, k_ = C.c_int32(), C.c_uint32()
        check(lib.st_sw_score(ctx.handle, int(ids[q]), tt.ctypes.data, tt.size, op, ex, C.byref(s_), C.byref(k_)))
        want = O.gotoh_score(rows[q], targets[t], op, ex)
        ctx.free_profiles(ids)
        assert s_.value == want, (rnd, q, t, op, ex, s_.value, want)
