"""Seed hits and a direct restatement of the prefilter's evidence stage, for the
tests of the evidence / chain / gate path.

brute_seed_hits: every (query position, target position) whose k-mer pair
scores at least kmer_score, plus exact k-mer matches (exact_seeds).  This is
the hit set of the reference's similar-k-mer enumeration (src/prefilter.rs:
475-700) whenever no query window has more than max_kmers_per_pos (512)
similar k-mers, which similar_kmer_count checks.

py_prefilter: a pure-Python restatement of evaluate_block_kadane +
score_and_gate + ranking (src/prefilter.rs:1194-1225, 1412-1660, 1074-1083),
kept deliberately literal (small inputs only); it checks the C oracle.
"""
import numpy as np

STD = 20  # standard residues; k-mers with X or other codes are not seeded


def similar_kmer_count(score_matrix, q, k, kmer_score):
    """Largest number of k-mers over the 20 standard residues scoring >= kmer_score
    against any query window (the generator keeps at most max_kmers_per_pos)."""
    sm = np.asarray(score_matrix)[:STD, :STD].astype(np.int64)
    worst = 0
    for p in range(len(q) - k + 1):
        acc = np.zeros(1, dtype=np.int64)
        for l in range(k):
            acc = np.add.outer(acc, sm[q[p + l]]).ravel()
        worst = max(worst, int((acc >= kmer_score).sum()))
    return worst


def brute_seed_hits(score_matrix, q, targets, k, kmer_score, exact=True, query_id=0):
    """All seed hits of q against targets as (query, target, diag, qpos) tuples."""
    sm = np.asarray(score_matrix).astype(np.int64)
    q = np.asarray(q, dtype=np.int64)
    out = []
    m = len(q)
    if m < k:
        return out
    for ti, t in enumerate(targets):
        t = np.asarray(t, dtype=np.int64)
        n = len(t)
        if n < k:
            continue
        S = sm[q[:, None], t[None, :]]
        W = np.zeros((m - k + 1, n - k + 1), dtype=np.int64)
        E = np.ones_like(W, dtype=bool)
        ok = np.ones_like(W, dtype=bool)
        for l in range(k):
            W += S[l:l + m - k + 1, l:l + n - k + 1]
            E &= q[l:l + m - k + 1, None] == t[None, l:l + n - k + 1]
            ok &= (q[l:l + m - k + 1, None] < STD) & (t[None, l:l + n - k + 1] < STD)
        hit = ok & ((W >= kmer_score) | (E if exact else False))
        for qp, tp in zip(*np.nonzero(hit)):
            out.append((query_id, ti, int(tp) - int(qp), int(qp)))
    return out


def _diag_range(m, n, d):
    lo = max(-d, 0)
    hi = min(m, n - d)
    return (lo, hi) if hi > lo else (0, 0)


def _kadane_segment(rows, t, d, lo, hi):
    best, bs, be = 0, 0, 0
    cur, cs = 0, lo
    for q in range(lo, hi):
        tr = int(t[q + d])
        s = int(rows[q][tr]) if tr < 21 else 0
        if cur <= 0:
            cur, cs = s, q
        else:
            cur += s
        if cur > best:
            best, bs, be = cur, cs, q
    return best, bs, be


def _gap(open_, ext, length):
    return 0 if length == 0 else open_ + (length - 1) * ext


def py_prefilter(rows, targets, hits, p, query_id=0):
    """One query's hits [(target, diag, qpos)] -> ranked candidate tuples
    (query, target, hits, diag_score, best_diag, t_lo, t_hi) and stats."""
    st = dict(targets_hit=0, targets_evaluated=0, diagonals_scored=0, chains_used=0, candidates=0,
              candidates_capped=0)
    m = len(rows)
    by_t = {}
    for t, d, qp in hits:
        by_t.setdefault(int(t), []).append((int(d), int(qp)))
    out = []
    for tid in sorted(by_t):
        group = sorted(by_t[tid], key=lambda x: x[0])
        st["targets_hit"] += 1
        if len(group) < p["min_hits"]:
            continue
        top = []  # [diag, count, qmin, qmax], top_diagonals
        i = 0
        while i < len(group):
            j = i
            d = group[i][0]
            qs = []
            while j < len(group) and group[j][0] == d:
                qs.append(group[j][1])
                j += 1
            run = [d, j - i, min(qs), max(qs)]
            i = j
            pos = next((x for x, tt in enumerate(top) if run[1] > tt[1]), len(top))
            if pos < p["max_diagonals"]:
                top.insert(pos, run)
                if len(top) > p["max_diagonals"]:
                    top.pop()
        if top[0][1] < p["diag_hits"]:
            continue
        st["targets_evaluated"] += 1
        n = len(targets[tid])
        segs = []
        for d, _, qmin, qmax in top[:16]:
            lo, hi = _diag_range(m, n, d)
            if p["diag_window"] > 0:
                lo = max(lo, max(qmin - p["diag_window"], 0))
                hi = min(hi, qmax + p["span"] + p["diag_window"])
            hi = max(hi, lo)
            s, a, b = _kadane_segment(rows, targets[tid], d, lo, hi)
            segs.append((s, a, b, d))
        st["diagonals_scored"] += len(segs)
        ns = len(segs)
        if ns == 1 and segs[0][0] < p["min_diag_score"]:
            continue
        best, bi = 0, 0
        for k, sg in enumerate(segs):
            if sg[0] > best:
                best, bi = sg[0], k
        chain = (None, 0, 0)
        for x in range(ns):
            for y in range(ns):
                if x == y:
                    continue
                sx, _, qex, dx = segs[x]
                sy, qsy, _, dy = segs[y]
                if sx <= 0 or sy <= 0 or dx == dy:
                    continue
                c = sx + sy - _gap(p["gap_open"], p["gap_ext"], abs(dy - dx))
                if c <= best or (chain[0] is not None and c <= chain[0]):
                    continue
                if qex < qsy and qex + dx < qsy + dy:
                    chain = (c, x, y)
        if chain[0] is not None and chain[0] > best:
            st["chains_used"] += 1
            score, used = chain[0], (chain[1], chain[2])
        else:
            score, used = best, (bi, bi)
        if score < p["min_diag_score"]:
            continue
        if p["regions"]:
            lo_r = min(max(segs[u][1] + segs[u][3], 0) for u in used)
            hi_r = max(max(segs[u][2] + segs[u][3], 0) for u in used)
        else:
            lo_r, hi_r = 0, 0xFFFFFFFF
        out.append((query_id, tid, len(group), score, segs[bi][3], lo_r, hi_r))
    out.sort(key=lambda c: (-c[3], c[1]))
    if p["max_candidates"] > 0 and len(out) > p["max_candidates"]:
        st["candidates_capped"] = len(out) - p["max_candidates"]
        out = out[:p["max_candidates"]]
    st["candidates"] = len(out)
    return out, st


def default_params(**kw):
    """The reference's sequence_default evidence fields (src/prefilter.rs:309-331), span 6, gaps 11/1."""
    p = dict(min_hits=1, diag_hits=1, max_diagonals=4, diag_window=48, span=6, min_diag_score=42, gap_open=11,
             gap_ext=1, max_candidates=0, regions=0)
    p.update(kw)
    return p
