"""ctypes wrapper of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker / CPU baseline; never by the sabertooth_b200 package.  Each
function follows the reference file:line cited in oracle.h.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
NPROF = 21


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    srcs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".c", ".h"))]
    if not os.path.exists(LIB) or any(os.path.getmtime(f) > os.path.getmtime(LIB) for f in srcs):
        build()
    lib = C.CDLL(LIB)
    P, u32, i32, u64, i64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64, C.c_int64
    lib.or_diag_range.argtypes = [u64, u64, i64, P, P]
    lib.or_kadane_score.restype = i32
    lib.or_kadane_score.argtypes = [P, P, i64, u64, u64]
    lib.or_kadane_segment.restype = i32
    lib.or_kadane_segment.argtypes = [P, P, i64, u64, u64, P, P]
    lib.or_gotoh_score_end.restype = C.c_int
    lib.or_gotoh_score_end.argtypes = [P, u32, P, u32, i32, i32, P, P, P]
    lib.or_gotoh_score.restype = i32
    lib.or_gotoh_score.argtypes = [P, u32, P, u32, i32, i32]
    lib.or_reference_score.restype = i32
    lib.or_reference_score.argtypes = [P, u32, P, u32, i32, i32]
    lib.or_band_score.restype = i32
    lib.or_band_score.argtypes = [P, u32, P, u32, i32, i32, i64, i64]
    lib.or_sw_pairs.argtypes = [P, P, P, P, P, P, P, P, P, u64, i32, i32, P, C.c_int]
    lib.or_ungapped_hits.argtypes = [P, P, P, P, P, P, P, P, u64, P, C.c_int]
    lib.or_ungapped_hits_avx2.argtypes = [P, P, P, P, P, P, P, P, u64, P, C.c_int]
    lib.or_striped_queries.argtypes = [P, P, P, u32, P, P, P, P, i32, i32, P, P, C.c_int]
    lib.or_prefilter_queries.argtypes = [P, P, P, P, u32, P, P, P, P, P, P, P, C.c_int, P, P, P, C.c_int]
    lib.or_background_cum.argtypes = [P, P]
    lib.or_stream_seed.restype = u64
    lib.or_stream_seed.argtypes = [u64, u64, u64]
    lib.or_calibration_target.argtypes = [P, u32, u64, u64, P, P, P]
    lib.or_fit_gumbel_ml.restype = C.c_int
    lib.or_fit_gumbel_ml.argtypes = [P, u64, P, P]
    lib.or_calibrate_profile.restype = C.c_int
    lib.or_calibrate_profile.argtypes = [P, u32, P, u32, u32, u64, P, i32, i32, P, P, P, P, C.c_int]
    lib.or_top_kmers.restype = C.c_int
    lib.or_top_kmers.argtypes = [P, C.c_int, i32, u32, P, P, P]
    lib.or_top_kmers_dfs.restype = C.c_int
    lib.or_top_kmers_dfs.argtypes = [P, C.c_int, i32, u32, P, P, P]
    lib.or_index_count.restype = u64
    lib.or_index_count.argtypes = [P, P, u32, P, u32, u32]
    lib.or_index_build.argtypes = [P, P, u32, P, u32, u32, P]
    lib.or_index_direct_build.restype = u64
    lib.or_index_direct_build.argtypes = [P, P, u32, P, u32, u32, P, P, P, C.c_int]
    lib.or_prefilter_search.argtypes = [P, P, P, P, u32, P, P, P, u32, u32, P, P, P, P, P, P, u64, P, P, C.c_int]
    lib.or_seed_hits.restype = u64
    lib.or_seed_hits.argtypes = [P, P, u32, P, u32, u32, P, P, u64, u32, P, P, P, u64, P]
    lib.or_comp_bias.argtypes = [P, u32, P, P, C.c_int, P]
    lib.or_low_complexity_mask.restype = u32
    lib.or_low_complexity_mask.argtypes = [P, u32, u32, C.c_double, C.c_double, P]
    return lib


lib = _load()


def _p(a):
    return None if a is None else a.ctypes.data


def _rows(rows):
    return np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, NPROF)


def _t(t):
    return np.ascontiguousarray(t, dtype=np.uint8)


def diag_range(m, n, d):
    lo, hi = C.c_uint64(), C.c_uint64()
    lib.or_diag_range(m, n, d, C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def kadane_score(rows, t, d, lo, hi):
    r, tt = _rows(rows), _t(t)
    return lib.or_kadane_score(_p(r), _p(tt), d, lo, hi)


def kadane_segment(rows, t, d, lo, hi):
    r, tt = _rows(rows), _t(t)
    a, b = C.c_uint64(), C.c_uint64()
    s = lib.or_kadane_segment(_p(r), _p(tt), d, lo, hi, C.byref(a), C.byref(b))
    return s, a.value, b.value


def gotoh_score(rows, t, open_, ext):
    r, tt = _rows(rows), _t(t)
    return lib.or_gotoh_score(_p(r), r.shape[0], _p(tt) if tt.size else None, tt.size, open_, ext)


def gotoh_score_end(rows, t, open_, ext):
    r, tt = _rows(rows), _t(t)
    s, qi, tj = C.c_int32(), C.c_uint32(), C.c_uint32()
    ok = lib.or_gotoh_score_end(_p(r), r.shape[0], _p(tt) if tt.size else None, tt.size, open_, ext,
                                C.byref(s), C.byref(qi), C.byref(tj))
    return (s.value, qi.value, tj.value) if ok else None


def reference_score(rows, t, open_, ext):
    r, tt = _rows(rows), _t(t)
    return lib.or_reference_score(_p(r), r.shape[0], _p(tt) if tt.size else None, tt.size, open_, ext)


def band_score(rows, t, open_, ext, center, radius):
    r, tt = _rows(rows), _t(t)
    return lib.or_band_score(_p(r), r.shape[0], _p(tt) if tt.size else None, tt.size, open_, ext, center, radius)


def comp_bias(q, score, p_back, penalize_only=False):
    """local_bias_correction_mode (src/compbias.rs:38-70): per-position integer corrections."""
    qq = _t(q)
    sc = np.ascontiguousarray(score, dtype=np.int32).reshape(NPROF, NPROF)
    pb = np.ascontiguousarray(p_back[:20], dtype=np.float64)
    out = np.zeros(max(qq.size, 1), dtype=np.int32)
    lib.or_comp_bias(_p(qq), qq.size, _p(sc), _p(pb), int(penalize_only), _p(out))
    return out[:qq.size]


def low_complexity_mask(seq, window, locut, hicut):
    """low_complexity_mask (src/mask.rs:62-128): a bool per position."""
    s = _t(seq)
    out = np.zeros(max(s.size, 1), dtype=np.uint8)
    lib.or_low_complexity_mask(_p(s), s.size, window, locut, hicut, _p(out))
    return out[:s.size].astype(bool)


def search_rows(q, score, p_back, comp_bias_corr=True, mask_scoring=(15, 2.3, 2.3)):
    """A sequence query's alignment rows as the reference's search builds them (src/search.rs:432-455):
    matrix rows, plus the composition-bias correction of each column, and the X row for positions that
    the scoring mask covers."""
    qq = _t(q)
    sc = np.ascontiguousarray(score, dtype=np.int32).reshape(NPROF, NPROF)
    rows = sc[np.minimum(qq, NPROF - 1)].astype(np.int32)
    if comp_bias_corr:
        rows = rows + comp_bias(qq, sc, p_back)[:, None]
    if mask_scoring is not None:
        mk = low_complexity_mask(qq, *mask_scoring)
        rows[mk] = sc[NPROF - 1]
    return np.ascontiguousarray(rows, dtype=np.int32)


class Arena:
    """Concatenated query rows and targets, the layout of the batched oracle calls."""

    def __init__(self, rows_list, targets):
        self.qlen = np.array([len(r) for r in rows_list], dtype=np.uint32)
        self.row_off = np.zeros(len(rows_list), dtype=np.uint64)
        if len(rows_list) > 1:
            self.row_off[1:] = np.cumsum(self.qlen.astype(np.uint64))[:-1]
        parts = [_rows(r) for r in rows_list if len(r)]
        self.rows = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros((1, NPROF), np.int32))
        self.tgt_off = np.zeros(len(targets) + 1, dtype=np.uint64)
        self.tgt_off[1:] = np.cumsum([len(t) for t in targets])
        tp = [_t(t) for t in targets if len(t)]
        self.tgt = np.ascontiguousarray(np.concatenate(tp) if tp else np.zeros(1, np.uint8))


def sw_pairs(arena: Arena, pq, pt, open_, ext, center=None, radius=None, threads=0):
    pq = np.ascontiguousarray(pq, dtype=np.uint32)
    pt = np.ascontiguousarray(pt, dtype=np.uint32)
    n = len(pq)
    c = None if center is None else np.ascontiguousarray(center, dtype=np.int64)
    r = None if radius is None else np.ascontiguousarray(radius, dtype=np.int64)
    out = np.zeros(n, dtype=np.int32)
    lib.or_sw_pairs(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), _p(arena.tgt), _p(arena.tgt_off), _p(pq),
                    _p(pt), _p(c), _p(r), n, open_, ext, _p(out), threads or os.cpu_count() or 1)
    return out


def ungapped_hits(arena: Arena, hq, ht, hd, threads=0):
    hq = np.ascontiguousarray(hq, dtype=np.uint32)
    ht = np.ascontiguousarray(ht, dtype=np.uint32)
    hd = np.ascontiguousarray(hd, dtype=np.int32)
    n = len(hq)
    out = np.zeros(n, dtype=np.int32)
    lib.or_ungapped_hits(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), _p(arena.tgt), _p(arena.tgt_off),
                         _p(hq), _p(ht), _p(hd), n, _p(out), threads or os.cpu_count() or 1)
    return out


def ungapped_hits_avx2(arena: Arena, hq, ht, hd, threads=0):
    """The reference's AVX2 batched Kadane over hits (grouped by query), results in hit order."""
    hq = np.ascontiguousarray(hq, dtype=np.uint32)
    ht = np.ascontiguousarray(ht, dtype=np.uint32)
    hd = np.ascontiguousarray(hd, dtype=np.int32)
    out = np.zeros(len(hq), dtype=np.int32)
    lib.or_ungapped_hits_avx2(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), _p(arena.tgt), _p(arena.tgt_off),
                              _p(hq), _p(ht), _p(hd), len(hq), _p(out), threads or os.cpu_count() or 1)
    return out


def striped_pairs(arena: Arena, pq, pt, open_, ext, threads=0, with_kinds=False):
    """The reference's default AVX2 CPU path over pairs (grouped by query internally), results in pair order."""
    pq = np.asarray(pq, dtype=np.uint32)
    pt = np.asarray(pt, dtype=np.uint32)
    order = np.argsort(pq, kind="stable")
    nq = len(arena.qlen)
    counts = np.bincount(pq, minlength=nq).astype(np.uint64)
    qstart = np.zeros(nq + 1, dtype=np.uint64)
    qstart[1:] = np.cumsum(counts)
    tlist = np.ascontiguousarray(pt[order])
    out = np.zeros(len(pq), dtype=np.int32)
    used = np.zeros(len(pq), dtype=np.uint8)
    lib.or_striped_queries(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), nq, _p(arena.tgt), _p(arena.tgt_off),
                           _p(qstart), _p(tlist), open_, ext, _p(out), _p(used), threads or os.cpu_count() or 1)
    res = np.zeros_like(out)
    res[order] = out
    kinds = np.zeros_like(used)
    kinds[order] = used
    return (res, kinds) if with_kinds else res


# ---- prefilter evidence, chain and gate (gate.c) -------------------------------
CANDIDATE_DTYPE = np.dtype([("query", "<u4"), ("target", "<u4"), ("hits", "<u4"), ("diag_score", "<i4"),
                            ("best_diag", "<i8"), ("t_lo", "<u4"), ("t_hi", "<u4")])
STATS_FIELDS = ("targets_hit", "targets_evaluated", "diagonals_scored", "chains_used", "candidates",
                "candidates_capped")
PARAM_FIELDS = ("min_hits", "diag_hits", "max_diagonals", "diag_window", "span", "min_diag_score", "gap_open",
                "gap_ext", "max_candidates", "regions")
_PARAM_DTYPE = np.dtype([(f, "<i4" if f in ("min_diag_score", "gap_open", "gap_ext") else "<u4")
                         for f in PARAM_FIELDS])


def prefilter_queries(arena: Arena, hq, ht, hd, hqpos, params: dict, simd=True, threads=0):
    """The reference's segment evidence + chain + gate + ranking per query
    (src/prefilter.rs:1412-1660, 1074-1083).  params: the PARAM_FIELDS keys.
    Returns (candidates ordered by query id, then rank; summed stats dict)."""
    hq = np.asarray(hq, dtype=np.uint32)
    order = np.argsort(hq, kind="stable")
    ht = np.ascontiguousarray(np.asarray(ht, dtype=np.uint32)[order])
    hd = np.ascontiguousarray(np.asarray(hd, dtype=np.int32)[order])
    hqpos = np.ascontiguousarray(np.asarray(hqpos, dtype=np.uint32)[order])
    qs = hq[order]
    qids, first = np.unique(qs, return_index=True)
    qids = np.ascontiguousarray(qids, dtype=np.uint32)
    hstart = np.zeros(len(qids) + 1, dtype=np.uint64)
    hstart[:-1] = first
    hstart[-1] = len(qs)
    prm = np.zeros(1, dtype=_PARAM_DTYPE)
    for f in PARAM_FIELDS:
        prm[f] = params[f]
    out = np.zeros(max(len(qs), 1), dtype=CANDIDATE_DTYPE)
    n_out = np.zeros(max(len(qids), 1), dtype=np.uint64)
    stats = np.zeros((max(len(qids), 1), len(STATS_FIELDS)), dtype=np.uint64)
    if len(qids):
        lib.or_prefilter_queries(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), _p(qids), len(qids),
                                 _p(arena.tgt), _p(arena.tgt_off), _p(hstart), _p(ht), _p(hd), _p(hqpos), _p(prm),
                                 1 if simd else 0, _p(out), _p(n_out), _p(stats), threads or os.cpu_count() or 1)
    parts = [out[int(hstart[i]):int(hstart[i]) + int(n_out[i])] for i in range(len(qids))]
    cands = np.concatenate(parts) if parts else np.zeros(0, dtype=CANDIDATE_DTYPE)
    tot = stats[:len(qids)].sum(axis=0) if len(qids) else np.zeros(len(STATS_FIELDS), np.uint64)
    return cands, {f: int(v) for f, v in zip(STATS_FIELDS, tot)}


# ---- per-profile calibration (calib.c) ------------------------------------------
def background_cum(p_back20):
    p = np.ascontiguousarray(p_back20, dtype=np.float64)
    out = np.zeros(20, dtype=np.float64)
    lib.or_background_cum(_p(p), _p(out))
    return out


def calibration_target(lengths, seed, i, p_back20):
    """Background target i of the calibration stream (src/evalue.rs:728-731)."""
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    cum = background_cum(p_back20)
    out = np.zeros(int(lengths.max()) + 1, dtype=np.uint8)
    n = C.c_uint32()
    lib.or_calibration_target(_p(lengths), len(lengths), seed, i, _p(cum), _p(out), C.byref(n))
    return out[:n.value].copy()


def fit_gumbel_ml(xs):
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    lam, mu = C.c_double(), C.c_double()
    ok = lib.or_fit_gumbel_ml(_p(xs), len(xs), C.byref(lam), C.byref(mu))
    return (lam.value, mu.value) if ok else None


def calibrate_profile(rows, lengths, samples, seed, p_back20, open_, ext, threads=0):
    """(lambda, k, mu, scores) of calibrate_profile (src/evalue.rs:714-748); None parameters where it returns None."""
    r = _rows(rows)
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    p = np.ascontiguousarray(p_back20, dtype=np.float64)
    scores = np.zeros(max(samples, 1), dtype=np.int32)
    lam, k, mu = C.c_double(), C.c_double(), C.c_double()
    ok = lib.or_calibrate_profile(_p(r), r.shape[0], _p(lengths), len(lengths), samples, seed, _p(p), open_, ext,
                                  _p(scores), C.byref(lam), C.byref(k), C.byref(mu), threads or os.cpu_count() or 1)
    return ((lam.value, k.value, mu.value) if ok else None), scores[:samples].copy()


# ---- seed hits (seeds.c) -----------------------------------------------------------
SEED_STATS_FIELDS = ("windows", "windows_skipped", "kmers_generated", "windows_at_cap", "exact_seeds_added", "seeds",
                     "postings_visited", "seeds_over_occ_cap", "postings_skipped_occ")
_POSTING_DTYPE = np.dtype([("code", "<u8"), ("tid", "<u4"), ("tpos", "<u4")])
_SEED_PARAM_DTYPE = np.dtype([("kmer_score", "<i4"), ("max_kmers_per_pos", "<u4"), ("exact_seeds", "<u4"),
                              ("max_seed_occ", "<u4")])


def pattern_offsets(mask):
    """SeedPattern::from_mask (src/prefilter.rs:101-124): care offsets and span."""
    offs = [i for i, c in enumerate(mask) if c == "1"]
    return np.array(offs, dtype=np.uint32), len(mask)


def top_kmers(rows_w, thr, cap):
    """(codes, scores, capped): the first cap k-mers >= thr in canonical order."""
    r = _rows(rows_w)
    codes = np.zeros(max(cap, 1), dtype=np.uint64)
    scores = np.zeros(max(cap, 1), dtype=np.int32)
    n = C.c_uint32()
    capped = lib.or_top_kmers(_p(r), r.shape[0], thr, cap, _p(codes), _p(scores), C.byref(n))
    return codes[:n.value].copy(), scores[:n.value].copy(), bool(capped)


def top_kmers_dfs(rows_w, thr, cap):
    """(codes, scores, capped) of the reference's default depth-first generator (walk order)."""
    r = _rows(rows_w)
    codes = np.zeros(cap + 2, dtype=np.uint64)
    scores = np.zeros(cap + 2, dtype=np.int32)
    n = C.c_uint32()
    capped = lib.or_top_kmers_dfs(_p(r), r.shape[0], thr, cap, _p(codes), _p(scores), C.byref(n))
    return codes[:n.value].copy(), scores[:n.value].copy(), bool(capped)


class SeedIndex:
    """The CPU seed index of a target list (window_ok, src/index.rs:1059-1074)."""

    def __init__(self, arena: Arena, mask):
        self.offs, self.span = pattern_offsets(mask)
        self.w = len(self.offs)
        nt = len(arena.tgt_off) - 1
        n = lib.or_index_count(_p(arena.tgt), _p(arena.tgt_off), nt, _p(self.offs), self.w, self.span)
        self.post = np.zeros(max(int(n), 1), dtype=_POSTING_DTYPE)
        lib.or_index_build(_p(arena.tgt), _p(arena.tgt_off), nt, _p(self.offs), self.w, self.span, _p(self.post))
        self.n = int(n)


def seed_hits(rows, residues, index: SeedIndex, kmer_score, max_kmers_per_pos=512, exact_seeds=True,
              max_seed_occ=0):
    """One query's seed hits: (target, diag, qpos) arrays and the seed counters."""
    r = _rows(rows)
    res = None if residues is None else np.ascontiguousarray(residues, dtype=np.uint8)
    prm = np.zeros(1, dtype=_SEED_PARAM_DTYPE)
    prm["kmer_score"], prm["max_kmers_per_pos"] = kmer_score, max_kmers_per_pos
    prm["exact_seeds"], prm["max_seed_occ"] = int(bool(exact_seeds)), max_seed_occ
    st = np.zeros(len(SEED_STATS_FIELDS), dtype=np.uint64)
    args = (_p(r), _p(res), r.shape[0], _p(index.offs), index.w, index.span, _p(prm), _p(index.post), index.n, 0)
    n = int(lib.or_seed_hits(*args, None, None, None, 0, _p(st)))
    ht = np.zeros(max(n, 1), dtype=np.uint32)
    hd = np.zeros(max(n, 1), dtype=np.int32)
    hq = np.zeros(max(n, 1), dtype=np.uint32)
    lib.or_seed_hits(*args, _p(ht), _p(hd), _p(hq), n, _p(st))
    return ht[:n], hd[:n], hq[:n], {f: int(v) for f, v in zip(SEED_STATS_FIELDS, st)}


class DirectSeedIndex:
    """The CPU seed index as a direct table (counting sort over all windows)."""

    def __init__(self, tgt_arena, tgt_off, mask):
        self.offs, self.span = pattern_offsets(mask)
        self.w = len(self.offs)
        self.tgt = np.ascontiguousarray(tgt_arena, dtype=np.uint8)
        self.tgt_off = np.ascontiguousarray(tgt_off, dtype=np.uint64)
        nt = len(self.tgt_off) - 1
        self.off = np.zeros(20 ** self.w + 1, dtype=np.uint64)
        n = int(lib.or_index_direct_build(_p(self.tgt), _p(self.tgt_off), nt, _p(self.offs), self.w, self.span,
                                          _p(self.off), None, None, 1))
        self.post_t = np.zeros(max(n, 1), dtype=np.uint32)
        self.post_p = np.zeros(max(n, 1), dtype=np.uint32)
        lib.or_index_direct_build(_p(self.tgt), _p(self.tgt_off), nt, _p(self.offs), self.w, self.span,
                                  _p(self.off), _p(self.post_t), _p(self.post_p), 0)
        self.off[1:] = self.off[:-1].copy()
        self.off[0] = 0
        self.n = n


def prefilter_search(rows_list, residues, index: DirectSeedIndex, seed_p: dict, gate_p: dict, cap_per_query=4096,
                     threads=0):
    """Seeds + evidence + gate for each query over a DirectSeedIndex, queries in parallel:
    (candidates per query, truncated to cap_per_query; candidate counts; hit counts)."""
    arena = Arena(rows_list, [])
    nq = len(rows_list)
    res = None
    if residues is not None:
        res = np.ascontiguousarray(np.concatenate([np.asarray(r, np.uint8) for r in residues]))
    sp = np.zeros(1, dtype=_SEED_PARAM_DTYPE)
    for f in _SEED_PARAM_DTYPE.names:
        sp[f] = seed_p[f]
    gp = np.zeros(1, dtype=_PARAM_DTYPE)
    for f in PARAM_FIELDS:
        gp[f] = gate_p[f]
    out = np.zeros(nq * cap_per_query, dtype=CANDIDATE_DTYPE)
    n_cand = np.zeros(nq, dtype=np.uint64)
    n_hits = np.zeros(nq, dtype=np.uint64)
    lib.or_prefilter_search(_p(arena.rows), _p(arena.row_off), _p(arena.qlen), _p(res), nq, _p(index.tgt),
                            _p(index.tgt_off), _p(index.offs), index.w, index.span, _p(index.off), _p(index.post_t),
                            _p(index.post_p), _p(sp), _p(gp), _p(out), cap_per_query, _p(n_cand), _p(n_hits),
                            threads or os.cpu_count() or 1)
    cands = [out[q * cap_per_query:q * cap_per_query + min(int(n_cand[q]), cap_per_query)] for q in range(nq)]
    return cands, n_cand, n_hits
